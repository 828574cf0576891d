// Diffusion (reference: src/Solvers/Diffusion.h): scalar diffusion with unit diffusivity, one
// linear solve per solve(timeStep), on the device library's caffe_diffusion handle.  Reads
// Boundaries.<face>.type (fixed | zeroGradient | empty) and .refValue
// (PrimitiveBoundaryCondition.tpp:7-30), Solver.timeAccurate, and phi from
// case/initialConditions.info; optional LinearSolvers.diffusion (bicgstab_jacobi | cg_jacobi),
// tolerance and maxIterations for the solve.  solve() returns ||A x - b||_inf.
#pragma once
#include "Solver.h"

class Diffusion : public Solver {
public:
    Diffusion(const Input& input, const HexaFvmMesh& mesh);
    ~Diffusion() override;

    double solve(double timeStep) override;
    void displayUpdateMessage() override;
    // "phi", "gradPhi" (3 planes), "cc" (3 planes), "phiFaceI/J/K", ...
    std::vector<double> field(const std::string& name) const override;
    void setField(const std::string& name, const std::vector<double>& values) override;
    std::vector<std::pair<std::string, int>> tecplotFields() const override { return {{"phi", 1}, {"gradPhi", 3}}; }
    caffe_diffusion* diffusionHandle() const { return hd_; }

private:
    caffe_diffusion* hd_ = nullptr;
    double residual_ = 0.;
    int iters_ = 0;
    double relres_ = 0.;
};
