// Coupled (reference: src/Solvers/Coupled.h): momentum and continuity solved as one block
// system of 4 N unknowns each solve(timeStep), on the device library's caffe_coupled handle.
// Reads Boundaries.<face>, Solver.timeAccurate, Solver.numberOfInnerIterations (unsteady),
// Solver.relaxationFactorMomentum, Solver.rho and Solver.mu as the reference does
// (Coupled.cpp:5-34), plus the optional LinearSolvers.momentum / tolerance /
// absoluteTolerance / maxIterations keys for the block solve.  u and p start at zero.
#pragma once
#include "Solver.h"

class Coupled : public Solver {
public:
    Coupled(const Input& input, const HexaFvmMesh& mesh);
    ~Coupled() override;

    double solve(double timeStep) override;
    void displayUpdateMessage() override;
    // "u" (3 planes), "p", "d", "gradP" (3 planes), "h" (3 planes), "massFlowI/J/K" (faces),
    // "massFlow" (the cell array the reference registers for output; Coupled never sets it)
    std::vector<double> field(const std::string& name) const override;
    void setField(const std::string& name, const std::vector<double>& values) override;
    caffe_coupled* coupledHandle() const { return hc_; }

private:
    caffe_coupled* hc_ = nullptr;
    double continuity_ = 0.;
};
