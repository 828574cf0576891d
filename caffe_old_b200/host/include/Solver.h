// Solver interface of the host layer (reference: src/Solvers/Solver.h:12-39).  A solver owns
// one device handle of the B200 library (include/caffe_b200.h): mesh metrics, fields, both
// linear systems and the Krylov workspace stay in HBM; solve(timeStep) advances one outer
// iteration / time step on the GPU and returns the maximum continuity error.
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "HexaFvmMesh.h"
#include "Input.h"
#include "caffe_b200.h"

class Solver {
public:
    enum TimeDependent { ON, OFF };

    Solver(const Input& input, const HexaFvmMesh& mesh, int kind);
    virtual ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    virtual double solve(double timeStep) = 0;
    virtual void displayUpdateMessage();

    // host copies of device fields, component planes of nCells each: "u" (3 planes), "p",
    // "pCorr", "massFlowI/J/K", ... (names of caffe_dev_array)
    virtual std::vector<double> field(const std::string& name) const;
    virtual void setField(const std::string& name, const std::vector<double>& values);
    // the cell fields the solver registers for Tecplot output, in the order they are written,
    // with their component counts (Simple.cpp:57-59: p, massFlow, then the vector u)
    virtual std::vector<std::pair<std::string, int>> tecplotFields() const { return {{"p", 1}, {"massFlow", 1}, {"u", 3}}; }
    const caffe_step_stats& lastStats() const { return stats_; }
    const caffe_case& caseParameters() const { return case_; }
    caffe_dev* handle() const { return h_; }
    const HexaFvmMesh& mesh() const { return mesh_; }
    const char* className() const { return name_; }

    // the keys the solvers read from case/case.info, as the device library's case record
    static caffe_case caseFromInput(const Input& input, int kind);

protected:
    // a solver with its own device handle (Coupled, Diffusion): no flow-solver handle
    Solver(const HexaFvmMesh& mesh, const char* name);
    double step(double timeStep);
    const HexaFvmMesh& mesh_;
    caffe_case case_;
    caffe_dev* h_ = nullptr;
    caffe_step_stats stats_{};
    const char* name_ = "Solver";
};
