// SIMPLE (reference: src/Solvers/Simple.h:33): one outer iteration per solve(timeStep).
#pragma once
#include "Solver.h"

class Simple : public Solver {
public:
    Simple(const Input& input, const HexaFvmMesh& mesh);
    double solve(double timeStep) override;

protected:
    Simple(const Input& input, const HexaFvmMesh& mesh, int kind);
};
