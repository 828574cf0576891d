// PISO (reference: src/Solvers/Piso.h:6): inner iterations x pressure corrections per step.
#pragma once
#include "Simple.h"

class Piso : public Simple {
public:
    Piso(const Input& input, const HexaFvmMesh& mesh);
    double solve(double timeStep) override;

protected:
    Piso(const Input& input, const HexaFvmMesh& mesh, int kind);
};
