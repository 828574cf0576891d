// Ghost-cell immersed-boundary PISO with one sphere (reference: src/Solvers/IbPiso.h:33),
// ImmersedBoundaries.Sphere.{radius,center} from case/case.info.
#pragma once
#include "Piso.h"

class IbPiso : public Piso {
public:
    IbPiso(const Input& input, const HexaFvmMesh& mesh);
    double solve(double timeStep) override;
};
