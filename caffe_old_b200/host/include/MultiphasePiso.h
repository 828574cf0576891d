// MultiphasePiso (reference: src/Solvers/MultiphasePiso.h, MultiphasePiso.cpp).  In the
// reference, solve() is Piso's step followed by computeAlpha, computeCurvature and the
// Courant and continuity computations (MultiphasePiso.cpp:27-47).  computeAlpha assembles an
// upwind advection system for the volume fraction into the momentum matrix's storage but
// never solves it (:58-111); the next step's momentum assembly overwrites every entry it
// wrote.  computeCurvature is empty (:113-116).  The volume fraction therefore never leaves
// its initial zero, and u and p evolve exactly as Piso's.  This class runs the Piso step on
// the device; the alpha, gradAlpha and k fields the reference adds to its Tecplot output
// (all zero) are not written.
#pragma once
#include "Piso.h"

class MultiphasePiso : public Piso {
public:
    MultiphasePiso(const Input& input, const HexaFvmMesh& mesh);
    double solve(double timeStep) override;
};
