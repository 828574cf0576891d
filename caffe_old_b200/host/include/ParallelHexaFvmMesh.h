// Decomposed mesh (reference: src/Domains/HexaFvmMesh/ParallelHexaFvmMesh.h).  A case runs
// on one GPU without domain decomposition, so Parallel::nProcesses() is 1 and the module
// mains never construct this class; initialising one reports that.
#pragma once
#include "HexaFvmMesh.h"

class ParallelHexaFvmMesh : public HexaFvmMesh {
public:
    void initialize(const std::string& filename) override;
};
