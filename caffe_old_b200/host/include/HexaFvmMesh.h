// Structured hexahedral mesh of the host layer (reference:
// src/Domains/HexaFvmMesh/HexaFvmMesh.h).  It holds the node coordinates; the finite-volume
// metrics are computed from them on the GPU when a solver is constructed.  writeTec360
// writes the nodes and the cell-centred fields of the solver built on this mesh.
#pragma once
#include <fstream>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "Vector3D.h"

class Solver;

class HexaFvmMesh {
public:
    virtual ~HexaFvmMesh() = default;
    // Tecplot ASCII grid file in BLOCK packing (what hexaMesh writes; StructuredMesh.cpp:27-67)
    virtual void initialize(const std::string& filename);
    // trilinear box between 8 vertices (HexaMeshGen's construction) with the given cells
    virtual void initialize(const std::vector<Point3D>& vertices, int nCellsI, int nCellsJ, int nCellsK);
    virtual void initializeCartesianMesh(double xLength, double yLength, double zLength, int nCellsI, int nCellsJ, int nCellsK);
    virtual std::string meshStats();

    int nCellsI() const { return nI_; }
    int nCellsJ() const { return nJ_; }
    int nCellsK() const { return nK_; }
    int nCells() const { return nI_ * nJ_ * nK_; }
    // (nK+1)(nJ+1)(nI+1) nodes x 3 coordinates, i fastest
    const std::vector<double>& nodes() const { return nodes_; }
    const std::string& name() const { return name_; }

    void writeTec360(double time, const std::string& directory);
    // the solver whose fields writeTec360 writes (set by the solver's constructor)
    void attachSolver(const Solver* s) const { solver_ = s; }
    void detachSolver(const Solver* s) const { if (solver_ == s) solver_ = nullptr; }

protected:
    int nI_ = 0, nJ_ = 0, nK_ = 0;
    std::vector<double> nodes_;
    std::string name_ = "mesh";
    mutable const Solver* solver_ = nullptr;
    std::ofstream foutTec360_;
    std::vector<std::pair<std::string, int>> tecVars_;   // the variables of the open Tecplot file
};
