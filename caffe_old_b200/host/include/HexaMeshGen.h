// Structured mesh generator of the hexaMesh module (reference:
// src/Domains/HexaFvmMesh/HexaMeshGen.h): reads mesh/structuredMesh.info (MeshName,
// MetricConversion, Vertices.v1..v8, Resolution in nodes), fills the nodes by linear
// interpolation between opposite faces, and writes mesh/structuredMesh.dat.
#pragma once
#include <string>
#include <vector>

#include "Vector3D.h"

class HexaMeshGen {
public:
    void readFile(const std::string& directory);
    void generateMesh();
    void checkMesh();
    void writeMeshFile(const std::string& directory);
    const std::vector<Point3D>& nodes() const { return nodes_; }

private:
    std::string meshName_;
    double metricConversion_ = 1.;
    Point3D vertices_[8];
    int nNodes_[3] = {0, 0, 0};
    std::vector<Point3D> nodes_;
    Point3D& node(int i, int j, int k) { return nodes_[((size_t)k * nNodes_[1] + j) * nNodes_[0] + i]; }
};
