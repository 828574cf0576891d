// Structured mesh generation of the hexaMesh module (reference: HexaMeshGen.cpp): the nodes on
// the west and east faces come from linear interpolation along the k edges and then along j;
// interior nodes from linear interpolation along i between them.
#include "HexaMeshGen.h"

#include <cmath>
#include <fstream>
#include <iomanip>

#include "Input.h"
#include "Output.h"

void HexaMeshGen::readFile(const std::string& directory) {
    InfoTree t = InfoTree::readFile(directory + "structuredMesh.info");
    meshName_ = t.get<std::string>("MeshName");
    metricConversion_ = t.get<double>("MetricConversion");
    for (int i = 1; i <= 8; ++i) vertices_[i - 1] = metricConversion_ * std::stov(t.get<std::string>("Vertices.v" + std::to_string(i)));
    Vector3D res = std::stov(t.get<std::string>("Resolution"));
    for (int d = 0; d < 3; ++d) nNodes_[d] = (int)res(d);
    if (nNodes_[0] < 2 || nNodes_[1] < 2 || nNodes_[2] < 2) Output::raiseException("HexaMeshGen", "readFile", "resolution needs at least 2 nodes per direction");
    nodes_.assign((size_t)nNodes_[0] * nNodes_[1] * nNodes_[2], Point3D());
    Output::print("HexaMeshGen", "Successfully read file \"" + directory + "structuredMesh.info\".");
}

void HexaMeshGen::generateMesh() {
    const int uI = nNodes_[0] - 1, uJ = nNodes_[1] - 1, uK = nNodes_[2] - 1;
    for (int k = 0; k <= uK; ++k) {
        double s = double(k) / double(uK);
        node(0, 0, k) = (vertices_[4] - vertices_[0]) * s + vertices_[0];
        node(0, uJ, k) = (vertices_[7] - vertices_[3]) * s + vertices_[3];
        node(uI, 0, k) = (vertices_[5] - vertices_[1]) * s + vertices_[1];
        node(uI, uJ, k) = (vertices_[6] - vertices_[2]) * s + vertices_[2];
        Point3D west = node(0, uJ, k) - node(0, 0, k), east = node(uI, uJ, k) - node(uI, 0, k);
        for (int j = 0; j <= uJ; ++j) {
            double t = double(j) / double(uJ);
            node(0, j, k) = west * t + node(0, 0, k);
            node(uI, j, k) = east * t + node(uI, 0, k);
        }
    }
    for (int k = 0; k <= uK; ++k)
        for (int j = 0; j <= uJ; ++j) {
            Point3D d = node(uI, j, k) - node(0, j, k);
            for (int i = 0; i <= uI; ++i) node(i, j, k) = d * (double(i) / double(uI)) + node(0, j, k);
        }
    Output::print("HexaMeshGen", "Mesh generation complete.");
}

void HexaMeshGen::checkMesh() {
    // every face of the bounding hexahedron must be planar: the fourth vertex lies in the plane
    // of the other three (relative tolerance on the distance)
    static const int faces[6][4] = {{1, 2, 6, 5}, {0, 4, 7, 3}, {3, 7, 6, 2}, {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1}};
    for (const auto& f : faces) {
        Point3D a = vertices_[f[0]], b = vertices_[f[1]], c = vertices_[f[2]], d = vertices_[f[3]];
        Point3D u = b - a, v = c - a, w = d - a;
        Point3D n(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
        double nm = std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
        double wm = std::sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
        double dist = std::fabs(n.x * w.x + n.y * w.y + n.z * w.z) / (nm > 0. ? nm : 1.);
        if (dist > 1e-10 * (wm > 0. ? wm : 1.))
            Output::raiseException("HexaMeshGen", "checkMesh",
                                   "one or more surfaces of the mesh geometry is not planar, which is not currently supported.");
    }
}

void HexaMeshGen::writeMeshFile(const std::string& directory) {
    std::ofstream fout(directory + "structuredMesh.dat");
    if (!fout) Output::raiseException("HexaMeshGen", "writeMeshFile", "cannot write \"" + directory + "structuredMesh.dat\"");
    fout << std::setprecision(17);
    fout << "TITLE = \"" << meshName_ << "\"\n"
         << "VARIABLES = \"x\", \"y\", \"z\"\n"
         << "FILETYPE = GRID\n"
         << "ZONE I = " << nNodes_[0] << ", J = " << nNodes_[1] << ", K = " << nNodes_[2] << "\n"
         << "DATAPACKING = BLOCK\n";
    for (int l = 0; l < 3; ++l)
        for (int k = 0; k < nNodes_[2]; ++k)
            for (int j = 0; j < nNodes_[1]; ++j) {
                for (int i = 0; i < nNodes_[0]; ++i) fout << node(i, j, k)(l) << " ";
                fout << "\n";
            }
    Output::print("HexaMeshGen", "Finished writing mesh file.");
}
