// Mesh input / output of the host layer.
#include "HexaFvmMesh.h"

#include <iomanip>
#include <sstream>

#include "Output.h"
#include "ParallelHexaFvmMesh.h"
#include "Solver.h"

namespace {

// node of a trilinear box between vertices v[0..7] (HexaMeshGen vertex order), s in [0,1]^3
Point3D box_node(const std::vector<Point3D>& v, double si, double sj, double sk) {
    // edges along k at the four corners, then along j on the west and east sides, then along i
    Point3D w0 = (v[4] - v[0]) * sk + v[0], w1 = (v[7] - v[3]) * sk + v[3];
    Point3D e0 = (v[5] - v[1]) * sk + v[1], e1 = (v[6] - v[2]) * sk + v[2];
    Point3D w = (w1 - w0) * sj + w0, e = (e1 - e0) * sj + e0;
    return (e - w) * si + w;
}

}  // namespace

void HexaFvmMesh::initialize(const std::string& filename) {
    std::ifstream f(filename);
    if (!f) Output::raiseException("HexaFvmMesh", "initialize", "cannot open mesh file \"" + filename + "\"");
    std::string line;
    int nodesI = 0, nodesJ = 0, nodesK = 0;
    // header: TITLE, VARIABLES, FILETYPE, ZONE I = .., J = .., K = .., DATAPACKING
    while (std::getline(f, line)) {
        if (line.rfind("TITLE", 0) == 0) {
            size_t a = line.find('"'), b = line.rfind('"');
            if (a != std::string::npos && b > a) name_ = line.substr(a + 1, b - a - 1);
        }
        if (line.rfind("ZONE", 0) == 0) {
            std::string t;
            for (char ch : line) t += (ch == ',' || ch == '=') ? ' ' : ch;
            std::istringstream in(t);
            std::string tok;
            while (in >> tok) {
                if (tok == "I") in >> nodesI;
                else if (tok == "J") in >> nodesJ;
                else if (tok == "K") in >> nodesK;
            }
        }
        if (line.rfind("DATAPACKING", 0) == 0) break;
    }
    if (nodesI < 2 || nodesJ < 2 || nodesK < 2)
        Output::raiseException("HexaFvmMesh", "initialize", "mesh file \"" + filename + "\" has no valid ZONE line");
    nI_ = nodesI - 1; nJ_ = nodesJ - 1; nK_ = nodesK - 1;
    const size_t n = (size_t)nodesI * nodesJ * nodesK;
    nodes_.assign(3 * n, 0.);
    for (int l = 0; l < 3; ++l)
        for (size_t q = 0; q < n; ++q)
            if (!(f >> nodes_[3 * q + l])) Output::raiseException("HexaFvmMesh", "initialize", "mesh file \"" + filename + "\" is truncated");
}

void HexaFvmMesh::initialize(const std::vector<Point3D>& vertices, int nCellsI, int nCellsJ, int nCellsK) {
    if (vertices.size() != 8 || nCellsI < 1 || nCellsJ < 1 || nCellsK < 1)
        Output::raiseException("HexaFvmMesh", "initialize", "need 8 vertices and at least one cell per direction");
    nI_ = nCellsI; nJ_ = nCellsJ; nK_ = nCellsK;
    nodes_.assign((size_t)3 * (nI_ + 1) * (nJ_ + 1) * (nK_ + 1), 0.);
    for (int k = 0; k <= nK_; ++k)
        for (int j = 0; j <= nJ_; ++j)
            for (int i = 0; i <= nI_; ++i) {
                Point3D p = box_node(vertices, double(i) / nI_, double(j) / nJ_, double(k) / nK_);
                size_t q = ((size_t)k * (nJ_ + 1) + j) * (nI_ + 1) + i;
                nodes_[3 * q] = p.x; nodes_[3 * q + 1] = p.y; nodes_[3 * q + 2] = p.z;
            }
}

void HexaFvmMesh::initializeCartesianMesh(double xLength, double yLength, double zLength, int nCellsI, int nCellsJ, int nCellsK) {
    std::vector<Point3D> v = {{0, 0, 0}, {xLength, 0, 0}, {xLength, yLength, 0}, {0, yLength, 0},
                              {0, 0, zLength}, {xLength, 0, zLength}, {xLength, yLength, zLength}, {0, yLength, zLength}};
    initialize(v, nCellsI, nCellsJ, nCellsK);
}

std::string HexaFvmMesh::meshStats() {
    std::ostringstream m;
    m << "Mesh \"" << name_ << "\": " << nI_ << " x " << nJ_ << " x " << nK_ << " = " << (long long)nI_ * nJ_ * nK_ << " cells";
    return m.str();
}

void HexaFvmMesh::writeTec360(double time, const std::string& directory) {
    if (!solver_) Output::raiseException("HexaFvmMesh", "writeTec360", "no solver has been built on this mesh");
    Output::print("HexaFvmMesh", "Writing data to Tec360 ASCII...");
    if (!foutTec360_.is_open()) {
        foutTec360_.open(directory + name_ + ".dat");
        if (!foutTec360_) Output::raiseException("HexaFvmMesh", "writeTec360", "cannot open \"" + directory + name_ + ".dat\"");
        foutTec360_ << std::setprecision(16);
    }
    // the fields the solver registers for output, scalars first, then vectors by component
    // (HexaFvmMesh.cpp:479-611)
    const auto vars = solver_->tecplotFields();
    if (tecVars_.empty()) {
        static const char* comp[3] = {"_x", "_y", "_z"};
        foutTec360_ << "TITLE = \"" << name_ << "\"\n" << "VARIABLES = \"x\", \"y\", \"z\"";
        for (const auto& v : vars)
            for (int c = 0; c < v.second; ++c) foutTec360_ << ", \"" << v.first << (v.second > 1 ? comp[c] : "") << "\"";
        foutTec360_ << "\n";
        tecVars_ = vars;
    }
    int nVar = 0;
    for (const auto& v : tecVars_) nVar += v.second;
    const size_t N = (size_t)nI_ * nJ_ * nK_;
    foutTec360_ << "ZONE T = \"" << time << "\", I = " << nI_ + 1 << ", J = " << nJ_ + 1 << ", K = " << nK_ + 1
                << ", DATAPACKING = BLOCK, VARLOCATION = ([4-" << 3 + nVar << "] = CELLCENTERED), SOLUTIONTIME = " << time << "\n";
    const size_t nn = nodes_.size() / 3;
    for (int l = 0; l < 3; ++l) {
        for (size_t q = 0; q < nn; ++q) foutTec360_ << nodes_[3 * q + l] << (q % 8 == 7 ? '\n' : ' ');
        foutTec360_ << '\n';
    }
    auto block = [&](const double* a) {
        for (size_t q = 0; q < N; ++q) foutTec360_ << a[q] << (q % 8 == 7 ? '\n' : ' ');
        foutTec360_ << '\n';
    };
    for (const auto& v : tecVars_) {
        const std::vector<double> a = solver_->field(v.first);
        for (int c = 0; c < v.second; ++c) block(a.data() + c * N);
    }
    foutTec360_.flush();
}

void ParallelHexaFvmMesh::initialize(const std::string& filename) {
    (void)filename;
    Output::raiseException("ParallelHexaFvmMesh", "initialize",
                           "a case runs on one GPU without domain decomposition; start one process per case");
}
