// TEST INFRASTRUCTURE ONLY -- the CPU oracle.
//
// A plain C++ restatement of CAFFE's per-iteration finite-volume hot path
// (SIMPLE / PISO / IB-PISO on a structured hexahedral mesh), used by tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker of the
// CUDA library.  Nothing in the product links or calls this file.
//
// Every routine cites the reference file:line it restates (paths are relative to
// the CAFFE_old project root).  Floating-point expressions keep the reference's
// operand order, association and its Vector3D conventions (vector / scalar is a
// multiply by the reciprocal, Vector3D.cpp:98-107; tensor / scalar is a true
// divide, Tensor3D.cpp:155-168), so that everything outside the Krylov solves is
// bit-for-bit what the reference computes.  Build with -ffp-contract=off.
//
// The reference delegates every linear solve to PETSc (KSPBCGS + PCSOR,
// SparseMatrix.cpp:86-106); PETSc is an unvendored, unpinned dependency.  The
// Krylov solvers below restate the published algorithms instead:
//   * BiCGStab, van der Vorst (1992), left-preconditioned with one symmetric
//     Gauss-Seidel sweep (SOR omega = 1, its = lits = 1, zero initial guess) and
//     tested on the preconditioned residual norm -- the configuration the
//     reference selects (SparseMatrix.cpp:95-100, defaults SparseMatrix.h:40);
//   * BiCGStab, right-preconditioned with Jacobi, tested on the true residual;
//   * CG, Hestenes-Stiefel, Jacobi-preconditioned, tested on the true residual.
// Reductions are summed in fixed 2048-row chunks and then in chunk order, so the
// result does not depend on the OpenMP thread count.
//
// Pinning.  The geometry (hexahedron volume and centroid, face area, centroid and
// vector, point-in-cell test, sphere intersection), the mesh metric arrays (D_f,
// c_f), the velocity-gradient tensor, the cell storage order and the
// immersed-boundary geometry (solid cells, ghost cells, image-point stencils) are
// pinned bit for bit against the reference's
// own Geometry / Sphere / Vector3D / Tensor3D / Array3D code, compiled where it lies
// (tests/test_oracle_pinned_reference.py; tests/golden/reference_geometry.npz keeps
// the reference's outputs).  The rest -- the flow phases, the trilinear weights and
// the Krylov solves -- is parity unpinned: the reference needs MPI, PETSc, Boost and
// LAPACKE to build, none of which is present, so it follows the reference's source
// line by line and is checked by the known-answer tests only.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ----------------------------------------------------------------------------
// Small value types (Vector3D.cpp, Tensor3D.cpp)
// ----------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};
static inline V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }   // Vector3D.cpp:71-78
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }   // :80-87
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }                        // :119-122
static inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }     // :89-96
static inline V3 operator*(double s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }     // :129-132
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
// Vector3D::operator/= multiplies by the reciprocal (Vector3D.cpp:98-107).
static inline V3 operator/(V3 a, double s) { double r = 1. / s; return v3(a.x * r, a.y * r, a.z * r); }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }      // :171-174
static inline V3 cross(V3 u, V3 v) {                                                      // :183-188
    return v3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
static inline double mag(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }  // :55-58
static inline V3 unitv(V3 a) { double inv = 1. / mag(a); return v3(inv * a.x, inv * a.y, inv * a.z); } // :60-64
static inline double comp(const V3& a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }
static inline double& comp(V3& a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }

struct T3 {  // Tensor3D, row-major xx xy xz / yx yy yz / zx zy zz
    double m[9];
};
static inline T3 tensor(V3 u, V3 v) {  // Vector3D.cpp:176-181
    T3 t;
    t.m[0] = u.x * v.x; t.m[1] = u.x * v.y; t.m[2] = u.x * v.z;
    t.m[3] = u.y * v.x; t.m[4] = u.y * v.y; t.m[5] = u.y * v.z;
    t.m[6] = u.z * v.x; t.m[7] = u.z * v.y; t.m[8] = u.z * v.z;
    return t;
}
static inline T3 tadd(T3 a, const T3& b) { for (int q = 0; q < 9; ++q) a.m[q] += b.m[q]; return a; }
static inline T3 tdiv(T3 a, double s) { for (int q = 0; q < 9; ++q) a.m[q] /= s; return a; }  // Tensor3D.cpp:155-168
static inline T3 tscale(T3 a, double s) { for (int q = 0; q < 9; ++q) a.m[q] *= s; return a; }
static inline T3 operator*(double s, T3 a) { return tscale(a, s); }
static inline T3 operator+(T3 a, const T3& b) { return tadd(a, b); }
static inline V3 tdot(const T3& t, V3 v) {  // Tensor3D.cpp:223-228
    return v3(t.m[0] * v.x + t.m[1] * v.y + t.m[2] * v.z,
              t.m[3] * v.x + t.m[4] * v.y + t.m[5] * v.z,
              t.m[6] * v.x + t.m[7] * v.y + t.m[8] * v.z);
}

static inline V3 zero3() { return v3(0., 0., 0.); }
template <class T> static inline T zeroOf();
template <> inline double zeroOf<double>() { return 0.; }
template <> inline V3 zeroOf<V3>() { return zero3(); }
template <> inline T3 zeroOf<T3>() { T3 t; for (int q = 0; q < 9; ++q) t.m[q] = 0.; return t; }
template <> inline int zeroOf<int>() { return 0; }

// ----------------------------------------------------------------------------
// Geometry (Geometry.cpp)
// ----------------------------------------------------------------------------
static double quadArea(const V3* p) {  // Geometry.cpp:5-12
    V3 r01 = p[1] - p[0], r02 = p[2] - p[0], r03 = p[3] - p[0];
    return 0.5 * (mag(cross(r02, r01)) + mag(cross(r03, r02)));
}
static V3 quadCentroid(const V3* p) {  // Geometry.cpp:14-20
    V3 d1 = p[0] + 0.5 * (p[2] - p[0]);
    V3 d2 = p[1] + 0.5 * (p[3] - p[1]);
    return d1 + 0.5 * (d2 - d1);
}
static V3 quadNormalIb(const V3* p) {  // Geometry.cpp:22-25 (as written: the same cross product twice)
    return 0.5 * (cross(p[1] - p[0], p[2] - p[0]) + cross(p[1] - p[0], p[2] - p[0]));
}
static double hexVolume(const V3* p) {  // Geometry.cpp:40-59 (Pletcher, Tannehill, Anderson)
    V3 r16 = p[6] - p[1], r25 = p[5] - p[2];
    V3 s1265 = 0.5 * cross(r16, r25);
    V3 r57 = p[7] - p[5], r64 = p[4] - p[6];
    V3 s5674 = 0.5 * cross(r57, r64);
    V3 r27 = p[7] - p[2], r36 = p[6] - p[3];
    V3 s2376 = 0.5 * cross(r27, r36);
    return std::fabs(dot(s1265 + s5674 + s2376, p[6] - p[0]) / 3.);
}
static double tetVolume(const V3* p) {  // Geometry.cpp:258-267
    V3 a = p[1] - p[0], b = p[2] - p[0], c = p[3] - p[0];
    return std::fabs(dot(a, cross(b, c))) / 6.;
}
static V3 tetCentroid(const V3* p) {  // Geometry.cpp:269-277
    V3 s = zero3();
    for (int i = 0; i < 4; ++i) s += p[i];
    return 0.25 * s;
}
static V3 hexCentroid(const V3* p) {  // Geometry.cpp:61-109 (5-tetrahedron split)
    static const int tv[5][4] = {{4, 3, 6, 7}, {4, 1, 6, 5}, {4, 1, 6, 3}, {4, 0, 1, 3}, {3, 1, 2, 6}};
    V3 tc[5];
    double vol[5], sumV = 0.;
    for (int t = 0; t < 5; ++t) {
        V3 q[4];
        for (int m = 0; m < 4; ++m) q[m] = p[tv[t][m]];
        tc[t] = tetCentroid(q);
        vol[t] = tetVolume(q);
        sumV += vol[t];
    }
    V3 c = zero3();
    for (int t = 0; t < 5; ++t) c += vol[t] * tc[t];
    return c / sumV;
}
static bool insideHex(V3 pt, const V3* p) {  // Geometry.cpp:178-256
    static const int fv[6][4] = {{1, 2, 6, 5}, {0, 4, 7, 3}, {2, 3, 7, 6}, {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1}};
    for (int f = 0; f < 6; ++f) {
        V3 q[4];
        for (int m = 0; m < 4; ++m) q[m] = p[fv[f][m]];
        V3 xc = quadCentroid(q), n = quadNormalIb(q);
        if (dot(xc - pt, n) < 0.) return false;
    }
    return true;
}

// 8x8 solve for the trilinear image-point weights beta = m(x_IP)^T M^-1
// (Interpolation.cpp:135-180).  The reference inverts M with LAPACK getrf/getri;
// here M^T beta = m is solved by Gaussian elimination with partial pivoting.
static void trilinearCoeffs(const V3* pts, V3 ip, double* beta) {
    double A[8][9];
    double mrow[8][8];
    for (int i = 0; i < 8; ++i) {
        double x = pts[i].x, y = pts[i].y, z = pts[i].z;
        mrow[i][0] = 1.; mrow[i][1] = x * y * z; mrow[i][2] = x * y; mrow[i][3] = y * z;
        mrow[i][4] = x * z; mrow[i][5] = x; mrow[i][6] = y; mrow[i][7] = z;
    }
    double x = ip.x, y = ip.y, z = ip.z;
    double rhs[8] = {1., x * y * z, x * y, y * z, x * z, x, y, z};
    for (int r = 0; r < 8; ++r) {           // row r of M^T = column r of M
        for (int c = 0; c < 8; ++c) A[r][c] = mrow[c][r];
        A[r][8] = rhs[r];
    }
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        double best = std::fabs(A[c][c]);
        for (int r = c + 1; r < 8; ++r)
            if (std::fabs(A[r][c]) > best) { best = std::fabs(A[r][c]); piv = r; }
        if (piv != c)
            for (int q = 0; q < 9; ++q) std::swap(A[c][q], A[piv][q]);
        double inv = 1. / A[c][c];
        for (int r = c + 1; r < 8; ++r) {
            double f = A[r][c] * inv;
            if (f == 0.) continue;
            for (int q = c; q < 9; ++q) A[r][q] = A[r][q] - f * A[c][q];
        }
    }
    for (int r = 7; r >= 0; --r) {
        double s = A[r][8];
        for (int q = r + 1; q < 8; ++q) s = s - A[r][q] * beta[q];
        beta[r] = s / A[r][r];
    }
}

// ----------------------------------------------------------------------------
// Mesh (HexaFvmMesh.cpp, StructuredMesh.cpp)
// ----------------------------------------------------------------------------
struct Mesh {
    int nI, nJ, nK;           // cells
    std::vector<V3> nodes;    // (nI+1)(nJ+1)(nK+1), i fastest
    std::vector<V3> cc;       // cell centroids
    std::vector<double> vol;
    std::vector<V3> fcI, fcJ, fcK;   // face centroids
    std::vector<V3> fnI, fnJ, fnK;   // face area-normal vectors (+i/+j/+k)
    std::vector<V3> c2cI, c2cJ, c2cK;
    std::vector<V3> c2f[6];   // cell-to-face vectors E W N S T B
    std::vector<double> d[6]; // |S|^2 / (S.r)
    std::vector<V3> cvec[6];  // non-orthogonal vectors S - r|S|^2/(S.r)
    std::vector<double> g[6]; // volume weights

    size_t N() const { return (size_t)nI * nJ * nK; }
    int cid(int i, int j, int k) const { return (k * nJ + j) * nI + i; }
    int nid(int i, int j, int k) const { return (k * (nJ + 1) + j) * (nI + 1) + i; }
    int fiI(int i, int j, int k) const { return (k * nJ + j) * (nI + 1) + i; }
    int fiJ(int i, int j, int k) const { return (k * (nJ + 1) + j) * nI + i; }
    int fiK(int i, int j, int k) const { return (k * nJ + j) * nI + i; }
    int uI() const { return nI - 1; }
    int uJ() const { return nJ - 1; }
    int uK() const { return nK - 1; }

    V3 SE(int i, int j, int k) const { return fnI[fiI(i + 1, j, k)]; }   // HexaFvmMesh.h:79-84
    V3 SW(int i, int j, int k) const { return -fnI[fiI(i, j, k)]; }
    V3 SN(int i, int j, int k) const { return fnJ[fiJ(i, j + 1, k)]; }
    V3 SS(int i, int j, int k) const { return -fnJ[fiJ(i, j, k)]; }
    V3 ST(int i, int j, int k) const { return fnK[fiK(i, j, k + 1)]; }
    V3 SB(int i, int j, int k) const { return -fnK[fiK(i, j, k)]; }
    V3 S(int f, int i, int j, int k) const {
        switch (f) { case 0: return SE(i, j, k); case 1: return SW(i, j, k); case 2: return SN(i, j, k);
                     case 3: return SS(i, j, k); case 4: return ST(i, j, k); default: return SB(i, j, k); }
    }
    // HexaFvmMesh.cpp:218-294 (single block, no neighbouring meshes)
    V3 rCell(int f, int i, int j, int k) const {
        int c = cid(i, j, k);
        switch (f) {
            case 0: return i == uI() ? c2f[0][c] : c2cI[(k * nJ + j) * (nI - 1) + i];
            case 1: return i == 0 ? c2f[1][c] : -c2cI[(k * nJ + j) * (nI - 1) + i - 1];
            case 2: return j == uJ() ? c2f[2][c] : c2cJ[(k * (nJ - 1) + j) * nI + i];
            case 3: return j == 0 ? c2f[3][c] : -c2cJ[(k * (nJ - 1) + j - 1) * nI + i];
            case 4: return k == uK() ? c2f[4][c] : c2cK[(k * nJ + j) * nI + i];
            default: return k == 0 ? c2f[5][c] : -c2cK[((k - 1) * nJ + j) * nI + i];
        }
    }

    void build(const double* xyz, int nNI, int nNJ, int nNK) {
        nI = nNI - 1; nJ = nNJ - 1; nK = nNK - 1;
        if (nI < 1 || nJ < 1 || nK < 1) throw std::runtime_error("mesh needs at least one cell per direction");
        nodes.resize((size_t)nNI * nNJ * nNK);
        for (size_t q = 0; q < nodes.size(); ++q) nodes[q] = v3(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]);
        size_t n = N();
        cc.resize(n); vol.resize(n);
        // initializeCells, HexaFvmMesh.cpp:626-655
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    V3 p[8] = {nodes[nid(i, j, k)], nodes[nid(i + 1, j, k)], nodes[nid(i + 1, j + 1, k)], nodes[nid(i, j + 1, k)],
                               nodes[nid(i, j, k + 1)], nodes[nid(i + 1, j, k + 1)], nodes[nid(i + 1, j + 1, k + 1)], nodes[nid(i, j + 1, k + 1)]};
                    cc[cid(i, j, k)] = hexCentroid(p);
                    vol[cid(i, j, k)] = hexVolume(p);
                }
        // initializeCellToCellParameters, :657-697
        c2cI.assign((size_t)(nI - 1) * nJ * nK, zero3());
        c2cJ.assign((size_t)nI * (nJ - 1) * nK, zero3());
        c2cK.assign((size_t)nI * nJ * (nK - 1), zero3());
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    if (i < nI - 1) c2cI[(k * nJ + j) * (nI - 1) + i] = cc[cid(i + 1, j, k)] - cc[cid(i, j, k)];
                    if (j < nJ - 1) c2cJ[(k * (nJ - 1) + j) * nI + i] = cc[cid(i, j + 1, k)] - cc[cid(i, j, k)];
                    if (k < nK - 1) c2cK[(k * nJ + j) * nI + i] = cc[cid(i, j, k + 1)] - cc[cid(i, j, k)];
                }
        // initializeFaces, :699-789
        fcI.resize((size_t)(nI + 1) * nJ * nK); fnI.resize(fcI.size());
        fcJ.resize((size_t)nI * (nJ + 1) * nK); fnJ.resize(fcJ.size());
        fcK.resize((size_t)nI * nJ * (nK + 1)); fnK.resize(fcK.size());
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i <= nI; ++i) {
                    V3 p[4] = {nodes[nid(i, j, k)], nodes[nid(i, j + 1, k)], nodes[nid(i, j + 1, k + 1)], nodes[nid(i, j, k + 1)]};
                    V3 t = unitv(cross(p[1] - p[0], p[2] - p[0]));
                    double a = quadArea(p);
                    fcI[fiI(i, j, k)] = quadCentroid(p);
                    fnI[fiI(i, j, k)] = t * a;
                }
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j <= nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    V3 p[4] = {nodes[nid(i, j, k)], nodes[nid(i, j, k + 1)], nodes[nid(i + 1, j, k + 1)], nodes[nid(i + 1, j, k)]};
                    V3 t = unitv(cross(p[1] - p[0], p[2] - p[0]));
                    double a = quadArea(p);
                    fcJ[fiJ(i, j, k)] = quadCentroid(p);
                    fnJ[fiJ(i, j, k)] = t * a;
                }
        for (int k = 0; k <= nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    V3 p[4] = {nodes[nid(i, j, k)], nodes[nid(i + 1, j, k)], nodes[nid(i + 1, j + 1, k)], nodes[nid(i, j + 1, k)]};
                    V3 t = unitv(cross(p[1] - p[0], p[2] - p[0]));
                    double a = quadArea(p);
                    fcK[fiK(i, j, k)] = quadCentroid(p);
                    fnK[fiK(i, j, k)] = t * a;
                }
        // initializeCellToFaceParameters, :791-839
        for (int f = 0; f < 6; ++f) c2f[f].resize(n);
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    int c = cid(i, j, k);
                    c2f[0][c] = fcI[fiI(i + 1, j, k)] - cc[c];
                    c2f[1][c] = fcI[fiI(i, j, k)] - cc[c];
                    c2f[2][c] = fcJ[fiJ(i, j + 1, k)] - cc[c];
                    c2f[3][c] = fcJ[fiJ(i, j, k)] - cc[c];
                    c2f[4][c] = fcK[fiK(i, j, k + 1)] - cc[c];
                    c2f[5][c] = fcK[fiK(i, j, k)] - cc[c];
                }
        // computeMeshMetrics, :841-918
        for (int f = 0; f < 6; ++f) { d[f].resize(n); cvec[f].resize(n); g[f].resize(n); }
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    int c = cid(i, j, k);
                    for (int f = 0; f < 6; ++f) {
                        V3 s = S(f, i, j, k), r = rCell(f, i, j, k);
                        d[f][c] = dot(s, s) / dot(s, r);
                        cvec[f][c] = s - (r * dot(s, s)) / dot(s, r);
                    }
                    g[0][c] = i < uI() ? vol[cid(i + 1, j, k)] / (vol[cid(i + 1, j, k)] + vol[c]) : 0.;
                    g[1][c] = i > 0 ? vol[cid(i - 1, j, k)] / (vol[cid(i - 1, j, k)] + vol[c]) : 0.;
                    g[2][c] = j < uJ() ? vol[cid(i, j + 1, k)] / (vol[cid(i, j + 1, k)] + vol[c]) : 0.;
                    g[3][c] = j > 0 ? vol[cid(i, j - 1, k)] / (vol[cid(i, j - 1, k)] + vol[c]) : 0.;
                    g[4][c] = k < uK() ? vol[cid(i, j, k + 1)] / (vol[cid(i, j, k + 1)] + vol[c]) : 0.;
                    g[5][c] = k > 0 ? vol[cid(i, j, k - 1)] / (vol[cid(i, j, k - 1)] + vol[c]) : 0.;
                }
    }

    std::vector<V3> hexOfNodes(int i, int j, int k) const {
        return {nodes[nid(i, j, k)], nodes[nid(i + 1, j, k)], nodes[nid(i + 1, j + 1, k)], nodes[nid(i, j + 1, k)],
                nodes[nid(i, j, k + 1)], nodes[nid(i + 1, j, k + 1)], nodes[nid(i + 1, j + 1, k + 1)], nodes[nid(i, j + 1, k + 1)]};
    }
    // HexaFvmMesh::locateCell (:345-376) returns the first cell in k-j-i order whose
    // hexahedron contains the point.  In a valid mesh only cells next to the one that
    // contains the point can also contain it, so the search starts in a window around
    // a hint and falls back to the full scan the reference does.
    bool locateCell(V3 pt, int hi, int hj, int hk, int& ri, int& rj, int& rk) const {
        const int w = 5;
        int k0 = std::max(0, hk - w), k1 = std::min(nK - 1, hk + w);
        int j0 = std::max(0, hj - w), j1 = std::min(nJ - 1, hj + w);
        int i0 = std::max(0, hi - w), i1 = std::min(nI - 1, hi + w);
        bool found = false;
        for (int k = k0; k <= k1 && !found; ++k)
            for (int j = j0; j <= j1 && !found; ++j)
                for (int i = i0; i <= i1 && !found; ++i) {
                    std::vector<V3> p = hexOfNodes(i, j, k);
                    if (insideHex(pt, p.data())) { ri = i; rj = j; rk = k; found = true; }
                }
        if (found) {
            // any earlier (k-j-i order) containing cell would be a neighbour of this one
            int bi = ri, bj = rj, bk = rk;
            for (int k = std::max(0, bk - 1); k <= std::min(nK - 1, bk + 1); ++k)
                for (int j = std::max(0, bj - 1); j <= std::min(nJ - 1, bj + 1); ++j)
                    for (int i = std::max(0, bi - 1); i <= std::min(nI - 1, bi + 1); ++i) {
                        if (cid(i, j, k) >= cid(ri, rj, rk)) continue;
                        std::vector<V3> p = hexOfNodes(i, j, k);
                        if (insideHex(pt, p.data())) { ri = i; rj = j; rk = k; }
                    }
            return true;
        }
        for (int k = 0; k < nK; ++k)
            for (int j = 0; j < nJ; ++j)
                for (int i = 0; i < nI; ++i) {
                    std::vector<V3> p = hexOfNodes(i, j, k);
                    if (insideHex(pt, p.data())) { ri = i; rj = j; rk = k; return true; }
                }
        return false;
    }
    // HexaFvmMesh::locateEnclosingCells (:378-418)
    bool locateEnclosingCells(V3 pt, int hi, int hj, int hk, int* ii, int* jj, int* kk) const {
        int i0, j0, k0;
        if (!locateCell(pt, hi, hj, hk, i0, j0, k0)) return false;
        for (int k = k0 - 1; k <= k0; ++k)
            for (int j = j0 - 1; j <= j0; ++j)
                for (int i = i0 - 1; i <= i0; ++i) {
                    if (i < 0 || j < 0 || k < 0 || i + 1 >= nI || j + 1 >= nJ || k + 1 >= nK)
                        return false;  // Array3D bounds check throws in the reference (Array3D.tpp:41-48)
                    V3 p[8] = {cc[cid(i, j, k)], cc[cid(i + 1, j, k)], cc[cid(i + 1, j + 1, k)], cc[cid(i, j + 1, k)],
                               cc[cid(i, j, k + 1)], cc[cid(i + 1, j, k + 1)], cc[cid(i + 1, j + 1, k + 1)], cc[cid(i, j + 1, k + 1)]};
                    if (insideHex(pt, p)) {
                        const int di[8] = {0, 1, 1, 0, 0, 1, 1, 0}, dj[8] = {0, 0, 1, 1, 0, 0, 1, 1}, dk[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                        for (int m = 0; m < 8; ++m) { ii[m] = i + di[m]; jj[m] = j + dj[m]; kk[m] = k + dk[m]; }
                        return true;
                    }
                }
        return false;
    }
};

// ----------------------------------------------------------------------------
// Field with cell, face and boundary-patch storage (Field.h, Field.tpp)
// ----------------------------------------------------------------------------
template <class T>
struct Field {
    int nI = 0, nJ = 0, nK = 0;
    std::vector<T> c, fI, fJ, fK;
    std::vector<T> patch[6];  // E,W: (j,k)  N,S: (i,k)  T,B: (i,j)

    void allocate(int a, int b, int d) {  // Field.tpp:223-241
        nI = a; nJ = b; nK = d;
        T z = zeroOf<T>();
        c.assign((size_t)nI * nJ * nK, z);
        fI.assign((size_t)(nI + 1) * nJ * nK, z);
        fJ.assign((size_t)nI * (nJ + 1) * nK, z);
        fK.assign((size_t)nI * nJ * (nK + 1), z);
        patch[0].assign((size_t)nJ * nK, z); patch[1].assign((size_t)nJ * nK, z);
        patch[2].assign((size_t)nI * nK, z); patch[3].assign((size_t)nI * nK, z);
        patch[4].assign((size_t)nI * nJ, z); patch[5].assign((size_t)nI * nJ, z);
    }
    int cid(int i, int j, int k) const { return (k * nJ + j) * nI + i; }
    // Field<T>::operator()(i,j,k) with the boundary-patch mapping, Field.tpp:243-282
    T& at(int i, int j, int k) {
        if (i >= 0 && j >= 0 && k >= 0 && i < nI && j < nJ && k < nK) return c[cid(i, j, k)];
        if (i < 0) return patch[1][k * nJ + j];
        if (i >= nI) return patch[0][k * nJ + j];
        if (j < 0) return patch[3][k * nI + i];
        if (j >= nJ) return patch[2][k * nI + i];
        if (k < 0) return patch[5][j * nI + i];
        return patch[4][j * nI + i];
    }
    T& faceE(int i, int j, int k) { return fI[(k * nJ + j) * (nI + 1) + i + 1]; }   // Field.h:96-101
    T& faceW(int i, int j, int k) { return fI[(k * nJ + j) * (nI + 1) + i]; }
    T& faceN(int i, int j, int k) { return fJ[(k * (nJ + 1) + j + 1) * nI + i]; }
    T& faceS(int i, int j, int k) { return fJ[(k * (nJ + 1) + j) * nI + i]; }
    T& faceT(int i, int j, int k) { return fK[((k + 1) * nJ + j) * nI + i]; }
    T& faceB(int i, int j, int k) { return fK[(k * nJ + j) * nI + i]; }
    T& face(int f, int i, int j, int k) {
        switch (f) { case 0: return faceE(i, j, k); case 1: return faceW(i, j, k); case 2: return faceN(i, j, k);
                     case 3: return faceS(i, j, k); case 4: return faceT(i, j, k); default: return faceB(i, j, k); }
    }
    // setXFacesFromPatch, Field.tpp:434-516
    void facesFromPatch(int f) {
        if (f == 0 || f == 1) { int ii = f == 0 ? nI : 0;
            for (int k = 0; k < nK; ++k) for (int j = 0; j < nJ; ++j) fI[(k * nJ + j) * (nI + 1) + ii] = patch[f][k * nJ + j]; }
        else if (f == 2 || f == 3) { int jj = f == 2 ? nJ : 0;
            for (int k = 0; k < nK; ++k) for (int i = 0; i < nI; ++i) fJ[(k * (nJ + 1) + jj) * nI + i] = patch[f][k * nI + i]; }
        else { int kk = f == 4 ? nK : 0;
            for (int j = 0; j < nJ; ++j) for (int i = 0; i < nI; ++i) fK[(kk * nJ + j) * nI + i] = patch[f][j * nI + i]; }
    }
    // setZeroGradientBoundaryX, Field.tpp:518-558
    void zeroGradient(int f) {
        if (f == 0 || f == 1) { int ii = f == 0 ? nI - 1 : 0;
            for (int k = 0; k < nK; ++k) for (int j = 0; j < nJ; ++j) patch[f][k * nJ + j] = c[cid(ii, j, k)]; }
        else if (f == 2 || f == 3) { int jj = f == 2 ? nJ - 1 : 0;
            for (int k = 0; k < nK; ++k) for (int i = 0; i < nI; ++i) patch[f][k * nI + i] = c[cid(i, jj, k)]; }
        else { int kk = f == 4 ? nK - 1 : 0;
            for (int j = 0; j < nJ; ++j) for (int i = 0; i < nI; ++i) patch[f][j * nI + i] = c[cid(i, j, kk)]; }
        facesFromPatch(f);
    }
};

enum PType { P_FIXED = 0, P_ZERO_GRADIENT = 1, P_EMPTY = 2 };
enum FlowType { F_INLET = 0, F_OUTLET = 1, F_WALL = 2, F_EMPTY = 3, F_ZERO_GRADIENT = 4 };

// PrimitiveBoundaryCondition<T> (PrimitiveBoundaryCondition.tpp)
template <class T>
struct BC {
    PType type[6];
    T ref[6];
    Field<T>* fld = nullptr;
    int uI, uJ, uK;

    // PrimitiveBoundaryCondition(Field&), .tpp:32-40.  The reference leaves refValues_
    // uninitialised for double; they are taken as zero here (Vector3D's are zero).
    void init(Field<T>* f) {
        fld = f; uI = f->nI - 1; uJ = f->nJ - 1; uK = f->nK - 1;
        for (int i = 0; i < 6; ++i) { type[i] = P_FIXED; ref[i] = zeroOf<T>(); }
    }
    void setFixedBoundaries() {  // .tpp:284-294
        for (int f = 0; f < 6; ++f) {
            std::fill(fld->patch[f].begin(), fld->patch[f].end(), ref[f]);
            fld->facesFromPatch(f);
        }
    }
    void changeType(int i, PType t, T r) {  // .tpp:257-265
        type[i] = t; ref[i] = r;
        if (t == P_FIXED) setFixedBoundaries();
    }
    void setBoundaries() {  // .tpp:43-142 (no PARALLEL faces: one block)
        for (int f = 0; f < 6; ++f)
            if (type[f] == P_ZERO_GRADIENT || type[f] == P_EMPTY) fld->zeroGradient(f);
    }
    // .tpp:145-255
    void setImplicit(int i, int j, int k, double* a, T& b) {
        if (i == uI) { if (type[0] == P_FIXED) b -= a[1] * fld->patch[0][k * fld->nJ + j]; else { a[0] += a[1]; a[1] = 0.; } }
        if (i == 0) { if (type[1] == P_FIXED) b -= a[2] * fld->patch[1][k * fld->nJ + j]; else { a[0] += a[2]; a[2] = 0.; } }
        if (j == uJ) { if (type[2] == P_FIXED) b -= a[3] * fld->patch[2][k * fld->nI + i]; else { a[0] += a[3]; a[3] = 0.; } }
        if (j == 0) { if (type[3] == P_FIXED) b -= a[4] * fld->patch[3][k * fld->nI + i]; else { a[0] += a[4]; a[4] = 0.; } }
        if (k == uK) { if (type[4] == P_FIXED) b -= a[5] * fld->patch[4][j * fld->nI + i]; else { a[0] += a[5]; a[5] = 0.; } }
        if (k == 0) { if (type[5] == P_FIXED) b -= a[6] * fld->patch[5][j * fld->nI + i]; else { a[0] += a[6]; a[6] = 0.; } }
    }
};

// FvScheme::interpolateInteriorFaces, VOLUME_WEIGHTED branch (FvScheme.tpp:12-40), one block.
template <class T>
static void interpolateInteriorFaces(const Mesh& m, Field<T>& fl) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < m.nK; ++k)
        for (int j = 0; j < m.nJ; ++j)
            for (int i = 0; i < m.nI; ++i) {
                int c = m.cid(i, j, k);
                if (i < m.uI()) fl.faceE(i, j, k) = m.g[0][c] * fl.at(i, j, k) + (1. - m.g[0][c]) * fl.at(i + 1, j, k);
                if (j < m.uJ()) fl.faceN(i, j, k) = m.g[2][c] * fl.at(i, j, k) + (1. - m.g[2][c]) * fl.at(i, j + 1, k);
                if (k < m.uK()) fl.faceT(i, j, k) = m.g[4][c] * fl.at(i, j, k) + (1. - m.g[4][c]) * fl.at(i, j, k + 1);
            }
}
static V3 gradDT(const Mesh& m, Field<double>& fl, int i, int j, int k) {  // FvScalarScheme.cpp:48-66
    V3 s = fl.faceE(i, j, k) * m.SE(i, j, k);
    s += fl.faceW(i, j, k) * m.SW(i, j, k);
    s += fl.faceN(i, j, k) * m.SN(i, j, k);
    s += fl.faceS(i, j, k) * m.SS(i, j, k);
    s += fl.faceT(i, j, k) * m.ST(i, j, k);
    s += fl.faceB(i, j, k) * m.SB(i, j, k);
    return s / m.vol[m.cid(i, j, k)];
}
static void cellGradients(const Mesh& m, Field<double>& fl, Field<V3>& gr) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < m.nK; ++k)
        for (int j = 0; j < m.nJ; ++j)
            for (int i = 0; i < m.nI; ++i) gr.c[m.cid(i, j, k)] = gradDT(m, fl, i, j, k);
}
static void cellGradientsVec(const Mesh& m, Field<V3>& fl, Field<T3>& gr) {  // FvVectorScheme.cpp:56-74
#pragma omp parallel for schedule(static)
    for (int k = 0; k < m.nK; ++k)
        for (int j = 0; j < m.nJ; ++j)
            for (int i = 0; i < m.nI; ++i) {
                T3 s = tensor(fl.faceE(i, j, k), m.SE(i, j, k));
                s = tadd(s, tensor(fl.faceW(i, j, k), m.SW(i, j, k)));
                s = tadd(s, tensor(fl.faceN(i, j, k), m.SN(i, j, k)));
                s = tadd(s, tensor(fl.faceS(i, j, k), m.SS(i, j, k)));
                s = tadd(s, tensor(fl.faceT(i, j, k), m.ST(i, j, k)));
                s = tadd(s, tensor(fl.faceB(i, j, k), m.SB(i, j, k)));
                gr.c[m.cid(i, j, k)] = tdiv(s, m.vol[m.cid(i, j, k)]);
            }
}

// ----------------------------------------------------------------------------
// Sparse rows with PETSc INSERT_VALUES semantics: negative columns are ignored,
// a repeated column overwrites (SparseMatrix.cpp:73-76).
// ----------------------------------------------------------------------------
struct Rows {
    int n = 0, width = 9;
    std::vector<int> cnt, col;
    std::vector<double> val;
    void allocate(int rows, int w) { n = rows; width = w; cnt.assign(n, 0); col.assign((size_t)n * w, -1); val.assign((size_t)n * w, 0.); }
    void setRow(int r, int nc, const int* cs, const double* vs) {
        for (int q = 0; q < nc; ++q) {
            if (cs[q] < 0) continue;
            int* rc = &col[(size_t)r * width];
            double* rv = &val[(size_t)r * width];
            int p = 0;
            while (p < cnt[r] && rc[p] != cs[q]) ++p;
            if (p == cnt[r]) {
                if (cnt[r] == width) throw std::runtime_error("row preallocation exceeded");
                rc[p] = cs[q]; ++cnt[r];
            }
            rv[p] = vs[q];
        }
    }
    double diag(int r) const {
        for (int p = 0; p < cnt[r]; ++p) if (col[(size_t)r * width + p] == r) return val[(size_t)r * width + p];
        return 0.;
    }
    void mult(const std::vector<double>& x, std::vector<double>& y) const {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r) {
            double s = 0.;
            for (int p = 0; p < cnt[r]; ++p) s += val[(size_t)r * width + p] * x[col[(size_t)r * width + p]];
            y[r] = s;
        }
    }
};

static double dotv(const std::vector<double>& a, const std::vector<double>& b) {
    const int CH = 2048;
    int n = (int)a.size(), nc = (n + CH - 1) / CH;
    std::vector<double> part(nc, 0.);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < nc; ++q) {
        double s = 0.;
        int e = std::min(n, (q + 1) * CH);
        for (int r = q * CH; r < e; ++r) s += a[r] * b[r];
        part[q] = s;
    }
    double s = 0.;
    for (int q = 0; q < nc; ++q) s += part[q];
    return s;
}

enum KspMethod { K_BICGSTAB_SGS = 0, K_BICGSTAB_JACOBI = 1, K_CG_JACOBI = 2 };

struct KspStats { int iters; double rel_res; int status; };  // status 0 ok, 1 maxit, 2 breakdown

// One symmetric Gauss-Seidel sweep from a zero guess (PCSOR, SOR_LOCAL_SYMMETRIC_SWEEP,
// omega 1, its 1, lits 1).
static void sgsApply(const Rows& A, const std::vector<double>& r, std::vector<double>& z) {
    int n = A.n;
    std::fill(z.begin(), z.end(), 0.);
    for (int i = 0; i < n; ++i) {
        double s = r[i], dg = 0.;
        for (int p = 0; p < A.cnt[i]; ++p) {
            int c = A.col[(size_t)i * A.width + p]; double v = A.val[(size_t)i * A.width + p];
            if (c == i) dg = v; else s -= v * z[c];
        }
        z[i] = s / dg;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = r[i], dg = 0.;
        for (int p = 0; p < A.cnt[i]; ++p) {
            int c = A.col[(size_t)i * A.width + p]; double v = A.val[(size_t)i * A.width + p];
            if (c == i) dg = v; else s -= v * z[c];
        }
        z[i] = s / dg;
    }
}

// BiCGStab (van der Vorst 1992), left preconditioned by SGS; convergence on the
// preconditioned residual norm relative to the initial one, as PETSc's default
// test for KSPBCGS.  x starts at zero (KSPSolve default).
static KspStats bicgstabSgs(const Rows& A, const std::vector<double>& b, std::vector<double>& x, double rtol, double atol, int maxit) {
    int n = A.n;
    std::vector<double> r(n), rp(n), p(n, 0.), v(n, 0.), s(n), t(n), tmp(n);
    std::fill(x.begin(), x.end(), 0.);
    sgsApply(A, b, r);
    rp = r;
    double r0 = std::sqrt(dotv(r, r));
    KspStats st{0, 0., 0};
    double rnorm = r0;
    if (r0 == 0.) { st.rel_res = 0.; return st; }
    double rho_old = 1., alpha = 1., omega = 1.;
    for (int it = 1; it <= maxit; ++it) {
        double rho = dotv(r, rp);
        if (rho == 0.) { st.status = 2; st.iters = it - 1; break; }
        double beta = (rho / rho_old) * (alpha / omega);
        for (int q = 0; q < n; ++q) p[q] = r[q] + beta * (p[q] - omega * v[q]);
        A.mult(p, tmp); sgsApply(A, tmp, v);
        alpha = rho / dotv(rp, v);
        for (int q = 0; q < n; ++q) s[q] = r[q] - alpha * v[q];
        A.mult(s, tmp); sgsApply(A, tmp, t);
        double tt = dotv(t, t);
        omega = tt == 0. ? 0. : dotv(t, s) / tt;
        for (int q = 0; q < n; ++q) { x[q] += alpha * p[q] + omega * s[q]; r[q] = s[q] - omega * t[q]; }
        rnorm = std::sqrt(dotv(r, r));
        st.iters = it;
        if (rnorm <= std::max(rtol * r0, atol)) break;
        if (omega == 0.) { st.status = 2; break; }
        rho_old = rho;
        if (it == maxit) st.status = 1;
    }
    st.rel_res = rnorm / r0;
    return st;
}

static double trueRelRes(const Rows& A, const std::vector<double>& b, const std::vector<double>& x, std::vector<double>& r) {
    A.mult(x, r);
    for (int q = 0; q < A.n; ++q) r[q] = b[q] - r[q];
    double bn = std::sqrt(dotv(b, b));
    return bn == 0. ? 0. : std::sqrt(dotv(r, r)) / bn;
}

// BiCGStab right-preconditioned with Jacobi; tests ||b - A x|| <= max(rtol ||b||, atol) (the
// test of PETSc's KSPConvergedDefault, with its rtol and atol) on the recursive residual and
// confirms with the true residual, restarting from it.
static KspStats bicgstabJacobi(const Rows& A, const std::vector<double>& b, std::vector<double>& x, double rtol, int maxit,
                               double atol) {
    int n = A.n;
    std::vector<double> idg(n), r(n), rp(n), p(n), v(n), s(n), t(n), ph(n), sh(n);
    for (int q = 0; q < n; ++q) { double dg = A.diag(q); idg[q] = dg != 0. ? 1. / dg : 1.; }
    std::fill(x.begin(), x.end(), 0.);
    double bn = std::sqrt(dotv(b, b));
    KspStats st{0, 0., 0};
    if (bn == 0.) return st;
    const double tol = std::max(rtol * bn, atol);
    if (bn <= tol) { st.rel_res = 1.; return st; }   // x = 0 already meets the absolute floor
    int it = 0;
    r = b;
    double rnorm = bn;
    while (it < maxit) {
        rp = r;
        std::fill(p.begin(), p.end(), 0.); std::fill(v.begin(), v.end(), 0.);
        double rho_old = 1., alpha = 1., omega = 1.;
        bool restart = false;
        while (it < maxit) {
            ++it;
            double rho = dotv(r, rp);
            if (rho == 0.) { restart = true; break; }
            double beta = (rho / rho_old) * (alpha / omega);
            for (int q = 0; q < n; ++q) p[q] = r[q] + beta * (p[q] - omega * v[q]);
            for (int q = 0; q < n; ++q) ph[q] = idg[q] * p[q];
            A.mult(ph, v);
            double rv = dotv(rp, v);
            if (rv == 0.) { restart = true; break; }
            alpha = rho / rv;
            for (int q = 0; q < n; ++q) s[q] = r[q] - alpha * v[q];
            for (int q = 0; q < n; ++q) sh[q] = idg[q] * s[q];
            A.mult(sh, t);
            double tt = dotv(t, t);
            omega = tt == 0. ? 0. : dotv(t, s) / tt;
            for (int q = 0; q < n; ++q) { x[q] += alpha * ph[q] + omega * sh[q]; r[q] = s[q] - omega * t[q]; }
            rnorm = std::sqrt(dotv(r, r));
            if (rnorm <= tol) break;
            if (omega == 0.) { restart = true; break; }
            rho_old = rho;
        }
        double tr = trueRelRes(A, b, x, r);
        rnorm = tr * bn;
        if (rnorm <= tol) { st.iters = it; st.rel_res = tr; return st; }
        (void)restart;
    }
    st.iters = it; st.rel_res = rnorm / bn; st.status = 1;
    return st;
}

static KspStats cgJacobi(const Rows& A, const std::vector<double>& b, std::vector<double>& x, double rtol, int maxit, double atol) {
    int n = A.n;
    std::vector<double> idg(n), r(n), z(n), p(n), q(n);
    for (int i = 0; i < n; ++i) { double dg = A.diag(i); idg[i] = dg != 0. ? 1. / dg : 1.; }
    std::fill(x.begin(), x.end(), 0.);
    double bn = std::sqrt(dotv(b, b));
    KspStats st{0, 0., 0};
    if (bn == 0.) return st;
    const double tol = std::max(rtol * bn, atol);
    if (bn <= tol) { st.rel_res = 1.; return st; }   // x = 0 already meets the absolute floor
    r = b;
    int it = 0;
    double rnorm = bn;
    while (it < maxit) {
        for (int i = 0; i < n; ++i) z[i] = idg[i] * r[i];
        p = z;
        double rz = dotv(r, z);
        while (it < maxit) {
            ++it;
            A.mult(p, q);
            double pq = dotv(p, q);
            if (pq == 0.) break;
            double alpha = rz / pq;
            for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; z[i] = idg[i] * r[i]; }
            double rzn = dotv(r, z);
            rnorm = std::sqrt(dotv(r, r));
            if (rnorm <= tol) break;
            double beta = rzn / rz;
            rz = rzn;
            for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
        double tr = trueRelRes(A, b, x, r);
        rnorm = tr * bn;
        if (rnorm <= tol) { st.iters = it; st.rel_res = tr; return st; }
    }
    st.iters = it; st.rel_res = rnorm / bn; st.status = 1;
    return st;
}

// atol: absolute floor of the stopping test; the reference leaves PETSc's default 1e-50
// (src/Math/SparseMatrix.cpp:95-105), which the SGS form keeps when atol is 0.
static KspStats kspSolve(int method, const Rows& A, const std::vector<double>& b, std::vector<double>& x, double rtol, int maxit,
                         double atol = 0.) {
    if (method == K_BICGSTAB_SGS) return bicgstabSgs(A, b, x, rtol, atol > 0. ? atol : 1e-50, maxit);
    if (method == K_BICGSTAB_JACOBI) return bicgstabJacobi(A, b, x, rtol, maxit, atol);
    return cgJacobi(A, b, x, rtol, maxit, atol);
}

// ----------------------------------------------------------------------------
// Diffusion (src/Solvers/Diffusion.cpp): scalar diffusion with unit diffusivity on one
// block, one linear solve per call.  The reference's coefficients are kept as written
// (Diffusion.cpp:73-85): a_nb = +D_f, a_P = -sum D_f + V/dt, b = (V/dt) phi0.  For a steady
// case (a0P = 0) this is the Laplace equation; for an unsteady one it reads
// (V/dt)(phi_P - phi0) = sum D_f (phi_P - phi_nb), the sign of the diffusion term opposite
// to the heat equation's.
// ----------------------------------------------------------------------------
struct Diffusion {
    Mesh m;
    int N = 0;
    int unsteady = 0, method = K_BICGSTAB_SGS, maxit = 10000;
    double rtol = 1e-8;
    Field<double> phi;
    Field<V3> gradPhi;
    BC<double> bc;
    Rows A;
    std::vector<double> b, x, res;
    int iters = 0;
    double relRes = 0., resInf = 0.;

    // Diffusion::Diffusion (Diffusion.cpp:35-53): boundary types and reference values
    // (PrimitiveBoundaryCondition(input, field), PrimitiveBoundaryCondition.tpp:4-30, which
    // fixes the patches), then the uniform initial value of phi.
    void init(const double* xyz, int nNI, int nNJ, int nNK, const int* types, const double* refs, int timeAccurate, double phi0,
              int kspMethod, double tol, int maxIters) {
        m.build(xyz, nNI, nNJ, nNK);
        N = (int)m.N();
        unsteady = timeAccurate; method = kspMethod; rtol = tol; maxit = maxIters;
        phi.allocate(m.nI, m.nJ, m.nK);
        gradPhi.allocate(m.nI, m.nJ, m.nK);
        bc.init(&phi);
        for (int f = 0; f < 6; ++f) {
            if (types[f] < 0 || types[f] > 2) throw std::runtime_error("invalid boundary type");
            bc.type[f] = (PType)types[f];
            bc.ref[f] = refs[f];
        }
        bc.setFixedBoundaries();
        std::fill(phi.c.begin(), phi.c.end(), phi0);
        A.allocate(N, 7);
        b.assign(N, 0.); x.assign(N, 0.); res.assign(N, 0.);
    }

    // Diffusion::solve (Diffusion.cpp:58-131); returns ||A x - b||_inf
    double solve(double dt) {
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    double a0P = unsteady ? m.vol[c] / dt : 0.;
                    double a[7];
                    for (int f = 0; f < 6; ++f) a[f + 1] = m.d[f][c];
                    a[0] = -(a[1] + a[2] + a[3] + a[4] + a[5] + a[6]) + a0P;
                    double bb = a0P * phi.c[c];
                    bc.setImplicit(i, j, k, a, bb);
                    int cols[7] = {c, i < m.uI() ? c + 1 : -1, i > 0 ? c - 1 : -1, j < m.uJ() ? c + m.nI : -1,
                                   j > 0 ? c - m.nI : -1, k < m.uK() ? c + m.nI * m.nJ : -1, k > 0 ? c - m.nI * m.nJ : -1};
                    A.setRow(c, 7, cols, a);
                    b[c] = bb;
                }
        KspStats st = kspSolve(method, A, b, x, rtol, maxit);
        iters = st.iters;
        relRes = trueRelRes(A, b, x, res);
        phi.c = x;
        bc.setBoundaries();
        extrapolateInteriorFaces();
        cellGradients(m, phi, gradPhi);
        A.mult(x, res);                       // res = A x - b (Diffusion.cpp:127-130)
        resInf = 0.;
        for (int q = 0; q < N; ++q) { res[q] -= b[q]; resInf = std::max(resInf, std::fabs(res[q])); }
        return resInf;
    }

    // FvScalarScheme::extrapolateInteriorFaces (FvScalarScheme.cpp:70-156) on one block:
    // volume-weighted faces, divergence-theorem gradients, then every interior face from the
    // two cells' gradients, clamped to the range of the lower cell and its 6 neighbours.
    // Each interior face is written by its lower cell only, so the order does not matter.
    void extrapolateInteriorFaces() {
        interpolateInteriorFaces(m, phi);
        cellGradients(m, phi, gradPhi);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    double p = phi.c[c];
                    bool lE = false, lN = false, lT = false;
                    if (i < m.uI()) {
                        phi.faceE(i, j, k) = 0.5 * (p + dot(gradPhi.c[c], m.c2f[0][c]) + phi.c[c + 1] + dot(gradPhi.c[c + 1], m.c2f[1][c + 1]));
                        lE = true;
                    }
                    if (j < m.uJ()) {
                        int n = c + m.nI;
                        phi.faceN(i, j, k) = 0.5 * (p + dot(gradPhi.c[c], m.c2f[2][c]) + phi.c[n] + dot(gradPhi.c[n], m.c2f[3][n]));
                        lN = true;
                    }
                    if (k < m.uK()) {
                        int t = c + m.nI * m.nJ;
                        phi.faceT(i, j, k) = 0.5 * (p + dot(gradPhi.c[c], m.c2f[4][c]) + phi.c[t] + dot(gradPhi.c[t], m.c2f[5][t]));
                        lT = true;
                    }
                    // Field::maxNeighbour / minNeighbour (Field.tpp:407-438), boundary patches included
                    double hi = p, lo = p;
                    const double nb[6] = {phi.at(i + 1, j, k), phi.at(i - 1, j, k), phi.at(i, j + 1, k),
                                          phi.at(i, j - 1, k), phi.at(i, j, k + 1), phi.at(i, j, k - 1)};
                    for (double v : nb) { hi = std::max(hi, v); lo = std::min(lo, v); }
                    if (lE) phi.faceE(i, j, k) = std::max(std::min(hi, phi.faceE(i, j, k)), lo);
                    if (lN) phi.faceN(i, j, k) = std::max(std::min(hi, phi.faceN(i, j, k)), lo);
                    if (lT) phi.faceT(i, j, k) = std::max(std::min(hi, phi.faceT(i, j, k)), lo);
                }
    }
};

// ----------------------------------------------------------------------------
// Case description shared with the Python side (ctypes Structure of the same layout)
// ----------------------------------------------------------------------------
enum SolverKind { S_SIMPLE = 0, S_PISO = 1, S_IBPISO = 2 };

}  // namespace orc

extern "C" {
struct OracleCase {
    int kind;              // 0 Simple, 1 Piso, 2 IbPiso
    int bc_type[6];        // FlowBoundaryConditions::Type per face E W N S T B
    double ref_vec[6][3];  // Boundaries.<face>.refVector
    double ref_val[6];     // Boundaries.<face>.refValue
    double rho, mu;        // Solver.rho, Solver.mu
    int time_accurate;     // Solver.timeAccurate ON/OFF
    double omega_u, omega_p;
    int n_inner, n_pcorr;
    int convection;        // 0 upwind (reference), 1 central (extension)
    int nonorth;           // 0 off (reference), 1 volume-weighted face gradU (extension)
    int mom_method, p_method;
    double mom_rtol, p_rtol;
    int maxit;
    double ib_radius;
    double ib_center[3];
    double u_init[3];
    double p_init;
    double mom_atol, p_atol;   // absolute floors of the linear solves (0: relative test only)
};
}

namespace orc {

struct Solver {
    Mesh m;
    OracleCase cs;
    int N = 0;
    // IndexMap (IndexMap.cpp) single block
    std::vector<int> status, row;  // 0 ACTIVE, 1 GHOST, 2 INACTIVE
    int nRows = 0;
    Field<V3> u, h, gradP, gradPC, uf0;
    Field<double> p, pc, d, mf;
    Field<T3> gradU;
    Field<int> ib;   // IbPiso::CellType FLUID 0, IB 1, SOLID 2; patches stay FLUID
    BC<V3> uBc, hBc;
    BC<double> pBc, pcBc, dBc;
    int flow[6];
    Rows A[2];
    std::vector<double> bv[3], xv[3];
    KspStats momStats[3], pStats;
    int momItersTotal = 0, pItersLast = 0, pItersTotal = 0, nPSolves = 0;
    double pResMax = 0., momResMax = 0.;
    double continuity = 0., courant = 0.;
    int nGhost = 0;

    bool active(int c) const { return status[c] == 0; }
    bool inactive(int c) const { return status[c] == 2; }
    int rowOf(int i, int j, int k) const {  // IndexMap::operator(), IndexMap.cpp:47-78
        if (i < 0 || j < 0 || k < 0 || i >= m.nI || j >= m.nJ || k >= m.nK) return -1;
        return row[m.cid(i, j, k)];
    }
    void generateLocalIndices() {  // IndexMap.cpp:128-148
        nRows = 0;
        for (int c = 0; c < N; ++c) row[c] = status[c] == 2 ? -1 : nRows++;
    }
    bool massCorr(int f) const { return flow[f] == F_OUTLET; }  // SimpleBoundaryCondition.cpp:34-62

    void createMatrices(int nnz) {  // Solver.cpp:23-41
        for (int q = 0; q < 2; ++q) A[q].allocate(nRows, nnz);
        for (int q = 0; q < 3; ++q) { bv[q].assign(nRows, 0.); xv[q].assign(nRows, 0.); }
    }

    void init(const double* xyz, int nNI, int nNJ, int nNK, const OracleCase& c) {
        cs = c;
        m.build(xyz, nNI, nNJ, nNK);
        N = (int)m.N();
        status.assign(N, 0); row.assign(N, 0);
        generateLocalIndices();   // IndexMap::initialize, IndexMap.cpp:34-45
        u.allocate(m.nI, m.nJ, m.nK); h.allocate(m.nI, m.nJ, m.nK); gradP.allocate(m.nI, m.nJ, m.nK);
        gradPC.allocate(m.nI, m.nJ, m.nK); uf0.allocate(m.nI, m.nJ, m.nK);
        p.allocate(m.nI, m.nJ, m.nK); pc.allocate(m.nI, m.nJ, m.nK); d.allocate(m.nI, m.nJ, m.nK); mf.allocate(m.nI, m.nJ, m.nK);
        if (cs.nonorth) gradU.allocate(m.nI, m.nJ, m.nK);
        ib.allocate(m.nI, m.nJ, m.nK);
        uBc.init(&u); hBc.init(&h); pBc.init(&p); pcBc.init(&pc); dBc.init(&d);
        // FlowBoundaryConditions ctor, FlowBoundaryConditions.cpp:3-73
        for (int f = 0; f < 6; ++f) {
            flow[f] = cs.bc_type[f];
            V3 rv = v3(cs.ref_vec[f][0], cs.ref_vec[f][1], cs.ref_vec[f][2]);
            double rp = cs.ref_val[f];
            if (flow[f] == F_INLET || flow[f] == F_WALL) {
                uBc.changeType(f, P_FIXED, rv); pBc.changeType(f, P_ZERO_GRADIENT, rp); hBc.changeType(f, P_FIXED, rv);
            } else if (flow[f] == F_OUTLET) {
                uBc.changeType(f, P_ZERO_GRADIENT, rv); pBc.changeType(f, P_FIXED, rp); hBc.changeType(f, P_ZERO_GRADIENT, rv);
            } else if (flow[f] == F_EMPTY) {
                uBc.changeType(f, P_EMPTY, rv); pBc.changeType(f, P_EMPTY, rp); hBc.changeType(f, P_EMPTY, rv);
            } else if (flow[f] == F_ZERO_GRADIENT) {
                uBc.changeType(f, P_ZERO_GRADIENT, rv); pBc.changeType(f, P_ZERO_GRADIENT, rp); hBc.changeType(f, P_ZERO_GRADIENT, rv);
            } else throw std::runtime_error("invalid boundary type");
            dBc.changeType(f, P_ZERO_GRADIENT, 0.);
        }
        // SimpleBoundaryCondition ctor, SimpleBoundaryCondition.cpp:3-15
        for (int f = 0; f < 6; ++f) pcBc.changeType(f, pBc.type[f], 0.);
        createMatrices(cs.kind == S_IBPISO ? 9 : 7);
        // uniform initial conditions (InitialConditions.tpp:31-35) set cells only
        for (int q = 0; q < N; ++q) { u.c[q] = v3(cs.u_init[0], cs.u_init[1], cs.u_init[2]); p.c[q] = cs.p_init; }
    }

    // ---------------------------------------------------------------- IB (IbPiso.cpp)
    bool sphereInside(V3 x) const {  // Sphere.cpp:49-55
        V3 c = v3(cs.ib_center[0], cs.ib_center[1], cs.ib_center[2]);
        return mag(x - c) <= cs.ib_radius;
    }
    void computeIbField() {  // IbPiso.cpp:65-117
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (sphereInside(m.cc[c])) { ib.c[c] = 2; status[c] = 2; u.c[c] = zero3(); p.c[c] = 0.; }
                    else { ib.c[c] = 0; status[c] = 0; }
                }
        nGhost = 0;
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (ib.c[c] == 2) {
                        if (ib.at(i + 1, j, k) == 0 || ib.at(i - 1, j, k) == 0 || ib.at(i, j + 1, k) == 0 ||
                            ib.at(i, j - 1, k) == 0 || ib.at(i, j, k + 1) == 0 || ib.at(i, j, k - 1) == 0) {
                            ib.c[c] = 1; status[c] = 1; ++nGhost;
                        }
                    }
                }
        generateLocalIndices();
        createMatrices(9);
    }
    std::vector<double> ibBeta;  // per ghost (k-j-i order): 8 weights
    std::vector<int> ibStencil;  // per ghost: 8 cell ids
    void computeIbCoeffs() {  // IbPiso.cpp:119-190
        V3 ctr = v3(cs.ib_center[0], cs.ib_center[1], cs.ib_center[2]);
        ibBeta.clear(); ibStencil.clear();
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (ib.c[c] != 1) continue;
                    V3 l = unitv(m.cc[c] - ctr);                       // Sphere::nearestIntersect, Sphere.cpp:23-30
                    V3 bp = ctr + cs.ib_radius * l;
                    V3 ip = 2. * bp - m.cc[c];
                    int ii[8], jj[8], kk[8];
                    if (!m.locateEnclosingCells(ip, i, j, k, ii, jj, kk))
                        throw std::runtime_error("image point outside the cell-centre lattice");
                    V3 pts[8];
                    for (int q = 0; q < 8; ++q) pts[q] = m.cc[m.cid(ii[q], jj[q], kk[q])];
                    double beta[8];
                    trilinearCoeffs(pts, ip, beta);
                    int cols[9]; double vals[9];
                    vals[0] = 1.; cols[0] = rowOf(i, j, k);
                    for (int q = 0; q < 8; ++q) {
                        if (ii[q] == i && jj[q] == j && kk[q] == k) { vals[0] += beta[q]; cols[q + 1] = -1; }
                        else { vals[q + 1] = beta[q]; cols[q + 1] = rowOf(ii[q], jj[q], kk[q]); }
                    }
                    A[0].setRow(rowOf(i, j, k), 9, cols, vals);
                    for (int q = 0; q < 8; ++q) {   // the diagonal is reset on every pass (IbPiso.cpp:168-183)
                        vals[0] = -1; cols[0] = rowOf(i, j, k);
                        if (ii[q] == i && jj[q] == j && kk[q] == k) { vals[0] += beta[q]; cols[q + 1] = -1; }
                        else { vals[q + 1] = beta[q]; cols[q + 1] = rowOf(ii[q], jj[q], kk[q]); }
                    }
                    A[1].setRow(rowOf(i, j, k), 9, cols, vals);
                    for (int q = 0; q < 8; ++q) { ibBeta.push_back(beta[q]); ibStencil.push_back(m.cid(ii[q], jj[q], kk[q])); }
                }
    }

    // ---------------------------------------------------------------- Simple.cpp
    std::vector<double> momA;  // per cell: 7 coefficients (after BC folding), for kernel tests
    std::vector<V3> momB;

    void assembleMomentum(double dt) {  // Simple.cpp:117-179
        bool unsteady = cs.time_accurate != 0;
        double om = cs.omega_u, mu = cs.mu;
        if (cs.nonorth) {  // extension: volume-weighted face gradU (boundary faces: zero gradient)
            for (int f = 0; f < 6; ++f) gradU.patch[f].assign(gradU.patch[f].size(), zeroOf<T3>());
            for (int f = 0; f < 6; ++f) gradU.zeroGradient(f);
            interpolateInteriorFaces(m, gradU);
        }
        momA.assign((size_t)N * 7, 0.);
        momB.assign(N, zero3());
        std::vector<int> colsAll((size_t)N * 7);
        std::vector<double> valsAll((size_t)N * 7);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (!active(c)) continue;
                    double a0P = unsteady ? cs.rho * m.vol[c] / dt : 0.;
                    double FE = mf.faceE(i, j, k), FW = mf.faceW(i, j, k), FN = mf.faceN(i, j, k);
                    double FS = mf.faceS(i, j, k), FT = mf.faceT(i, j, k), FB = mf.faceB(i, j, k);
                    double a[7];
                    if (cs.convection == 0) {
                        a[1] = std::min(FE, 0.) - mu * m.d[0][c];
                        a[2] = -std::max(FW, 0.) - mu * m.d[1][c];
                        a[3] = std::min(FN, 0.) - mu * m.d[2][c];
                        a[4] = -std::max(FS, 0.) - mu * m.d[3][c];
                        a[5] = std::min(FT, 0.) - mu * m.d[4][c];
                        a[6] = -std::max(FB, 0.) - mu * m.d[5][c];
                        a[0] = (std::max(FE, 0.) + mu * m.d[0][c] - std::min(FW, 0.) + mu * m.d[1][c]
                                + std::max(FN, 0.) + mu * m.d[2][c] - std::min(FS, 0.) + mu * m.d[3][c]
                                + std::max(FT, 0.) + mu * m.d[4][c] - std::min(FB, 0.) + mu * m.d[5][c] + a0P) / om;
                    } else {
                        // extension: implicit volume-weighted central differencing; the face
                        // value seen from cell P is g_f phi_P + (1 - g_f) phi_nb (g_f of cell P)
                        const double* gg[6] = {&m.g[0][c], &m.g[1][c], &m.g[2][c], &m.g[3][c], &m.g[4][c], &m.g[5][c]};
                        a[1] = FE * (1. - *gg[0]) - mu * m.d[0][c];
                        a[2] = -FW * (1. - *gg[1]) - mu * m.d[1][c];
                        a[3] = FN * (1. - *gg[2]) - mu * m.d[2][c];
                        a[4] = -FS * (1. - *gg[3]) - mu * m.d[3][c];
                        a[5] = FT * (1. - *gg[4]) - mu * m.d[4][c];
                        a[6] = -FB * (1. - *gg[5]) - mu * m.d[5][c];
                        a[0] = (FE * *gg[0] + mu * m.d[0][c] - FW * *gg[1] + mu * m.d[1][c]
                                + FN * *gg[2] + mu * m.d[2][c] - FS * *gg[3] + mu * m.d[3][c]
                                + FT * *gg[4] + mu * m.d[4][c] - FB * *gg[5] + mu * m.d[5][c] + a0P) / om;
                    }
                    V3 b = a0P * uf0.c[c];
                    b += -m.vol[c] * gradP.c[c];
                    b += (1. - om) * a[0] * u.c[c];
                    if (cs.nonorth) {
                        b += mu * tdot(gradU.faceE(i, j, k), m.cvec[0][c]);
                        b += mu * tdot(gradU.faceW(i, j, k), m.cvec[1][c]);
                        b += mu * tdot(gradU.faceN(i, j, k), m.cvec[2][c]);
                        b += mu * tdot(gradU.faceS(i, j, k), m.cvec[3][c]);
                        b += mu * tdot(gradU.faceT(i, j, k), m.cvec[4][c]);
                        b += mu * tdot(gradU.faceB(i, j, k), m.cvec[5][c]);
                    }
                    uBc.setImplicit(i, j, k, a, b);
                    int* cols = &colsAll[(size_t)c * 7];
                    cols[0] = rowOf(i, j, k);
                    cols[1] = rowOf(i + 1, j, k); cols[2] = rowOf(i - 1, j, k);
                    cols[3] = rowOf(i, j + 1, k); cols[4] = rowOf(i, j - 1, k);
                    cols[5] = rowOf(i, j, k + 1); cols[6] = rowOf(i, j, k - 1);
                    for (int q = 0; q < 7; ++q) { valsAll[(size_t)c * 7 + q] = a[q]; momA[(size_t)c * 7 + q] = cols[q] < 0 ? 0. : a[q]; }
                    momB[c] = b;
                    d.c[c] = m.vol[c] / a[0];
                }
        for (int c = 0; c < N; ++c) {
            if (!active(c)) continue;
            int r = row[c];
            A[0].setRow(r, 7, &colsAll[(size_t)c * 7], &valsAll[(size_t)c * 7]);
            bv[0][r] = momB[c].x; bv[1][r] = momB[c].y; bv[2][r] = momB[c].z;
        }
    }
    void solveMomentum() {  // Simple.cpp:184-207
        for (int comp = 0; comp < 3; ++comp) {
            momStats[comp] = kspSolve(cs.mom_method, A[0], bv[comp], xv[comp], cs.mom_rtol, cs.maxit, cs.mom_atol);
            momItersTotal += momStats[comp].iters;
            momResMax = std::max(momResMax, momStats[comp].rel_res);
#pragma omp parallel for schedule(static)
            for (int c = 0; c < N; ++c) {
                if (inactive(c)) continue;
                double val = xv[comp][row[c]];
                orc::comp(u.c[c], comp) = val;
                if (active(c)) orc::comp(h.c[c], comp) = val + d.c[c] * orc::comp(gradP.c[c], comp);
                else orc::comp(h.c[c], comp) = val;
            }
        }
    }
    void rhieChow() {  // Simple.cpp:410-449
        double rho = cs.rho;
#pragma omp parallel for schedule(static)
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (inactive(c)) continue;
                    if (i == 0) { mf.faceW(i, j, k) = -dot(h.faceW(i, j, k), m.SW(i, j, k)) + d.faceW(i, j, k) * (p.at(i - 1, j, k) - p.at(i, j, k)) * m.d[1][c];
                                  mf.faceW(i, j, k) *= rho; }
                    if (j == 0) { mf.faceS(i, j, k) = -dot(h.faceS(i, j, k), m.SS(i, j, k)) + d.faceS(i, j, k) * (p.at(i, j - 1, k) - p.at(i, j, k)) * m.d[3][c];
                                  mf.faceS(i, j, k) *= rho; }
                    if (k == 0) { mf.faceB(i, j, k) = -dot(h.faceB(i, j, k), m.SB(i, j, k)) + d.faceB(i, j, k) * (p.at(i, j, k - 1) - p.at(i, j, k)) * m.d[5][c];
                                  mf.faceB(i, j, k) *= rho; }
                    mf.faceE(i, j, k) = dot(h.faceE(i, j, k), m.SE(i, j, k)) - d.faceE(i, j, k) * (p.at(i + 1, j, k) - p.at(i, j, k)) * m.d[0][c];
                    mf.faceN(i, j, k) = dot(h.faceN(i, j, k), m.SN(i, j, k)) - d.faceN(i, j, k) * (p.at(i, j + 1, k) - p.at(i, j, k)) * m.d[2][c];
                    mf.faceT(i, j, k) = dot(h.faceT(i, j, k), m.ST(i, j, k)) - d.faceT(i, j, k) * (p.at(i, j, k + 1) - p.at(i, j, k)) * m.d[4][c];
                    mf.faceE(i, j, k) *= rho; mf.faceN(i, j, k) *= rho; mf.faceT(i, j, k) *= rho;
                }
    }
    void momentumPost() {  // Simple.cpp:213-220
        uBc.setBoundaries(); dBc.setBoundaries(); hBc.setBoundaries();
        interpolateInteriorFaces(m, d);
        interpolateInteriorFaces(m, h);
        rhieChow();
    }
    void computeMomentum(double dt) { assembleMomentum(dt); solveMomentum(); momentumPost(); }

    std::vector<double> pcA;   // per cell 7 coefficients after folding (dropped columns zero)
    std::vector<double> pcB;
    void assemblePCorr() {  // Simple.cpp:230-269
        double rho = cs.rho;
        pcA.assign((size_t)N * 7, 0.); pcB.assign(N, 0.);
        std::vector<int> colsAll((size_t)N * 7);
        std::vector<double> valsAll((size_t)N * 7);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (!active(c)) continue;
                    double a[7];
                    a[1] = rho * d.faceE(i, j, k) * m.d[0][c];
                    a[2] = rho * d.faceW(i, j, k) * m.d[1][c];
                    a[3] = rho * d.faceN(i, j, k) * m.d[2][c];
                    a[4] = rho * d.faceS(i, j, k) * m.d[3][c];
                    a[5] = rho * d.faceT(i, j, k) * m.d[4][c];
                    a[6] = rho * d.faceB(i, j, k) * m.d[5][c];
                    a[0] = -(a[1] + a[2] + a[3] + a[4] + a[5] + a[6]);
                    double b = mf.faceE(i, j, k) - mf.faceW(i, j, k) + mf.faceN(i, j, k) - mf.faceS(i, j, k)
                             + mf.faceT(i, j, k) - mf.faceB(i, j, k);
                    pcBc.setImplicit(i, j, k, a, b);
                    int* cols = &colsAll[(size_t)c * 7];
                    cols[0] = rowOf(i, j, k);
                    cols[1] = rowOf(i + 1, j, k); cols[2] = rowOf(i - 1, j, k);
                    cols[3] = rowOf(i, j + 1, k); cols[4] = rowOf(i, j - 1, k);
                    cols[5] = rowOf(i, j, k + 1); cols[6] = rowOf(i, j, k - 1);
                    for (int q = 0; q < 7; ++q) { valsAll[(size_t)c * 7 + q] = a[q]; pcA[(size_t)c * 7 + q] = cols[q] < 0 ? 0. : a[q]; }
                    pcB[c] = b;
                }
        for (int c = 0; c < N; ++c) {
            if (!active(c)) continue;
            A[1].setRow(row[c], 7, &colsAll[(size_t)c * 7], &valsAll[(size_t)c * 7]);
            bv[0][row[c]] = pcB[c];
        }
    }
    // With no fixed-pressure face and no immersed boundary the p' matrix has the constant
    // vector as its null space.  Its right-hand side then carries a round-off component
    // along that null space (the second PISO corrector's right-hand side is round-off
    // sized), which no Krylov method can reduce; the right-hand side is projected onto
    // the range by removing its mean (an extension: PETSc's default 1e-5 preconditioned
    // tolerance never meets this floor, a 1e-8 true-residual tolerance does).
    bool pSingular() const {
        if (cs.kind == S_IBPISO) return false;
        for (int f = 0; f < 6; ++f) if (pBc.type[f] == P_FIXED) return false;
        return true;
    }
    void solvePCorr() {  // Simple.cpp:274-298
        if (pSingular()) {
            std::vector<double> ones(bv[0].size(), 1.);
            double mean = dotv(bv[0], ones) / (double)bv[0].size();
            for (double& v : bv[0]) v -= mean;
        }
        pStats = kspSolve(cs.p_method, A[1], bv[0], xv[0], cs.p_rtol, cs.maxit, cs.p_atol);
        if (pSingular()) {
            // the solution is defined up to a constant, and on meshes with non-planar faces the
            // discrete gradient (sum of face values times area vectors) is not blind to that
            // constant: it is fixed to zero mean so that every Krylov method gives the same p'
            std::vector<double> ones(xv[0].size(), 1.);
            double mean = dotv(xv[0], ones) / (double)xv[0].size();
            for (double& v : xv[0]) v -= mean;
        }
        pItersLast = pStats.iters; pItersTotal += pStats.iters; ++nPSolves;
        pResMax = std::max(pResMax, pStats.rel_res);
        for (int c = 0; c < N; ++c) if (!inactive(c)) pc.c[c] = xv[0][row[c]];
        pcBc.setBoundaries();
        interpolateInteriorFaces(m, pc);
        cellGradients(m, pc, gradPC);
    }
    void computePCorr() { assemblePCorr(); solvePCorr(); }

    void correct() {  // Simple.cpp:301-356
        double rho = cs.rho, omp = cs.omega_p;
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (inactive(c)) continue;
                    if (i == 0 && massCorr(1)) mf.faceW(i, j, k) += rho * d.faceW(i, j, k) * (pc.at(i - 1, j, k) - pc.at(i, j, k)) * m.d[1][c];
                    if (j == 0 && massCorr(3)) mf.faceS(i, j, k) += rho * d.faceS(i, j, k) * (pc.at(i, j - 1, k) - pc.at(i, j, k)) * m.d[3][c];
                    if (k == 0 && massCorr(5)) mf.faceB(i, j, k) += rho * d.faceB(i, j, k) * (pc.at(i, j, k - 1) - pc.at(i, j, k)) * m.d[5][c];
                    if (i < m.uI() || massCorr(0)) mf.faceE(i, j, k) += -rho * d.faceE(i, j, k) * (pc.at(i + 1, j, k) - pc.at(i, j, k)) * m.d[0][c];
                    if (j < m.uJ() || massCorr(2)) mf.faceN(i, j, k) += -rho * d.faceN(i, j, k) * (pc.at(i, j + 1, k) - pc.at(i, j, k)) * m.d[2][c];
                    if (k < m.uK() || massCorr(4)) mf.faceT(i, j, k) += -rho * d.faceT(i, j, k) * (pc.at(i, j, k + 1) - pc.at(i, j, k)) * m.d[4][c];
                    mf.c[c] = mf.faceE(i, j, k) - mf.faceW(i, j, k) + mf.faceN(i, j, k) - mf.faceS(i, j, k)
                            + mf.faceT(i, j, k) - mf.faceB(i, j, k);
                    p.c[c] += omp * pc.c[c];
                    u.c[c] += -d.c[c] * gradPC.c[c];
                }
        pBc.setBoundaries(); uBc.setBoundaries();
        interpolateInteriorFaces(m, p);
        interpolateInteriorFaces(m, u);
        cellGradients(m, p, gradP);
        if (cs.nonorth) cellGradientsVec(m, u, gradU);   // only consumed by the extension
    }
    double computeContinuityError() {  // Simple.cpp:358-380 (compare |m| against a stored |m|/V)
        double ce = 0.;
        for (int c = 0; c < N; ++c) {
            if (!active(c)) continue;
            if (std::fabs(mf.c[c]) > ce) ce = std::fabs(mf.c[c]) / m.vol[c];
        }
        continuity = ce;
        return ce;
    }
    double computeCourantNumber(double dt) {  // Simple.cpp:382-408
        double mx = 0.;
        for (int c = 0; c < N; ++c) {
            V3 rI = m.c2f[0][c] - m.c2f[1][c], rJ = m.c2f[2][c] - m.c2f[3][c], rK = m.c2f[4][c] - m.c2f[5][c];
            double uI = std::fabs(dot(u.c[c], unitv(rI)));
            double uJ = std::fabs(dot(u.c[c], unitv(rJ)));
            double uK = std::fabs(dot(u.c[c], unitv(rK)));
            double co = dt * (uI / mag(rI) + uJ / mag(rJ) + uK / mag(rK));
            if (co > mx) mx = co;
        }
        courant = mx;
        return mx;
    }
    double solve(double dt) {
        momItersTotal = 0; pItersTotal = 0; nPSolves = 0; pResMax = 0.; momResMax = 0.;
        uf0.c = u.c;  // uField0_ = uField_ (AUXILLARY: cells only)
        if (cs.kind == S_SIMPLE) {  // Simple::solve, Simple.cpp:78-91
            int nIn = cs.time_accurate ? cs.n_inner : 1;
            for (int it = 0; it < nIn; ++it) { computeMomentum(dt); computePCorr(); correct(); }
            computeCourantNumber(dt);
            return computeContinuityError();
        } else if (cs.kind == S_PISO) {  // Piso::solve, Piso.cpp:12-29
            int nIn = cs.time_accurate ? cs.n_inner : 1;
            for (int it = 0; it < nIn; ++it) {
                computeMomentum(dt);
                for (int q = 0; q < cs.n_pcorr; ++q) { computePCorr(); correct(); }
            }
            computeCourantNumber(dt);
            return computeContinuityError();
        } else {  // IbPiso::solve, IbPiso.cpp:43-61
            computeIbField();
            int nIn = cs.time_accurate ? cs.n_inner : 1;
            for (int it = 0; it < nIn; ++it) {
                computeIbCoeffs();
                computeMomentum(dt);
                for (int q = 0; q < cs.n_pcorr; ++q) { computePCorr(); correct(); }
            }
            return computeContinuityError();
        }
    }
};

// ----------------------------------------------------------------------------
// Coupled (src/Solvers/Coupled.cpp): momentum and continuity in one linear system of
// 4 N unknowns (u_x, u_y, u_z, p, blocked by variable: row = cell + var N, IndexMap.cpp:47-52),
// on one block without an immersed boundary.  Momentum rows hold 7 velocity and 7 pressure
// coefficients, continuity rows 3 x 7 velocity and 7 pressure coefficients (28).  The
// reference's own conventions are kept: rho and mu are constant fields (Field::setAll,
// Field.tpp:271-278), the face mass flux carries no rho (Coupled.cpp:282-314), the boundary
// faces of the pressure-gradient field stay zero, p is never interpolated to interior faces
// before its gradient (Coupled.cpp:257-258, so those faces keep their initial zero), and u and
// p start at zero (the constructor applies no initial conditions).
// ----------------------------------------------------------------------------
struct Coupled {
    Mesh m;
    OracleCase cs;
    int N = 0;
    Field<V3> u, h, gradP, u0, uStar;
    Field<double> p, d, mf;
    BC<V3> uBc, hBc;
    BC<double> pBc, dBc;
    Rows A;
    std::vector<double> b, x;
    KspStats st{0, 0., 0};
    int nInner = 1;
    double omega = 1., rho = 1., mu = 1.;

    // Coupled::Coupled (Coupled.cpp:5-34) with FlowBoundaryConditions (FlowBoundaryConditions.cpp:3-73)
    void init(const double* xyz, int nNI, int nNJ, int nNK, const OracleCase& c) {
        cs = c;
        m.build(xyz, nNI, nNJ, nNK);
        N = (int)m.N();
        u.allocate(m.nI, m.nJ, m.nK); h.allocate(m.nI, m.nJ, m.nK); gradP.allocate(m.nI, m.nJ, m.nK);
        u0.allocate(m.nI, m.nJ, m.nK); uStar.allocate(m.nI, m.nJ, m.nK);
        p.allocate(m.nI, m.nJ, m.nK); d.allocate(m.nI, m.nJ, m.nK); mf.allocate(m.nI, m.nJ, m.nK);
        uBc.init(&u); hBc.init(&h); pBc.init(&p); dBc.init(&d);
        for (int f = 0; f < 6; ++f) {
            int t = cs.bc_type[f];
            V3 rv = v3(cs.ref_vec[f][0], cs.ref_vec[f][1], cs.ref_vec[f][2]);
            double rp = cs.ref_val[f];
            if (t == F_INLET || t == F_WALL) {
                uBc.changeType(f, P_FIXED, rv); pBc.changeType(f, P_ZERO_GRADIENT, rp); hBc.changeType(f, P_FIXED, rv);
            } else if (t == F_OUTLET) {
                uBc.changeType(f, P_ZERO_GRADIENT, rv); pBc.changeType(f, P_FIXED, rp); hBc.changeType(f, P_ZERO_GRADIENT, rv);
            } else if (t == F_EMPTY) {
                uBc.changeType(f, P_EMPTY, rv); pBc.changeType(f, P_EMPTY, rp); hBc.changeType(f, P_EMPTY, rv);
            } else if (t == F_ZERO_GRADIENT) {
                uBc.changeType(f, P_ZERO_GRADIENT, rv); pBc.changeType(f, P_ZERO_GRADIENT, rp); hBc.changeType(f, P_ZERO_GRADIENT, rv);
            } else throw std::runtime_error("invalid boundary type");
            dBc.changeType(f, P_ZERO_GRADIENT, 0.);
        }
        nInner = cs.time_accurate ? cs.n_inner : 1;
        omega = cs.omega_u; rho = cs.rho; mu = cs.mu;
        A.allocate(4 * N, 28);
        b.assign(4 * (size_t)N, 0.); x.assign(4 * (size_t)N, 0.);
    }
    int idx(int i, int j, int k, int var) const {  // IndexMap::operator(), one block, every cell active
        if (i < 0 || j < 0 || k < 0 || i >= m.nI || j >= m.nJ || k >= m.nK) return -1;
        return m.cid(i, j, k) + var * N;
    }

    // Coupled::solve (Coupled.cpp:38-50)
    double solve(double dt) {
        u0.c = u.c;
        for (int it = 0; it < nInner; ++it) computeMomentumAndPressure(dt);
        return computeContinuityError();
    }

    // Coupled::computeMomentumAndPressure (Coupled.cpp:54-280), in three parts: the assembly of
    // the block system, its solve and what follows the solve
    void computeMomentumAndPressure(double dt) {
        assemble(dt);
        solveSystem();
        post();
    }

    // Coupled.cpp:54-245: momentum rows, d and its faces, continuity rows
    void assemble(double dt) {
        uStar.c = u.c;
        const int dI[7] = {0, 1, -1, 0, 0, 0, 0}, dJ[7] = {0, 0, 0, 1, -1, 0, 0}, dK[7] = {0, 0, 0, 0, 0, 1, -1};
        // momentum rows
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    double a0P = cs.time_accurate ? rho * m.vol[c] / dt : 0.;
                    double FE = mf.faceE(i, j, k), FW = mf.faceW(i, j, k), FN = mf.faceN(i, j, k), FS = mf.faceS(i, j, k),
                           FT = mf.faceT(i, j, k), FB = mf.faceB(i, j, k);
                    double a[14];
                    a[0] = (std::max(FE, 0.) + mu * m.d[0][c] - std::min(FW, 0.) + mu * m.d[1][c] + std::max(FN, 0.) + mu * m.d[2][c] -
                            std::min(FS, 0.) + mu * m.d[3][c] + std::max(FT, 0.) + mu * m.d[4][c] - std::min(FB, 0.) + mu * m.d[5][c] +
                            a0P) / omega;
                    a[1] = std::min(FE, 0.) - mu * m.d[0][c];
                    a[2] = -std::max(FW, 0.) - mu * m.d[1][c];
                    a[3] = std::min(FN, 0.) - mu * m.d[2][c];
                    a[4] = -std::max(FS, 0.) - mu * m.d[3][c];
                    a[5] = std::min(FT, 0.) - mu * m.d[4][c];
                    a[6] = -std::max(FB, 0.) - mu * m.d[5][c];
                    V3 bu = a0P * u0.c[c];
                    bu += (1. - omega) * a[0] * uStar.c[c];
                    uBc.setImplicit(i, j, k, a, bu);
                    for (int q = 0; q < 3; ++q) {
                        double g[6], s[6];
                        for (int f = 0; f < 6; ++f) { g[f] = m.g[f][c]; s[f] = comp(m.S(f, i, j, k), q); }
                        a[7] = g[0] * s[0] + g[1] * s[1] + g[2] * s[2] + g[3] * s[3] + g[4] * s[4] + g[5] * s[5];
                        for (int f = 0; f < 6; ++f) a[8 + f] = (1. - g[f]) * s[f];
                        int cols[14];
                        for (int e = 0; e < 7; ++e) {
                            cols[e] = idx(i + dI[e], j + dJ[e], k + dK[e], q);
                            cols[7 + e] = idx(i + dI[e], j + dJ[e], k + dK[e], 3);
                        }
                        pBc.setImplicit(i, j, k, &a[7], comp(bu, q));
                        A.setRow(idx(i, j, k, q), 14, cols, a);
                        b[idx(i, j, k, q)] = comp(bu, q);
                    }
                    d.c[c] = m.vol[c] / a[0];
                }
        dBc.setBoundaries();
        interpolateInteriorFaces(m, d);
        // continuity rows
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    int rowNo = idx(i, j, k, 3);
                    double bp = 0.;
                    double a[7];
                    int cols[7];
                    for (int q = 0; q < 3; ++q) {
                        double g[6], s[6];
                        for (int f = 0; f < 6; ++f) { g[f] = m.g[f][c]; s[f] = comp(m.S(f, i, j, k), q); }
                        a[0] = rho * g[0] * s[0] + rho * g[1] * s[1] + rho * g[2] * s[2] + rho * g[3] * s[3] + rho * g[4] * s[4] +
                               rho * g[5] * s[5];
                        for (int f = 0; f < 6; ++f) a[1 + f] = rho * (1. - g[f]) * s[f];
                        for (int e = 0; e < 7; ++e) cols[e] = idx(i + dI[e], j + dJ[e], k + dK[e], q);
                        V3 bu = zero3();
                        uBc.setImplicit(i, j, k, a, bu);
                        bp += comp(bu, q);
                        A.setRow(rowNo, 7, cols, a);
                    }
                    // pressure part: the Rhie-Chow interpolation
                    double rd[6] = {rho * d.faceE(i, j, k) * m.d[0][c], rho * d.faceW(i, j, k) * m.d[1][c],
                                    rho * d.faceN(i, j, k) * m.d[2][c], rho * d.faceS(i, j, k) * m.d[3][c],
                                    rho * d.faceT(i, j, k) * m.d[4][c], rho * d.faceB(i, j, k) * m.d[5][c]};
                    a[0] = rd[0] + rd[1] + rd[2] + rd[3] + rd[4] + rd[5];
                    for (int f = 0; f < 6; ++f) a[1 + f] = -rd[f];
                    for (int e = 0; e < 7; ++e) cols[e] = idx(i + dI[e], j + dJ[e], k + dK[e], 3);
                    bp -= rho * d.faceE(i, j, k) * dot(gradP.faceE(i, j, k), m.SE(i, j, k)) +
                          rho * d.faceW(i, j, k) * dot(gradP.faceW(i, j, k), m.SW(i, j, k)) +
                          rho * d.faceN(i, j, k) * dot(gradP.faceN(i, j, k), m.SN(i, j, k)) +
                          rho * d.faceS(i, j, k) * dot(gradP.faceS(i, j, k), m.SS(i, j, k)) +
                          rho * d.faceT(i, j, k) * dot(gradP.faceT(i, j, k), m.ST(i, j, k)) +
                          rho * d.faceB(i, j, k) * dot(gradP.faceB(i, j, k), m.SB(i, j, k));
                    pBc.setImplicit(i, j, k, a, bp);
                    A.setRow(rowNo, 7, cols, a);
                    b[rowNo] = bp;
                }
    }

    // Coupled.cpp:247-249
    void solveSystem() { st = kspSolve(cs.mom_method, A, b, x, cs.mom_rtol, cs.maxit, cs.mom_atol); }

    // Coupled.cpp:251-278
    void post() {
        for (int c = 0; c < N; ++c) {
            u.c[c] = v3(x[c], x[c + N], x[c + 2 * (size_t)N]);
            p.c[c] = x[c + 3 * (size_t)N];
        }
        pBc.setBoundaries();
        cellGradients(m, p, gradP);
        interpolateInteriorFaces(m, gradP);
        for (int c = 0; c < N; ++c) h.c[c] = u.c[c] + d.c[c] * gradP.c[c];
        hBc.setBoundaries();
        interpolateInteriorFaces(m, h);
        uBc.setBoundaries();
        rhieChowInterpolateFaces();
    }

    // Coupled::rhieChowInterpolateFaces (Coupled.cpp:282-314): no rho in the face flux
    void rhieChowInterpolateFaces() {
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    int c = m.cid(i, j, k);
                    if (i == 0)
                        mf.faceW(i, j, k) = -dot(h.faceW(i, j, k), m.SW(i, j, k)) - d.faceW(i, j, k) * (p.at(i - 1, j, k) - p.c[c]) * m.d[1][c];
                    if (j == 0)
                        mf.faceS(i, j, k) = -dot(h.faceS(i, j, k), m.SS(i, j, k)) - d.faceS(i, j, k) * (p.at(i, j - 1, k) - p.c[c]) * m.d[3][c];
                    if (k == 0)
                        mf.faceB(i, j, k) = -dot(h.faceB(i, j, k), m.SB(i, j, k)) - d.faceB(i, j, k) * (p.at(i, j, k - 1) - p.c[c]) * m.d[5][c];
                    mf.faceE(i, j, k) = dot(h.faceE(i, j, k), m.SE(i, j, k)) - d.faceE(i, j, k) * (p.at(i + 1, j, k) - p.c[c]) * m.d[0][c];
                    mf.faceN(i, j, k) = dot(h.faceN(i, j, k), m.SN(i, j, k)) - d.faceN(i, j, k) * (p.at(i, j + 1, k) - p.c[c]) * m.d[2][c];
                    mf.faceT(i, j, k) = dot(h.faceT(i, j, k), m.ST(i, j, k)) - d.faceT(i, j, k) * (p.at(i, j, k + 1) - p.c[c]) * m.d[4][c];
                }
    }

    // Coupled::computeContinuityError (Coupled.cpp:316-339)
    double computeContinuityError() {
        double mx = 0.;
        for (int k = 0; k < m.nK; ++k)
            for (int j = 0; j < m.nJ; ++j)
                for (int i = 0; i < m.nI; ++i) {
                    double e = std::fabs(mf.faceE(i, j, k) - mf.faceW(i, j, k) + mf.faceN(i, j, k) - mf.faceS(i, j, k) +
                                         mf.faceT(i, j, k) - mf.faceB(i, j, k)) / m.vol[m.cid(i, j, k)];
                    if (e > mx) mx = e;
                }
        return mx;
    }
};

}  // namespace orc

// ----------------------------------------------------------------------------
// C ABI for ctypes
// ----------------------------------------------------------------------------
static thread_local std::string g_err;

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int oracle_get_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void* oracle_create(const double* xyz, int nNI, int nNJ, int nNK, const OracleCase* cs) {
    try {
        auto* s = new orc::Solver();
        s->init(xyz, nNI, nNJ, nNK, *cs);
        return s;
    } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}
void oracle_destroy(void* h) { delete static_cast<orc::Solver*>(h); }

int oracle_solve(void* h, double dt, double* continuity) {
    try { *continuity = static_cast<orc::Solver*>(h)->solve(dt); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// Individual phases (names follow Simple.h:44-51, IbPiso.h:46-47).
int oracle_phase(void* hh, const char* name, double dt) {
    auto* s = static_cast<orc::Solver*>(hh);
    try {
        std::string n(name);
        if (n == "save_u0") s->uf0.c = s->u.c;
        else if (n == "assemble_momentum") s->assembleMomentum(dt);
        else if (n == "solve_momentum") s->solveMomentum();
        else if (n == "momentum_post") s->momentumPost();
        else if (n == "assemble_pcorr") s->assemblePCorr();
        else if (n == "solve_pcorr") s->solvePCorr();
        else if (n == "correct") s->correct();
        else if (n == "continuity") s->computeContinuityError();
        else if (n == "courant") s->computeCourantNumber(dt);
        else if (n == "ib_field") s->computeIbField();
        else if (n == "ib_coeffs") s->computeIbCoeffs();
        else if (n == "compute_h") {   // the h scatter of Simple.cpp:198-203 for the current u, d, grad p
            for (int c = 0; c < s->N; ++c) {
                if (s->inactive(c)) continue;
                for (int q = 0; q < 3; ++q)
                    orc::comp(s->h.c[c], q) = s->active(c) ? orc::comp(s->u.c[c], q) + s->d.c[c] * orc::comp(s->gradP.c[c], q)
                                                           : orc::comp(s->u.c[c], q);
            }
        }
        else if (n == "pcorr_post") {  // Simple.cpp:295-298 for the current p'
            s->pcBc.setBoundaries();
            orc::interpolateInteriorFaces(s->m, s->pc);
            orc::cellGradients(s->m, s->pc, s->gradPC);
        }
        else { g_err = "unknown phase " + n; return 2; }
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// Scalar statistics: continuity, courant, momentum iterations (sum of 3), last p' iterations,
// total p' iterations, p' solves, worst p' relative residual, worst momentum residual, ghosts, rows
// The assembled system `which` (0 momentum, 1 pressure correction) as the rows were set, in
// the row numbering of IndexMap: rows, row width, entries per row, columns, values (row-major,
// width per row); b receives right-hand side `comp` (the momentum component, 0 for p').  Called
// with null arrays it returns the row count and width only.  For pinning against the
// reference's own assembly (its KSPSolve inputs), right after an assemble phase.
int oracle_system(void* hh, int which, int comp, int* width, int* cnt, int* col, double* val, double* b) {
    auto* s = static_cast<orc::Solver*>(hh);
    if (which < 0 || which > 1 || comp < 0 || comp > 2) return -1;
    const orc::Rows& A = s->A[which];
    if (width) *width = A.width;
    if (cnt) std::memcpy(cnt, A.cnt.data(), sizeof(int) * A.cnt.size());
    if (col) std::memcpy(col, A.col.data(), sizeof(int) * A.col.size());
    if (val) std::memcpy(val, A.val.data(), sizeof(double) * A.val.size());
    if (b) std::memcpy(b, s->bv[comp].data(), sizeof(double) * s->bv[comp].size());
    return A.n;
}

void oracle_stats(void* hh, double* out) {
    auto* s = static_cast<orc::Solver*>(hh);
    out[0] = s->continuity; out[1] = s->courant; out[2] = s->momItersTotal; out[3] = s->pItersLast;
    out[4] = s->pItersTotal; out[5] = s->nPSolves; out[6] = s->pResMax; out[7] = s->momResMax;
    out[8] = s->nGhost; out[9] = s->nRows;
}

// Copy a named array out (dir 0) or in (dir 1).  count is in doubles.  Returns the
// element count in doubles, or -1 for an unknown name.
long oracle_array(void* hh, const char* name, double* buf, long count, int dir) {
    auto* s = static_cast<orc::Solver*>(hh);
    std::string n(name);
    auto vecv = [&](std::vector<orc::V3>& v) -> long {
        long need = (long)v.size() * 3;
        if (buf && count >= need) {
            for (size_t q = 0; q < v.size(); ++q) {
                if (dir == 0) { buf[3 * q] = v[q].x; buf[3 * q + 1] = v[q].y; buf[3 * q + 2] = v[q].z; }
                else v[q] = orc::v3(buf[3 * q], buf[3 * q + 1], buf[3 * q + 2]);
            }
        }
        return need;
    };
    auto vecd = [&](std::vector<double>& v) -> long {
        long need = (long)v.size();
        if (buf && count >= need) {
            if (dir == 0) std::memcpy(buf, v.data(), sizeof(double) * need);
            else std::memcpy(v.data(), buf, sizeof(double) * need);
        }
        return need;
    };
    orc::Mesh& m = s->m;
    if (n == "u") return vecv(s->u.c);
    if (n == "h") return vecv(s->h.c);
    if (n == "gradP") return vecv(s->gradP.c);
    if (n == "gradPCorr") return vecv(s->gradPC.c);
    if (n == "uFaceI") return vecv(s->u.fI);
    if (n == "uFaceJ") return vecv(s->u.fJ);
    if (n == "uFaceK") return vecv(s->u.fK);
    if (n == "gradU") {   // N x 9, row-major xx xy xz / yx yy yz / zx zy zz (non-orthogonal correction only)
        long need = 9L * (long)s->gradU.c.size();
        if (buf && count >= need && dir == 0)
            for (size_t q = 0; q < s->gradU.c.size(); ++q) std::memcpy(buf + 9 * q, s->gradU.c[q].m, 9 * sizeof(double));
        return need;
    }
    if (n == "u0") return vecv(s->uf0.c);
    if (n == "p") return vecd(s->p.c);
    if (n == "pCorr") return vecd(s->pc.c);
    if (n == "d") return vecd(s->d.c);
    if (n == "massFlow") return vecd(s->mf.c);
    if (n == "massFlowI") return vecd(s->mf.fI);
    if (n == "massFlowJ") return vecd(s->mf.fJ);
    if (n == "massFlowK") return vecd(s->mf.fK);
    if (n.rfind("pPatch", 0) == 0) return vecd(s->p.patch[n[6] - '0']);
    if (n == "vol") return vecd(m.vol);
    if (n == "cc") return vecv(m.cc);
    if (n == "SI") return vecv(m.fnI);
    if (n == "SJ") return vecv(m.fnJ);
    if (n == "SK") return vecv(m.fnK);
    if (n == "fcI") return vecv(m.fcI);
    if (n == "fcJ") return vecv(m.fcJ);
    if (n == "fcK") return vecv(m.fcK);
    if (n.rfind("dmet", 0) == 0) return vecd(m.d[n[4] - '0']);
    if (n.rfind("cvec", 0) == 0) return vecv(m.cvec[n[4] - '0']);
    if (n.rfind("gmet", 0) == 0) return vecd(m.g[n[4] - '0']);
    if (n == "momA") return vecd(s->momA);
    if (n == "momB") return vecv(s->momB);
    if (n == "pcA") return vecd(s->pcA);
    if (n == "pcB") return vecd(s->pcB);
    if (n == "ibBeta") return vecd(s->ibBeta);
    if (n == "status") {
        long need = s->N;
        if (buf && count >= need && dir == 0) for (int q = 0; q < s->N; ++q) buf[q] = s->status[q];
        return need;
    }
    if (n == "rowOfCell") {
        long need = s->N;
        if (buf && count >= need && dir == 0) for (int q = 0; q < s->N; ++q) buf[q] = s->row[q];
        return need;
    }
    if (n == "A0coo" || n == "A1coo") {   // (row, col, value) triplets of a system matrix
        orc::Rows& R = s->A[n[1] - '0'];
        long nnz = 0;
        for (int r = 0; r < R.n; ++r) nnz += R.cnt[r];
        long need = 3 * nnz;
        if (buf && count >= need && dir == 0) {
            long q = 0;
            for (int r = 0; r < R.n; ++r)
                for (int e = 0; e < R.cnt[r]; ++e) {
                    buf[q++] = r; buf[q++] = R.col[(size_t)r * R.width + e]; buf[q++] = R.val[(size_t)r * R.width + e];
                }
        }
        return need;
    }
    if (n == "b0") return vecd(s->bv[0]);
    if (n == "ibStencil") {
        long need = (long)s->ibStencil.size();
        if (buf && count >= need && dir == 0) for (size_t q = 0; q < s->ibStencil.size(); ++q) buf[q] = s->ibStencil[q];
        return need;
    }
    return -1;
}

// Stand-alone Krylov solve on a 7-point system given as 7 per-row coefficient arrays
// (aP, aE, aW, aN, aS, aT, aB; zero where a neighbour does not exist) on an
// nI x nJ x nK lattice.  Used to check the device Krylov kernels.
int oracle_ksp7(int nI, int nJ, int nK, const double* coef7, const double* b, double* x,
                int method, double rtol, int maxit, int* iters, double* rel_res, double atol) {
    int n = nI * nJ * nK;
    orc::Rows A; A.allocate(n, 7);
    for (int k = 0; k < nK; ++k)
        for (int j = 0; j < nJ; ++j)
            for (int i = 0; i < nI; ++i) {
                int c = (k * nJ + j) * nI + i;
                int cols[7] = {c, i + 1 < nI ? c + 1 : -1, i > 0 ? c - 1 : -1, j + 1 < nJ ? c + nI : -1, j > 0 ? c - nI : -1,
                               k + 1 < nK ? c + nI * nJ : -1, k > 0 ? c - nI * nJ : -1};
                double vals[7];
                for (int q = 0; q < 7; ++q) vals[q] = coef7[(size_t)q * n + c];
                A.setRow(c, 7, cols, vals);
            }
    std::vector<double> bb(b, b + n), xx(n, 0.);
    orc::KspStats st = orc::kspSolve(method, A, bb, xx, rtol, maxit, atol);
    std::memcpy(x, xx.data(), sizeof(double) * n);
    *iters = st.iters; *rel_res = st.rel_res;
    return st.status;
}

// Known-answer helpers for the reference's own unit tests.
double oracle_hex_volume(const double* p24) {
    orc::V3 p[8]; for (int q = 0; q < 8; ++q) p[q] = orc::v3(p24[3 * q], p24[3 * q + 1], p24[3 * q + 2]);
    return orc::hexVolume(p);
}
void oracle_hex_centroid(const double* p24, double* out) {
    orc::V3 p[8]; for (int q = 0; q < 8; ++q) p[q] = orc::v3(p24[3 * q], p24[3 * q + 1], p24[3 * q + 2]);
    orc::V3 c = orc::hexCentroid(p); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
double oracle_quad_area(const double* p12) {
    orc::V3 p[4]; for (int q = 0; q < 4; ++q) p[q] = orc::v3(p12[3 * q], p12[3 * q + 1], p12[3 * q + 2]);
    return orc::quadArea(p);
}
int oracle_inside_hex(const double* pt, const double* p24) {
    orc::V3 p[8]; for (int q = 0; q < 8; ++q) p[q] = orc::v3(p24[3 * q], p24[3 * q + 1], p24[3 * q + 2]);
    return orc::insideHex(orc::v3(pt[0], pt[1], pt[2]), p) ? 1 : 0;
}
void oracle_trilinear(const double* p24, const double* ip, double* beta) {
    orc::V3 p[8]; for (int q = 0; q < 8; ++q) p[q] = orc::v3(p24[3 * q], p24[3 * q + 1], p24[3 * q + 2]);
    orc::trilinearCoeffs(p, orc::v3(ip[0], ip[1], ip[2]), beta);
}
void oracle_nearest_intersect(double radius, const double* center, const double* pt, double* out) {
    orc::V3 c = orc::v3(center[0], center[1], center[2]);
    orc::V3 l = orc::unitv(orc::v3(pt[0], pt[1], pt[2]) - c);
    orc::V3 r = c + radius * l;
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// Coupled solver (kind is ignored; the boundary types, rho, mu, timeAccurate, relaxation of
// momentum, inner iterations and the Krylov settings mom_method / mom_rtol / maxit are used).
void* oracle_coupled_create(const double* xyz, int nNI, int nNJ, int nNK, const OracleCase* cs) {
    try {
        auto* s = new orc::Coupled();
        s->init(xyz, nNI, nNJ, nNK, *cs);
        return s;
    } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}
void oracle_coupled_destroy(void* h) { delete static_cast<orc::Coupled*>(h); }
int oracle_coupled_solve(void* h, double dt, double* continuity) {
    try { *continuity = static_cast<orc::Coupled*>(h)->solve(dt); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return 1; }
}
// Krylov iterations, relative residual and status of the last coupled solve
void oracle_coupled_stats(void* h, double* out) {
    auto* s = static_cast<orc::Coupled*>(h);
    out[0] = s->st.iters; out[1] = s->st.rel_res; out[2] = s->st.status;
}
// "u" (N x 3), "p", "d", "gradP" (N x 3), "massFlowI/J/K", "b" (4N); dir 0 out, 1 in
long oracle_coupled_array(void* hh, const char* name, double* buf, long count, int dir) {
    auto* s = static_cast<orc::Coupled*>(hh);
    std::string n(name);
    auto vecd = [&](std::vector<double>& v) -> long {
        long need = (long)v.size();
        if (buf && count >= need) {
            if (dir == 0) std::memcpy(buf, v.data(), sizeof(double) * need);
            else std::memcpy(v.data(), buf, sizeof(double) * need);
        }
        return need;
    };
    auto vecv = [&](std::vector<orc::V3>& v) -> long {
        long need = (long)v.size() * 3;
        if (buf && count >= need) {
            for (size_t q = 0; q < v.size(); ++q) {
                if (dir == 0) { buf[3 * q] = v[q].x; buf[3 * q + 1] = v[q].y; buf[3 * q + 2] = v[q].z; }
                else v[q] = orc::v3(buf[3 * q], buf[3 * q + 1], buf[3 * q + 2]);
            }
        }
        return need;
    };
    if (n == "u") return vecv(s->u.c);
    if (n == "gradP") return vecv(s->gradP.c);
    if (n == "p") return vecd(s->p.c);
    if (n == "d") return vecd(s->d.c);
    if (n == "massFlowI") return vecd(s->mf.fI);
    if (n == "massFlowJ") return vecd(s->mf.fJ);
    if (n == "massFlowK") return vecd(s->mf.fK);
    if (n == "b") return vecd(s->b);
    if (n == "x") return vecd(s->x);
    if (n == "h") return vecv(s->h.c);
    if (n == "u0") return vecv(s->u0.c);
    return -1;
}

// One part of Coupled::computeMomentumAndPressure: "save_u0" (the start of Coupled::solve),
// "assemble", "solve" or "post".
int oracle_coupled_phase(void* hh, const char* name, double dt) {
    auto* s = static_cast<orc::Coupled*>(hh);
    try {
        std::string n(name);
        if (n == "save_u0") s->u0.c = s->u.c;
        else if (n == "assemble") s->assemble(dt);
        else if (n == "solve") s->solveSystem();
        else if (n == "post") s->post();
        else { g_err = "unknown phase " + n; return 2; }
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// The assembled block system as its rows were set (the layout of oracle_system); returns the
// row count (4 N).
int oracle_coupled_system(void* hh, int* width, int* cnt, int* col, double* val) {
    auto* s = static_cast<orc::Coupled*>(hh);
    const orc::Rows& A = s->A;
    if (width) *width = A.width;
    if (cnt) std::memcpy(cnt, A.cnt.data(), sizeof(int) * A.cnt.size());
    if (col) std::memcpy(col, A.col.data(), sizeof(int) * A.col.size());
    if (val) std::memcpy(val, A.val.data(), sizeof(double) * A.val.size());
    return A.n;
}

// Diffusion solver.  types: per face E W N S T B, 0 fixed, 1 zeroGradient, 2 empty; refs:
// Boundaries.<face>.refValue; phi0: uniform initial phi.
void* oracle_diffusion_create(const double* xyz, int nNI, int nNJ, int nNK, const int* types, const double* refs, int time_accurate,
                              double phi0, int method, double rtol, int maxit) {
    try {
        auto* s = new orc::Diffusion();
        s->init(xyz, nNI, nNJ, nNK, types, refs, time_accurate, phi0, method, rtol, maxit);
        return s;
    } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}
void oracle_diffusion_destroy(void* h) { delete static_cast<orc::Diffusion*>(h); }
int oracle_diffusion_solve(void* h, double dt, double* residual_inf) {
    try { *residual_inf = static_cast<orc::Diffusion*>(h)->solve(dt); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return 1; }
}
// Krylov iterations and true relative residual of the last solve
void oracle_diffusion_stats(void* h, double* out) {
    auto* s = static_cast<orc::Diffusion*>(h);
    out[0] = s->iters; out[1] = s->relRes;
}
// "phi", "gradPhi" (N x 3), "phiFaceI/J/K", "phiPatch0".."phiPatch5", "A" (N x 7: aP aE aW aN
// aS aT aB as assembled), "b"; dir 0 out, 1 in.  Returns the count in doubles, -1 if unknown.
long oracle_diffusion_array(void* hh, const char* name, double* buf, long count, int dir) {
    auto* s = static_cast<orc::Diffusion*>(hh);
    std::string n(name);
    auto vecd = [&](std::vector<double>& v) -> long {
        long need = (long)v.size();
        if (buf && count >= need) {
            if (dir == 0) std::memcpy(buf, v.data(), sizeof(double) * need);
            else std::memcpy(v.data(), buf, sizeof(double) * need);
        }
        return need;
    };
    if (n == "phi") return vecd(s->phi.c);
    if (n == "phiFaceI") return vecd(s->phi.fI);
    if (n == "phiFaceJ") return vecd(s->phi.fJ);
    if (n == "phiFaceK") return vecd(s->phi.fK);
    if (n.rfind("phiPatch", 0) == 0 && n.size() == 9 && n[8] >= '0' && n[8] <= '5') return vecd(s->phi.patch[n[8] - '0']);
    if (n == "b") return vecd(s->b);
    if (n == "gradPhi") {
        long need = 3L * s->N;
        if (buf && count >= need && dir == 0)
            for (int q = 0; q < s->N; ++q) { buf[3 * q] = s->gradPhi.c[q].x; buf[3 * q + 1] = s->gradPhi.c[q].y; buf[3 * q + 2] = s->gradPhi.c[q].z; }
        return need;
    }
    if (n == "A") {
        long need = 7L * s->N;
        if (buf && count >= need && dir == 0) {
            const orc::Mesh& m = s->m;
            for (int c = 0; c < s->N; ++c) {
                int i = c % m.nI, j = (c / m.nI) % m.nJ, k = c / (m.nI * m.nJ);
                const int nb[7] = {c, i < m.uI() ? c + 1 : -2, i > 0 ? c - 1 : -2, j < m.uJ() ? c + m.nI : -2,
                                   j > 0 ? c - m.nI : -2, k < m.uK() ? c + m.nI * m.nJ : -2, k > 0 ? c - m.nI * m.nJ : -2};
                for (int q = 0; q < 7; ++q) {
                    double v = 0.;
                    for (int p = 0; p < s->A.cnt[c]; ++p)
                        if (s->A.col[(size_t)c * s->A.width + p] == nb[q]) v = s->A.val[(size_t)c * s->A.width + p];
                    buf[7 * (size_t)c + q] = v;
                }
            }
        }
        return need;
    }
    return -1;
}

}  // extern "C"
