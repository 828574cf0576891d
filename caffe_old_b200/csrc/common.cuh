// Shared definitions of the B200 device library: lattice indexing, the views the
// kernels receive, error handling.
//
// Layout in HBM (all float64 unless noted, i fastest, as Array3D):
//   cell arrays      N   = nI*nJ*nK,        c  = (k*nJ + j)*nI + i
//   I-face arrays    nFI = (nI+1)*nJ*nK,    fI = (k*nJ + j)*(nI+1) + i   (face i = west face of cell i)
//   J-face arrays    nFJ = nI*(nJ+1)*nK,    fJ = (k*(nJ+1) + j)*nI + i
//   K-face arrays    nFK = nI*nJ*(nK+1),    fK = (k*nJ + j)*nI + i
//   3-vectors are stored as three planes (x plane, y plane, z plane) of the same length.
//   Cell arrays carry a zero halo of H >= nI*nJ elements before and after each plane (plane
//   stride PS = N + 2H; element c of plane q at base + q*PS, base pointing at element 0), so
//   stencil loads at c +- 1, nI, nI*nJ never leave the allocation and need no index math;
//   a coefficient that couples to a neighbour outside the lattice is stored as zero.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace cb {

// ---------------------------------------------------------------- error handling
void set_error(const std::string& msg);
void clear_error();
std::string cuda_msg(cudaError_t e, const char* what, const char* file, int line);

#define CB_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::cb::set_error(::cb::cuda_msg(_e, #call, __FILE__, __LINE__));             \
            return 1;                                                                   \
        }                                                                               \
    } while (0)

#define CB_CHECK_LAUNCH()                                                               \
    do {                                                                                \
        cudaError_t _e = cudaGetLastError();                                            \
        if (_e != cudaSuccess) {                                                        \
            ::cb::set_error(::cb::cuda_msg(_e, "kernel launch", __FILE__, __LINE__));   \
            return 1;                                                                   \
        }                                                                               \
    } while (0)

// ---------------------------------------------------------------- enums (mirror caffe_b200.h)
enum PType { P_FIXED = 0, P_ZERO_GRADIENT = 1, P_EMPTY = 2 };
enum FlowType { F_INLET = 0, F_OUTLET = 1, F_WALL = 2, F_EMPTY = 3, F_ZERO_GRADIENT = 4 };
enum CellStatus { ST_ACTIVE = 0, ST_GHOST = 1, ST_INACTIVE = 2 };

// ---------------------------------------------------------------- lattice
struct Lat {
    int nI, nJ, nK;
    long long N, nFI, nFJ, nFK;
    long long nIJ;
    long long H;    // zero halo before and after every cell array (>= nIJ), so c +- 1, nI, nIJ is addressable
    long long PS;   // plane stride of cell arrays: N + 2H
    __host__ __device__ __forceinline__ long long cid(int i, int j, int k) const { return ((long long)k * nJ + j) * nI + i; }
    __host__ __device__ __forceinline__ long long fiI(int i, int j, int k) const { return ((long long)k * nJ + j) * (nI + 1) + i; }
    __host__ __device__ __forceinline__ long long fiJ(int i, int j, int k) const { return ((long long)k * (nJ + 1) + j) * nI + i; }
    __host__ __device__ __forceinline__ long long fiK(int i, int j, int k) const { return ((long long)k * nJ + j) * nI + i; }
    __host__ __device__ __forceinline__ void ijk(long long c, int& i, int& j, int& k) const {
        i = (int)(c % nI);
        long long t = c / nI;
        j = (int)(t % nJ);
        k = (int)(t / nJ);
    }
};

static inline Lat make_lat(int nI, int nJ, int nK) {
    Lat L;
    L.nI = nI; L.nJ = nJ; L.nK = nK;
    L.N = (long long)nI * nJ * nK;
    L.nFI = (long long)(nI + 1) * nJ * nK;
    L.nFJ = (long long)nI * (nJ + 1) * nK;
    L.nFK = (long long)nI * nJ * (nK + 1);
    L.nIJ = (long long)nI * nJ;
    L.H = ((L.nIJ + 31) / 32) * 32;
    L.PS = L.N + 2 * L.H;
    return L;
}

// ---------------------------------------------------------------- geometry view
struct Geo {
    Lat L;
    const double* vol;
    const double* cc;          // 3 planes of N
    const double* S[3];        // S[dir]: 3 planes of nF(dir): face area-normal along +i/+j/+k
    const double* fc[3];       // face centroids, 3 planes
    const double* D[3];        // |S|^2 / (S.r) per face
    const double* cv[3];       // non-orthogonal vectors per face (east-side orientation), 3 planes
};

// Boundary description: per face, the primitive types of u/h and p (p' shares p's types
// with reference value 0, d is zero-gradient everywhere), the reference values and the
// flow type (FlowBoundaryConditions.cpp:44-71, SimpleBoundaryCondition.cpp:3-15).
struct Bc {
    int flow[6];
    int uType[6];
    int pType[6];
    double uRef[6][3];
    double pRef[6];
};

// ---------------------------------------------------------------- small vector helpers
struct d3 { double x, y, z; };
__device__ __forceinline__ d3 mk3(double x, double y, double z) { d3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ d3 ld3(const double* p, long long n, long long idx) { return mk3(p[idx], p[idx + n], p[idx + 2 * n]); }
__device__ __forceinline__ void st3(double* p, long long n, long long idx, d3 v) { p[idx] = v.x; p[idx + n] = v.y; p[idx + 2 * n] = v.z; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static inline int grid_for(long long n, int block) { return (int)((n + block - 1) / block); }

}  // namespace cb
