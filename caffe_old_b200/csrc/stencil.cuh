// Stencil operators shared by the Krylov kernels: y = A x for the 7-point (momentum), the
// symmetric 7-point (pressure correction) and the compressed-row operators, with the
// immersed-boundary ghost rows, and the diagonal each preconditioner inverts.
#pragma once
#include "krylov.cuh"

namespace cb {

__device__ __forceinline__ int ghost_index(const GhostRows& gh, long long c) {
    int lo = 0, hi = gh.n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(gh.cell + mid) < c) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <int NR, class X>
__device__ __forceinline__ void ghost_fix(const GhostRows& gh, long long c, X&& x, double (&y)[NR]) {
    uint32_t w = __ldg(gh.bits + (c >> 5));
    if ((w >> (c & 31)) & 1u) {
        int g = ghost_index(gh, c);
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            double s = 0.;
            for (int m = 0; m < 9; ++m) {
                int col = __ldg(gh.col + 9 * g + m);
                if (col >= 0) s += __ldg(gh.val + 9 * g + m) * x(q, (long long)col);
            }
            y[q] = s;
        }
    }
}

template <int NR, class X>
__device__ __forceinline__ void apply(const Op7& A, long long c, X&& x, double (&y)[NR]) {
    double aP = __ldg(A.a[0] + c), aE = __ldg(A.a[1] + c), aW = __ldg(A.a[2] + c), aN = __ldg(A.a[3] + c);
    double aS = __ldg(A.a[4] + c), aT = __ldg(A.a[5] + c), aB = __ldg(A.a[6] + c);
#pragma unroll
    for (int q = 0; q < NR; ++q)
        y[q] = aP * x(q, c) + aE * x(q, c + 1) + aW * x(q, c - 1) + aN * x(q, c + A.nI) + aS * x(q, c - A.nI)
               + aT * x(q, c + A.nIJ) + aB * x(q, c - A.nIJ);
    if (A.gh.n > 0) ghost_fix<NR>(A.gh, c, x, y);
}

template <int NR, class X>
__device__ __forceinline__ void apply(const OpSym& A, long long c, X&& x, double (&y)[NR]) {
    double aP = __ldg(A.aP + c), aE = __ldg(A.aE + c), aW = __ldg(A.aE + c - 1), aN = __ldg(A.aN + c);
    double aS = __ldg(A.aN + c - A.nI), aT = __ldg(A.aT + c), aB = __ldg(A.aT + c - A.nIJ);
#pragma unroll
    for (int q = 0; q < NR; ++q)
        y[q] = aP * x(q, c) + aE * x(q, c + 1) + aW * x(q, c - 1) + aN * x(q, c + A.nI) + aS * x(q, c - A.nI)
               + aT * x(q, c + A.nIJ) + aB * x(q, c - A.nIJ);
    if (A.gh.n > 0) ghost_fix<NR>(A.gh, c, x, y);
}

template <int NR, class X>
__device__ __forceinline__ void apply(const OpCSR& A, long long c, X&& x, double (&y)[NR]) {
    const int p0 = __ldg(A.ptr + c), p1 = __ldg(A.ptr + c + 1);
#pragma unroll
    for (int q = 0; q < NR; ++q) y[q] = 0.;
    for (int p = p0; p < p1; ++p) {
        const double v = __ldg(A.val + p);
        const long long e = __ldg(A.col + p);
#pragma unroll
        for (int q = 0; q < NR; ++q) y[q] += v * x(q, e);
    }
}

__device__ __forceinline__ double diag_of(const Op7& A, long long c) { return A.a[0][c]; }
__device__ __forceinline__ double diag_of(const OpCSR& A, long long c) {
    const int d = A.diag[c];
    return d >= 0 ? A.val[d] : 0.;
}
__device__ __forceinline__ double diag_of(const OpSym& A, long long c) { return A.aP[c]; }

}  // namespace cb
