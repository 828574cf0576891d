// Learned preconditioner in a flexible Krylov solve, and its training on the device.
//
// Preconditioner (additive multilevel with a learned level operator):
//   M(r) = D^-1 r + P_1 w_1,   w_l = gain_l s y_l + P_(l+1) w_(l+1),
//   y_l = (net(u_l / s, mask_l, l) - net(-u_l / s, mask_l, l)) / 2,
//   u_1 = R_1 (D^-1 r),  u_(l+1) = R_(l+1) u_l,
// on active cells (D^-1 r on ghost rows, 0 on inactive cells).  Level l halves every
// direction of level l-1 that is longer than one cell; P is cell-centred trilinear
// prolongation and R = P^T scaled to a cell average; gain_l = 4^l is the factor by which the
// inverse of the Jacobi-scaled operator grows per halving for the modes that level
// resolves; s is the RMS of D^-1 r over the active cells.  One set of network weights (the
// 4-layer tensor-core CNN of cnn.cu) serves every level; its input carries the restricted
// residual, the fraction of active cells and a constant level channel.  The network never
// runs on the cell lattice itself: on the 25M-cell lattice level 1 holds 1/8 of the cells, so
// the network costs a fraction of one fine-lattice sweep while the pyramid reaches the
// smooth error that a 9^3 receptive field cannot.  The network term is odd in the residual
// (the second evaluation negates only the residual channel): a network with biases and
// constant input channels has a part that does not depend on the residual, which would add
// the same vector to every preconditioned direction; the odd form gives M(0) = 0 and
// M(-r) = -M(r) exactly.  Levels finer than the first network level (netFrom) or coarser than
// the last one (netTo) use the
// identity.  Two reference forms use the same code: JACOBI (no levels: M = D^-1, the method
// without the network) and LEVELS (y_l = u_l / s, the pyramid with an identity in place of
// the network).
//
// Solve (learned + mixed precision): FP64 iterative refinement (true residual, update and
// convergence test in FP64) around an FP32 flexible Krylov solve that tolerates a
// preconditioner that changes from one application to the next:
//  * flexible CG (Notay 2000, truncated to one previous direction) for the symmetric p' matrix:
//      p_k = z_k - beta_k p_{k-1},  beta_k = (z_k, q_{k-1}) / (p_{k-1}, q_{k-1}),
//      q_k = A p_k,  alpha_k = (p_k, r_k) / (p_k, q_k),  x += alpha p,  r -= alpha q;
//  * right-preconditioned BiCGStab when immersed-boundary ghost rows make the matrix
//    non-symmetric and M is the fixed linear pyramid (BiCGStab needs a fixed linear
//    preconditioner);
//  * FGMRES(m) with re-orthogonalised classical Gram-Schmidt (CGS2) when the matrix is
//    non-symmetric and the network runs: one restart cycle per FP64 refinement pass.
// The refinement stops with status 2 (the plain FP64 solve then takes over) after three
// passes in a row that each leave more than 90% of the true residual.
// Each iteration is a short fixed sequence of kernels; their dot products go through block
// partials and a one-block finaliser into a device-side scalar record, so the host never
// waits inside an iteration.  Once the record's `done` flag is set every later kernel returns
// at entry; the host looks at the flag every few iterations.
//
// Training: pairs (b, x*) with A x* = b from the plain solver; loss per pair
//   L = ||M(b) - x*||^2_E / ||x*||^2_E
// in the energy norm of -A (the p' matrix is negative definite; with immersed-boundary cells,
// of its active-cell block), gradient dL/dz = 2 (-A)(z - x*) / ||x*||^2_E, carried through the
// prolongations (adjoint: P^T) to every level's network output and back-propagated by the
// tensor-core backward pass; Adam update.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <array>
#include <mutex>
#include <utility>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "cnn.cuh"
#include "krylov.cuh"
#include "learned.cuh"

namespace cb {

namespace {

constexpr int LB = 256;
constexpr int MAXP = 2048;   // partial slots (blocks) per reduction

struct Scal {
    double rr0, rr, tin2;       // inner: initial and current ||r||^2, stop threshold
    double s;                   // RMS of D^-1 r over active cells
    double zq, pq, pr;          // (z, q_prev), (p, q), (p, r)
    double alpha, beta;
    double bb, tol2, rr64;      // outer: ||b||^2, tolerance, current true ||r||^2
    double prev64;              // true ||r||^2 of the previous refinement pass
    double nact;
    double loss;
    double rho, omega, rv, ts, tt;   // flexible BiCGStab: (rhat, r), omega, (rhat, v), (t, s), (t, t)
    int done;                   // inner solve finished
    int odone;                  // outer solve finished
    int iters, outer, status, first;
    int stall;                  // consecutive refinement passes that cut ||r|| by less than 10%
};

__device__ __forceinline__ void block_sums(double* v, int K, double* part) {
    __shared__ double sm[4][LB / 32];
    for (int q = 0; q < K; ++q)
        for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int q = 0; q < K; ++q) sm[q][w] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < K; ++q) {
            double t = 0.;
            for (int u = 0; u < LB / 32; ++u) t += sm[q][u];
            part[(size_t)blockIdx.x * 4 + q] = t;
        }
    }
}

// one block: totals of K partial streams over nblk blocks, in a fixed order
__device__ __forceinline__ void totals(const double* part, int nblk, int K, double* out) {
    __shared__ double sm[4][LB];
    for (int q = 0; q < K; ++q) {
        double t = 0.;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) t += part[(size_t)b * 4 + q];
        sm[q][threadIdx.x] = t;
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int q = 0; q < K; ++q) sm[q][threadIdx.x] += sm[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < K; ++q) out[q] = sm[q][0];
    __syncthreads();
}

// the same totals read past L1 (the partials were written by other blocks of the running kernel)
__device__ __forceinline__ void totals_cg(const double* part, int nblk, int K, double* out) {
    __shared__ double sm[4][LB];
    for (int q = 0; q < K; ++q) {
        double t = 0.;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) t += __ldcg(part + (size_t)b * 4 + q);
        sm[q][threadIdx.x] = t;
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int q = 0; q < K; ++q) sm[q][threadIdx.x] += sm[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < K; ++q) out[q] = sm[q][0];
    __syncthreads();
}

// after block_sums: true in every thread of the block that finished last (its partial and all
// the others' are then in memory); that block resets the counter for the next kernel
__device__ __forceinline__ bool last_block(unsigned* ctr) {
    __shared__ int amLast;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) amLast = atomicAdd(ctr, 1u) == gridDim.x - 1;
    __syncthreads();
    if (amLast) __threadfence();
    return amLast != 0;
}

inline int nblocks(long long N) {
    long long b = (N + LB - 1) / LB;
    return (int)(b < MAXP ? b : MAXP);
}

__device__ __forceinline__ bool is_active(const uint8_t* st, long long c) { return st == nullptr || st[c] == ST_ACTIVE; }
__device__ __forceinline__ bool is_inactive(const uint8_t* st, long long c) { return st != nullptr && st[c] == ST_INACTIVE; }

// 4-cell vector access (cell arrays start 16-byte aligned: the halo H is a multiple of 32)
__device__ __forceinline__ float4 ld4(const float* p, long long q) { return reinterpret_cast<const float4*>(p)[q]; }
__device__ __forceinline__ void st4(float* p, long long q, const float (&v)[4]) {
    reinterpret_cast<float4*>(p)[q] = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void un4(const float4& v, float (&a)[4]) { a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w; }
__device__ __forceinline__ void st_flags4(const uint8_t* st, long long q, uint8_t (&f)[4]) {
    if (!st) { f[0] = f[1] = f[2] = f[3] = ST_ACTIVE; return; }
    uchar4 v = reinterpret_cast<const uchar4*>(st)[q];
    f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
}

// ---------------------------------------------------------------- outer (FP64) kernels
// r = b - A x (FP64), r32 = float(r), partial ||r||^2
__global__ void __launch_bounds__(LB) outer_residual_kernel(OpSym A, long long N, const double* b, const double* x, float* r32,
                                                            double* part, const Scal* S) {
    if (S->odone) return;
    double v[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        double y = __ldg(A.aP + c) * x[c] + __ldg(A.aE + c) * x[c + 1] + __ldg(A.aE + c - 1) * x[c - 1]
                   + __ldg(A.aN + c) * x[c + A.nI] + __ldg(A.aN + c - A.nI) * x[c - A.nI]
                   + __ldg(A.aT + c) * x[c + A.nIJ] + __ldg(A.aT + c - A.nIJ) * x[c - A.nIJ];
        if (A.gh.n > 0) {
            uint32_t w = __ldg(A.gh.bits + (c >> 5));
            if ((w >> (c & 31)) & 1u) {
                int lo = 0, hi = A.gh.n;
                while (lo < hi) { int mid = (lo + hi) >> 1; if (__ldg(A.gh.cell + mid) < c) lo = mid + 1; else hi = mid; }
                double s = 0.;
                for (int m = 0; m < 9; ++m) { int col = __ldg(A.gh.col + 9 * lo + m); if (col >= 0) s += __ldg(A.gh.val + 9 * lo + m) * x[col]; }
                y = s;
            }
        }
        double r = b[c] - y;
        r32[c] = (float)r;
        v[0] += r * r;
    }
    block_sums(v, 1, part);
}

__global__ void outer_check_kernel(const double* part, int nblk, Scal* S, int max_outer) {
    if (S->odone) return;
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) {
        S->rr64 = t[0];
        if (S->outer == 0 && S->first) { S->bb = t[0]; S->first = 0; }
        bool conv = t[0] <= S->tol2 || !(S->bb > 0.);
        if (t[0] != t[0]) { S->status = 3; conv = true; }
        if (!conv && S->outer >= max_outer) { S->status = 1; conv = true; }
        // stagnation: three refinement passes in a row that leave more than 90% of ||r|| end the
        // solve with status 2, so the plain FP64 solve takes over at once
        if (!conv && S->outer > 0) {
            S->stall = t[0] > 0.81 * S->prev64 ? S->stall + 1 : 0;
            if (S->stall >= 3) { S->status = 2; conv = true; }
        }
        S->prev64 = t[0];
        if (conv) S->odone = 1;
        S->done = S->odone;   // no inner solve when the outer one is finished
        S->outer += conv ? 0 : 1;
    }
}

__global__ void outer_update_kernel(long long N, double* x, const float* e, const Scal* S) {
    if (S->odone) return;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) x[c] = x[c] + (double)e[c];
}

// ---------------------------------------------------------------- inner flexible CG (FP32)
// start of an inner solve: e = 0, p = q = 0, ||r||^2 and ||D^-1 r||^2 over active cells
__global__ void __launch_bounds__(LB) inner_start_kernel(long long N, const float* r, const float* invD, const uint8_t* st, float* e,
                                                         float* p, float* q, double* part, const Scal* S) {
    if (S->done) return;
    double v[3] = {0., 0., 0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float rv = r[c];
        e[c] = 0.f; p[c] = 0.f; q[c] = 0.f;
        double u = (double)__ldg(invD + c) * rv;
        v[0] += (double)rv * rv;
        if (is_active(st, c)) { v[1] += u * u; v[2] += 1.; }
    }
    block_sums(v, 3, part);
}

__global__ void inner_start_finish_kernel(const double* part, int nblk, Scal* S, double eta) {
    if (S->done) return;
    double t[3];
    totals(part, nblk, 3, t);
    if (threadIdx.x == 0) {
        S->rr0 = t[0]; S->rr = t[0];
        S->tin2 = eta * eta * t[0];
        S->nact = t[2];
        S->s = t[2] > 0. ? sqrt(t[1] / t[2]) : 1.;
        if (!(S->s > 0.)) S->s = 1.;
        S->alpha = 0.; S->beta = 0.; S->pq = 1.;
        S->done = !(t[0] > 0.);
    }
}

// ---------------------------------------------------------------- level pyramid
// Cell-centred trilinear prolongation, per direction: fine cell f takes 3/4 of coarse cell
// f/2 and 1/4 of its other neighbour (f/2 - 1 for even f, f/2 + 1 for odd f), clamped to the
// lattice.  A direction of one cell is not coarsened (both weights land on cell 0).
struct Dims3 {
    int n0, n1, n2;
};
__device__ __forceinline__ int pclamp(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
__device__ __forceinline__ float rweight(int f, int I, int nc) {
    int J = pclamp((f & 1) ? (f >> 1) + 1 : (f >> 1) - 1, nc);
    return ((f >> 1) == I ? 0.75f : 0.f) + (J == I ? 0.25f : 0.f);
}
__device__ __forceinline__ float rweight_in(int f, int nf, int I, int nc) { return (f >= 0 && f < nf) ? rweight(f, I, nc) : 0.f; }

// out[I] = scale * (P^T v)[I],  v(f) = (fin ? fin[f] : 1) * (invD ? invD[f] : 1) * (active(f) if st)
// optional: out2 = mul2 * s * out; act0 row (out / s, mask, level channel) for the network.
// One CTA owns RCI x RCJ x RCK coarse cells: it stages the (2 RCI + 2) x (2 RCJ + 2) x
// (2 RCK + 2) fine cells they draw on in shared memory once, then applies the separable
// weights along i, j and k in three passes.
constexpr int RCI = 32, RCJ = 4, RCK = 4;
constexpr int RFI = 2 * RCI + 2, RFJ = 2 * RCJ + 2, RFK = 2 * RCK + 2;

__global__ void __launch_bounds__(256) restrict_kernel(Dims3 fd, Dims3 cd, const float* fin, const float* invD, const uint8_t* st,
                                                       float scale, float* out, float* out2, float mul2, __nv_bfloat16* act0,
                                                       __nv_bfloat16* act0n, const float* maskc, float chan, const Scal* S) {
    if (S && S->done) return;
    __shared__ __align__(16) float s0[RFK][RFJ][RFI];
    __shared__ float t1[RFK][RFJ][RCI];
    __shared__ float t2[RFK][RCJ][RCI];
    __shared__ float wI[RCI][4], wJ[RCJ][4], wK[RCK][4];   // clamped trilinear weights of this tile
    const int I0 = blockIdx.x * RCI, J0 = blockIdx.y * RCJ, K0 = blockIdx.z * RCK;
    const int fi0 = 2 * I0 - 1, fj0 = 2 * J0 - 1, fk0 = 2 * K0 - 1;
    const unsigned fsJ = (unsigned)fd.n0, fsK = (unsigned)fd.n0 * (unsigned)fd.n1;
    if (threadIdx.x < 4 * RCI) {
        int ci = threadIdx.x >> 2, m = threadIdx.x & 3, I = I0 + ci;
        wI[ci][m] = rweight_in(2 * I - 1 + m, fd.n0, I, cd.n0);
    } else if (threadIdx.x < 4 * RCI + 4 * RCJ) {
        int u = threadIdx.x - 4 * RCI, cj = u >> 2, m = u & 3, J = J0 + cj;
        wJ[cj][m] = rweight_in(2 * J - 1 + m, fd.n1, J, cd.n1);
    } else if (threadIdx.x < 4 * RCI + 4 * RCJ + 4 * RCK) {
        int u = threadIdx.x - 4 * RCI - 4 * RCJ, ck = u >> 2, m = u & 3, K = K0 + ck;
        wK[ck][m] = rweight_in(2 * K - 1 + m, fd.n2, K, cd.n2);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    // stage the fine tile: one warp per (j, k) row of RFI cells, lanes along i; a warp issues the
    // loads of RB rows (three 32-cell chunks each) before it stores any, so that on the small
    // coarse levels, where a few CTAs stage everything, each warp has RB rows in flight
    constexpr int CH = (RFI + 31) / 32, RB = 4;
    for (int row0 = warp; row0 < RFJ * RFK; row0 += RB * nwarp) {
        float fv[RB][CH], dv[RB][CH];
        uint8_t sv[RB][CH];
        bool in[RB][CH];
#pragma unroll
        for (int b = 0; b < RB; ++b) {
            const int row = row0 + b * nwarp;
            const int lj = row % RFJ, lk = row / RFJ;
            const int fj = fj0 + lj, fk = fk0 + lk;
            const bool rowIn = row < RFJ * RFK && fj >= 0 && fj < fd.n1 && fk >= 0 && fk < fd.n2;
            const unsigned rowBase = rowIn ? (unsigned)fk * fsK + (unsigned)fj * fsJ : 0u;
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                const int li = lane + 32 * u, fi = fi0 + li;
                in[b][u] = rowIn && li < RFI && fi >= 0 && fi < fd.n0;
                const unsigned f = in[b][u] ? rowBase + (unsigned)fi : 0u;
                fv[b][u] = (in[b][u] && fin) ? __ldg(fin + f) : 1.f;
                dv[b][u] = (in[b][u] && invD) ? __ldg(invD + f) : 1.f;
                sv[b][u] = (in[b][u] && st) ? __ldg(st + f) : (uint8_t)ST_ACTIVE;
            }
        }
#pragma unroll
        for (int b = 0; b < RB; ++b) {
            const int row = row0 + b * nwarp;
            if (row >= RFJ * RFK) continue;
            const int lj = row % RFJ, lk = row / RFJ;
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                const int li = lane + 32 * u;
                if (li < RFI) s0[lk][lj][li] = (in[b][u] && sv[b][u] == ST_ACTIVE) ? fv[b][u] * dv[b][u] : 0.f;
            }
        }
    }
    __syncthreads();
    // blockDim.x is a multiple of RCI * RCJ, so a thread keeps one coarse column ci (pass 1) and one
    // (ci, cj) pair (pass 2) for all its outputs: their weights stay in registers, and pass 1 reads
    // its four fine values as two 8-byte pairs (2 ci is even)
    {
        const int ci = threadIdx.x & (RCI - 1);
        const float w0 = wI[ci][0], w1 = wI[ci][1], w2 = wI[ci][2], w3 = wI[ci][3];
        for (int u = threadIdx.x; u < RFK * RFJ * RCI; u += blockDim.x) {
            const int rest = u / RCI, lj = rest % RFJ, lk = rest / RFJ;
            const float2 a01 = *reinterpret_cast<const float2*>(&s0[lk][lj][2 * ci]);
            const float2 a23 = *reinterpret_cast<const float2*>(&s0[lk][lj][2 * ci + 2]);
            t1[lk][lj][ci] = w0 * a01.x + w1 * a01.y + w2 * a23.x + w3 * a23.y;
        }
    }
    __syncthreads();
    {
        const int ci = threadIdx.x & (RCI - 1), cj = (threadIdx.x / RCI) & (RCJ - 1);
        const float w0 = wJ[cj][0], w1 = wJ[cj][1], w2 = wJ[cj][2], w3 = wJ[cj][3];
        for (int u = threadIdx.x; u < RFK * RCJ * RCI; u += blockDim.x) {
            const int lk = u / (RCI * RCJ);
            t2[lk][cj][ci] = w0 * t1[lk][2 * cj][ci] + w1 * t1[lk][2 * cj + 1][ci] + w2 * t1[lk][2 * cj + 2][ci] + w3 * t1[lk][2 * cj + 3][ci];
        }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < RCK * RCJ * RCI; u += blockDim.x) {
        const int ci = u & (RCI - 1), cj = (u / RCI) & (RCJ - 1), ck = u / (RCI * RCJ);
        const int I = I0 + ci, J = J0 + cj, K = K0 + ck;
        if (I >= cd.n0 || J >= cd.n1 || K >= cd.n2) continue;
        float acc = wK[ck][0] * t2[2 * ck][cj][ci] + wK[ck][1] * t2[2 * ck + 1][cj][ci] + wK[ck][2] * t2[2 * ck + 2][cj][ci] +
                    wK[ck][3] * t2[2 * ck + 3][cj][ci];
        acc *= scale;
        unsigned c = ((unsigned)K * (unsigned)cd.n1 + (unsigned)J) * (unsigned)cd.n0 + (unsigned)I;
        out[c] = acc;
        if (out2) out2[c] = mul2 * (float)S->s * acc;
        if (act0) {
            __align__(16) __nv_bfloat16 v[16];
            v[0] = __float2bfloat16_rn(acc * (float)(1. / S->s));
            v[1] = __float2bfloat16_rn(maskc[c]);
            v[2] = __float2bfloat16_rn(chan);
            for (int q = 3; q < 16; ++q) v[q] = __float2bfloat16_rn(0.f);
            uint4* dst = reinterpret_cast<uint4*>(act0 + (size_t)c * 16);
            dst[0] = reinterpret_cast<uint4*>(v)[0];
            dst[1] = reinterpret_cast<uint4*>(v)[1];
            if (act0n) {
                v[0] = __float2bfloat16_rn(-acc * (float)(1. / S->s));
                uint4* dn = reinterpret_cast<uint4*>(act0n + (size_t)c * 16);
                dn[0] = reinterpret_cast<uint4*>(v)[0];
                dn[1] = reinterpret_cast<uint4*>(v)[1];
            }
        }
    }
}

// ---------------------------------------------------------------- restriction to level 1, TMA-staged
// The same restriction from the cell lattice (v = fin * invD on active cells) as restrict_kernel,
// by persistent CTAs (one per SM) that walk the coarse tiles and stream each tile's fine box in
// by TMA while the previous tile is reduced: two stages, each holding the tile's fin, invD (FP32)
// and status (byte) boxes.  TMA wants the innermost start coordinate on a 16-byte boundary, so the
// float boxes start at fine i = 2 I0 - 4 (72 cells) and the status box at 2 I0 - 16 (96 bytes);
// boxes reaching outside the lattice are zero-filled, and zero fin contributes nothing.
constexpr int RT_BX = 72, RT_BXS = 96;
constexpr int RT_F_BYTES = RT_BX * RFJ * RFK * 4;            // 28800
constexpr int RT_S_BYTES = RT_BXS * RFJ * RFK;               // 9600
constexpr int RT_STAGE_BYTES = 2 * RT_F_BYTES + RT_S_BYTES;  // 67200
constexpr int RT_THREADS = 1024;
static_assert(RT_THREADS % (RCI * RCJ) == 0 && RT_THREADS >= RCK * RCJ * RCI, "restriction thread layout");
constexpr long long RT_WAIT_LIMIT = 1ll << 22;               // polls (each at most a short hardware wait)

__device__ __forceinline__ uint32_t rt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool rt_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// polled by one warp per CTA (the others wait at the barrier that follows), without a suspend
// hint, so that a tile starts as soon as its data has landed
__device__ __forceinline__ bool rt_wait(uint32_t bar, uint32_t parity) {
    for (long long t = 0; t < RT_WAIT_LIMIT; ++t)
        if (rt_try(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void rt_load3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :
        : "r"(dst), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

struct RestrictMaps {
    CUtensorMap fin, invD, st;   // this GPU's own buffers (no cluster multicast)
};

// PRE: the input is already v (D^-1 x on active cells, 0 elsewhere): one FP32 box per tile, no
// masking pass, three stages in less shared memory (two CTAs per SM)
template <bool PRE>
__global__ void __launch_bounds__(RT_THREADS, 2) restrict_tma_kernel(const __grid_constant__ RestrictMaps maps, Dims3 fd, Dims3 cd, int hasSt,
                                                                  float scale, float* out, int* err, const Scal* S) {
    constexpr int STAGE = PRE ? RT_F_BYTES : RT_STAGE_BYTES;
    constexpr int NS = PRE ? 3 : 2;   // stages: tiles in flight ahead of the one being reduced = NS - 1
    if (S && S->done) return;
    extern __shared__ __align__(1024) unsigned char rt_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)rt_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full[3];
    __shared__ float t1[RFK][RFJ][RCI];
    __shared__ float t2[RFK][RCJ][RCI];
    // weights of the tile being reduced, double-buffered by tile parity: tile n writes its set while
    // the last readers of tile n-1's pass 3 may still run, so no barrier ends a tile
    __shared__ float wI[2][RCI][4], wJ[2][RCJ][4], wK[2][RCK][4];
    const int tI = (cd.n0 + RCI - 1) / RCI, tJ = (cd.n1 + RCJ - 1) / RCJ, tK = (cd.n2 + RCK - 1) / RCK;
    const int T = tI * tJ * tK;
    // the tile's coordinates are stepped by gridDim.x = dI + tI (dJ + tJ dK) per iteration, with
    // carries, instead of divided every iteration
    const int G = (int)gridDim.x;
    const int dI = G % tI, dJ = (G / tI) % tJ, dK = G / (tI * tJ);
    int ti = (int)blockIdx.x % tI, tj = ((int)blockIdx.x / tI) % tJ, tk = (int)blockIdx.x / (tI * tJ);
    if (threadIdx.x == 0) {
        for (int q = 0; q < NS; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(rt_smem(&full[q])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued[3] = {0, 0, 0};   // thread 0: loads issued per stage
    auto issue = [&](int tile, int stage) {
        const int ti = tile % tI, tj = (tile / tI) % tJ, tk = tile / (tI * tJ);
        const int x = 2 * ti * RCI - 4, y = 2 * tj * RCJ - 1, z = 2 * tk * RCK - 1;
        unsigned char* b = smem + (size_t)stage * STAGE;
        const uint32_t bar = rt_smem(&full[stage]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after the generic writes of this stage's last tile
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"((uint32_t)(PRE ? RT_F_BYTES : (hasSt ? RT_STAGE_BYTES : 2 * RT_F_BYTES))) : "memory");
        rt_load3d(rt_smem(b), &maps.fin, x, y, z, bar);
        if (!PRE) {
            rt_load3d(rt_smem(b + RT_F_BYTES), &maps.invD, x, y, z, bar);
            if (hasSt) rt_load3d(rt_smem(b + 2 * RT_F_BYTES), &maps.st, x - 12, y, z, bar);
        }
        ++issued[stage];
    };
    if (threadIdx.x == 0)
        for (int q = 0; q < NS - 1; ++q)
            if ((int)blockIdx.x + q * (int)gridDim.x < T) issue(blockIdx.x + q * gridDim.x, q);
    bool failed = false;
    int n = 0;
    for (int tile = blockIdx.x; tile < T; tile += gridDim.x, ++n) {
        const int stage = n % NS;
        // the stage of tile n-1 is free once every thread has passed tile n-1's second barrier (its
        // last read of the stage is pass 1): it takes tile n + NS - 1
        const int ahead = tile + (NS - 1) * (int)gridDim.x;
        if (threadIdx.x == 0 && ahead < T) issue(ahead, (n + NS - 1) % NS);
        const int I0 = ti * RCI, J0 = tj * RCJ, K0 = tk * RCK;
        const int wb = n & 1;
        if (threadIdx.x < 4 * RCI) {
            int ci = threadIdx.x >> 2, m = threadIdx.x & 3, I = I0 + ci;
            wI[wb][ci][m] = rweight_in(2 * I - 1 + m, fd.n0, I, cd.n0);
        } else if (threadIdx.x < 4 * RCI + 4 * RCJ) {
            int u = threadIdx.x - 4 * RCI, cj = u >> 2, m = u & 3, J = J0 + cj;
            wJ[wb][cj][m] = rweight_in(2 * J - 1 + m, fd.n1, J, cd.n1);
        } else if (threadIdx.x < 4 * RCI + 4 * RCJ + 4 * RCK) {
            int u = threadIdx.x - 4 * RCI - 4 * RCJ, ck = u >> 2, m = u & 3, K = K0 + ck;
            wK[wb][ck][m] = rweight_in(2 * K - 1 + m, fd.n2, K, cd.n2);
        }
        // the next tile's coordinates
        ti += dI;
        if (ti >= tI) { ti -= tI; ++tj; }
        tj += dJ;
        if (tj >= tJ) { tj -= tJ; ++tk; }
        tk += dK;
        bool ok = true;
        if (threadIdx.x < 32) ok = rt_wait(rt_smem(&full[stage]), (uint32_t)((n / NS) & 1));
        if (__syncthreads_or(ok ? 0 : 1)) { failed = true; break; }
        float* sf = reinterpret_cast<float*>(smem + (size_t)stage * STAGE);
        if (!PRE) {
            const float* sd = sf + RT_F_BYTES / 4;
            const unsigned char* ss = smem + (size_t)stage * STAGE + 2 * RT_F_BYTES;
            // v = fin * invD on active cells, in place, for the 66 columns the tile draws on (3 .. 68)
            for (int e = threadIdx.x; e < RFK * RFJ * RFI; e += RT_THREADS) {
                const int li = e % RFI, row = e / RFI;
                const int o = row * RT_BX + 3 + li;
                const bool act = !hasSt || ss[row * RT_BXS + 15 + li] == ST_ACTIVE;
                sf[o] = act ? sf[o] * sd[o] : 0.f;
            }
            __syncthreads();
        }
        // each thread keeps one coarse column ci (RT_THREADS is a multiple of RCI * RCJ * 8), so its
        // weights stay in registers; the four fine values of pass 1 come as three aligned float2
        const int ci = threadIdx.x & (RCI - 1);
        {
            const float w0 = wI[wb][ci][0], w1 = wI[wb][ci][1], w2 = wI[wb][ci][2], w3 = wI[wb][ci][3];
            float* T1 = &t1[0][0][0];
            for (int row = threadIdx.x >> 5; row < RFK * RFJ; row += RT_THREADS / RCI) {
                const float2* v2 = reinterpret_cast<const float2*>(sf + row * RT_BX + 2 + 2 * ci);   // fine 2I-2 .. 2I+3
                const float2 a = v2[0], b = v2[1], c = v2[2];
                T1[row * RCI + ci] = w0 * a.y + w1 * b.x + w2 * b.y + w3 * c.x;
            }
        }
        __syncthreads();
        {
            const int cj = (threadIdx.x >> 5) & (RCJ - 1);
            const float w0 = wJ[wb][cj][0], w1 = wJ[wb][cj][1], w2 = wJ[wb][cj][2], w3 = wJ[wb][cj][3];
            for (int lk = threadIdx.x / (RCI * RCJ); lk < RFK; lk += RT_THREADS / (RCI * RCJ))
                t2[lk][cj][ci] = w0 * t1[lk][2 * cj][ci] + w1 * t1[lk][2 * cj + 1][ci] + w2 * t1[lk][2 * cj + 2][ci] + w3 * t1[lk][2 * cj + 3][ci];
        }
        __syncthreads();
        if (threadIdx.x < RCK * RCJ * RCI) {
            const int cj = (threadIdx.x >> 5) & (RCJ - 1), ck = threadIdx.x / (RCI * RCJ);
            const int I = I0 + ci, J = J0 + cj, K = K0 + ck;
            if (I < cd.n0 && J < cd.n1 && K < cd.n2) {
                const float acc = wK[wb][ck][0] * t2[2 * ck][cj][ci] + wK[wb][ck][1] * t2[2 * ck + 1][cj][ci] +
                                  wK[wb][ck][2] * t2[2 * ck + 2][cj][ci] + wK[wb][ck][3] * t2[2 * ck + 3][cj][ci];
                out[((unsigned)K * (unsigned)cd.n1 + (unsigned)J) * (unsigned)cd.n0 + (unsigned)I] = acc * scale;
            }
        }
        // no barrier here: tile n+1 writes t1 after its first barrier (all of tile n's pass 2 is
        // done by then), t2 after its second (all of tile n's pass 3 reads come before the first
        // barrier of tile n+1 is passed), and weights into the other buffer
    }
    if (threadIdx.x == 0) {
        if (failed) atomicExch(err, 1);
        // every load issued lands before the shared memory is released
        for (int q = 0; q < NS; ++q)
            if (issued[q] > 0) rt_wait(rt_smem(&full[q]), (uint32_t)((issued[q] - 1) & 1));
    }
    __syncthreads();
}

// tensor maps of the TMA restriction's inputs, kept per (buffer, lattice, element size)
PFN_cuTensorMapEncodeTiled_v12000 rt_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
const CUtensorMap* rt_map(const void* base, const Dims3& fd, int esize) {
    static std::vector<std::pair<std::array<long long, 5>, CUtensorMap>> cache;
    static std::mutex lock;
    std::lock_guard<std::mutex> guard(lock);
    const std::array<long long, 5> key = {(long long)(uintptr_t)base, fd.n0, fd.n1, fd.n2, esize};
    for (auto& e : cache)
        if (e.first == key) return &e.second;
    PFN_cuTensorMapEncodeTiled_v12000 fn = rt_encode_fn();
    if (!fn) return nullptr;
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)fd.n0, (cuuint64_t)fd.n1, (cuuint64_t)fd.n2};
    cuuint64_t strides[2] = {(cuuint64_t)fd.n0 * esize, (cuuint64_t)fd.n0 * fd.n1 * esize};
    cuuint32_t box[3] = {(cuuint32_t)(esize == 4 ? RT_BX : RT_BXS), (cuuint32_t)RFJ, (cuuint32_t)RFK};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(&m, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nullptr;
    cache.emplace_back(key, m);
    return &cache.back().second;
}

// whether the fine lattice and buffers meet TMA's rules for the staged restriction: rows of 16-byte
// multiples (status rows of bytes too) and 16-byte aligned bases
bool restrict_tma_usable(const Dims3& fd, const float* fin, const float* invD, const uint8_t* st) {
    auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    if (fd.n0 % 4 != 0 || !al(fin) || (invD && !al(invD))) return false;
    if (st && (fd.n0 % 16 != 0 || !al(st))) return false;
    return rt_encode_fn() != nullptr;
}

// invD null: fin is already v (pre-multiplied and masked)
int launch_restrict_tma(const Dims3& fd, const Dims3& cd, const float* fin, const float* invD, const uint8_t* st, float scale, float* out,
                        int* err, const Scal* S, cudaStream_t stream) {
    RestrictMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    const bool pre = invD == nullptr;
    const CUtensorMap* mf = rt_map(fin, fd, 4);
    const CUtensorMap* md = pre ? nullptr : rt_map(invD, fd, 4);
    const CUtensorMap* ms = (!pre && st) ? rt_map(st, fd, 1) : nullptr;
    if (!mf || (!pre && !md) || (!pre && st && !ms)) { set_error("tensor map encoding failed for the staged restriction"); return 1; }
    maps.fin = *mf;
    if (md) maps.invD = *md;
    if (ms) maps.st = *ms;
    const size_t smemFull = 1024 + 2 * (size_t)RT_STAGE_BYTES, smemPre = 1024 + 3 * (size_t)RT_F_BYTES;
    static bool attr = false;
    static int nsm = 0;
    if (!attr) {
        CB_CUDA(cudaFuncSetAttribute(restrict_tma_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemFull));
        CB_CUDA(cudaFuncSetAttribute(restrict_tma_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemPre));
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        attr = true;
    }
    const long long T = (long long)((cd.n0 + RCI - 1) / RCI) * ((cd.n1 + RCJ - 1) / RCJ) * ((cd.n2 + RCK - 1) / RCK);
    const int sms = nsm > 0 ? nsm : 148;
    if (pre) {
        const int grid = (int)std::min<long long>(T, 2LL * sms);   // two CTAs per SM
        restrict_tma_kernel<true><<<grid, RT_THREADS, smemPre, stream>>>(maps, fd, cd, 0, scale, out, err, S);
    } else {
        const int grid = (int)std::min<long long>(T, sms);
        restrict_tma_kernel<false><<<grid, RT_THREADS, smemFull, stream>>>(maps, fd, cd, st ? 1 : 0, scale, out, err, S);
    }
    CB_CHECK_LAUNCH();
    return 0;
}

inline long long restrict_tiles(const Dims3& cd) {
    return (long long)((cd.n0 + RCI - 1) / RCI) * ((cd.n1 + RCJ - 1) / RCJ) * ((cd.n2 + RCK - 1) / RCK);
}
inline dim3 restrict_grid(const Dims3& cd) {
    return dim3((unsigned)((cd.n0 + RCI - 1) / RCI), (unsigned)((cd.n1 + RCJ - 1) / RCJ), (unsigned)((cd.n2 + RCK - 1) / RCK));
}

// (P wc)[f] on the fine lattice fd from the coarse lattice cd (32-bit index arithmetic:
// lattices stay below 2^32 cells)
__device__ __forceinline__ float prolong_at(const Dims3& fd, const Dims3& cd, const float* wc, long long f) {
    const unsigned uf = (unsigned)f, n0 = (unsigned)fd.n0, n1 = (unsigned)fd.n1;
    const unsigned t = uf / n0;
    const int fi = (int)(uf - t * n0);
    const int fk = (int)(t / n1);
    const int fj = (int)(t - (unsigned)fk * n1);
    int I0 = fi >> 1, I1 = pclamp((fi & 1) ? I0 + 1 : I0 - 1, cd.n0);
    int J0 = fj >> 1, J1 = pclamp((fj & 1) ? J0 + 1 : J0 - 1, cd.n1);
    int K0 = fk >> 1, K1 = pclamp((fk & 1) ? K0 + 1 : K0 - 1, cd.n2);
    const unsigned sJ = (unsigned)cd.n0, sK = (unsigned)cd.n0 * (unsigned)cd.n1;
    auto row = [&](int K, int J) {
        const float* w = wc + (unsigned)K * sK + (unsigned)J * sJ;
        return 0.75f * __ldg(w + I0) + 0.25f * __ldg(w + I1);
    };
    float k0 = 0.75f * row(K0, J0) + 0.25f * row(K0, J1);
    float k1 = 0.75f * row(K1, J0) + 0.25f * row(K1, J1);
    return 0.75f * k0 + 0.25f * k1;
}

// (P wc) for the 4 consecutive cells 4q..4q+3 of the fine lattice fd: the (j, k) part of the
// index and the four coarse rows are computed once when the 4 cells share a row
__device__ __forceinline__ void prolong4_ijk(const Dims3& fd, const Dims3& cd, const float* wc, unsigned f0, int fi, int fj, int fk,
                                             float (&out)[4]);
__device__ __forceinline__ void prolong4(const Dims3& fd, const Dims3& cd, const float* wc, long long q, float (&out)[4]) {
    const unsigned f0 = (unsigned)(4 * q), n0 = (unsigned)fd.n0, n1 = (unsigned)fd.n1;
    const unsigned t = f0 / n0;
    const int fi = (int)(f0 - t * n0);
    const int fk = (int)(t / n1);
    const int fj = (int)(t - (unsigned)fk * n1);
    prolong4_ijk(fd, cd, wc, f0, fi, fj, fk, out);
}
// the same for the 4 cells from f0 = (fk nJ + fj) nI + fi, whose coordinates the caller knows
__device__ __forceinline__ void prolong4_ijk(const Dims3& fd, const Dims3& cd, const float* wc, unsigned f0, int fi, int fj, int fk,
                                             float (&out)[4]) {
    if (fi + 3 >= fd.n0) {   // the 4 cells span a row end
#pragma unroll
        for (int m = 0; m < 4; ++m) out[m] = prolong_at(fd, cd, wc, (long long)f0 + m);
        return;
    }
    const int J0 = fj >> 1, J1 = pclamp((fj & 1) ? J0 + 1 : J0 - 1, cd.n1);
    const int K0 = fk >> 1, K1 = pclamp((fk & 1) ? K0 + 1 : K0 - 1, cd.n2);
    const unsigned sJ = (unsigned)cd.n0, sK = (unsigned)cd.n0 * (unsigned)cd.n1;
    const float* r00 = wc + (unsigned)K0 * sK + (unsigned)J0 * sJ;
    const float* r01 = wc + (unsigned)K0 * sK + (unsigned)J1 * sJ;
    const float* r10 = wc + (unsigned)K1 * sK + (unsigned)J0 * sJ;
    const float* r11 = wc + (unsigned)K1 * sK + (unsigned)J1 * sJ;
    if ((fi & 1) == 0) {
        // the four fine cells fi .. fi+3 draw on coarse columns F-1 .. F+2 (F = fi / 2, clamped):
        // each of the four coarse rows is loaded once, 16 loads in all, and every fine value is
        // blended in the same order as prolong_at's
        const int F = fi >> 1;
        const int col[4] = {pclamp(F - 1, cd.n0), F, pclamp(F + 1, cd.n0), pclamp(F + 2, cd.n0)};
        float v00[4], v01[4], v10[4], v11[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v00[u] = __ldg(r00 + col[u]); v01[u] = __ldg(r01 + col[u]);
            v10[u] = __ldg(r10 + col[u]); v11[u] = __ldg(r11 + col[u]);
        }
        // (I0, I1) slots of fine cells fi, fi+1, fi+2, fi+3: (F, F-1), (F, F+1), (F+1, F), (F+1, F+2)
        const int s0[4] = {1, 1, 2, 2}, s1[4] = {0, 2, 1, 3};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            auto row = [&](const float (&v)[4]) { return 0.75f * v[s0[m]] + 0.25f * v[s1[m]]; };
            float k0 = 0.75f * row(v00) + 0.25f * row(v01);
            float k1 = 0.75f * row(v10) + 0.25f * row(v11);
            out[m] = 0.75f * k0 + 0.25f * k1;
        }
        return;
    }
    // the four fine cells draw on coarse columns I-1 .. I+2 around I = fi / 2
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const int i = fi + m;
        const int I0 = i >> 1, I1 = pclamp((i & 1) ? I0 + 1 : I0 - 1, cd.n0);
        auto row = [&](const float* w) { return 0.75f * __ldg(w + I0) + 0.25f * __ldg(w + I1); };
        float k0 = 0.75f * row(r00) + 0.25f * row(r01);
        float k1 = 0.75f * row(r10) + 0.25f * row(r11);
        out[m] = 0.75f * k0 + 0.25f * k1;
    }
}

// ---------------------------------------------------------------- coarse tail of the pyramid
// The coarsest levels in one CTA (pyramid mode): u_lt = R u_(lt-1), with u_(lt-1) staged from global
// memory into shared memory, u_(l+1) = R u_l, then w_last = gain u_last and
// w_l = gain_l u_l + P w_(l+1) back up to lt, all in shared memory; u_l and w_l of every tail level
// are written out.  It replaces 2 (levels - lt) launches of a few hundred cells each by one, with
// the arithmetic of restrict_kernel and prolong_kernel in the same order.
constexpr int TAIL_MAX_IN = 8192;       // cells of level lt-1 (staged)
constexpr int TAIL_THREADS = 1024;
struct TailArgs {
    int n;                              // tail levels lt .. lt+n-1
    Dims3 d[LEARN_MAX_LEVELS + 1];      // d[0]: level lt-1; d[1..n]: the tail levels
    float rscale[LEARN_MAX_LEVELS], gain[LEARN_MAX_LEVELS];
    const float* uin;                   // u of level lt-1
    float* u[LEARN_MAX_LEVELS];
    float* w[LEARN_MAX_LEVELS];
};

__device__ __forceinline__ float tail_restrict_at(const float* fin, const Dims3& fd, const Dims3& cd, int I, int J, int K, float scale) {
    float t2[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int fk = 2 * K - 1 + c;
        float t1[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int fj = 2 * J - 1 + b;
            float v[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int fi = 2 * I - 1 + a;
                const bool in = fi >= 0 && fi < fd.n0 && fj >= 0 && fj < fd.n1 && fk >= 0 && fk < fd.n2;
                v[a] = in ? fin[((unsigned)fk * (unsigned)fd.n1 + (unsigned)fj) * (unsigned)fd.n0 + (unsigned)fi] : 0.f;
            }
            t1[b] = rweight_in(2 * I - 1, fd.n0, I, cd.n0) * v[0] + rweight_in(2 * I, fd.n0, I, cd.n0) * v[1] +
                    rweight_in(2 * I + 1, fd.n0, I, cd.n0) * v[2] + rweight_in(2 * I + 2, fd.n0, I, cd.n0) * v[3];
        }
        t2[c] = rweight_in(2 * J - 1, fd.n1, J, cd.n1) * t1[0] + rweight_in(2 * J, fd.n1, J, cd.n1) * t1[1] +
                rweight_in(2 * J + 1, fd.n1, J, cd.n1) * t1[2] + rweight_in(2 * J + 2, fd.n1, J, cd.n1) * t1[3];
    }
    float acc = rweight_in(2 * K - 1, fd.n2, K, cd.n2) * t2[0] + rweight_in(2 * K, fd.n2, K, cd.n2) * t2[1] +
                rweight_in(2 * K + 1, fd.n2, K, cd.n2) * t2[2] + rweight_in(2 * K + 2, fd.n2, K, cd.n2) * t2[3];
    acc *= scale;
    return acc;
}

// prolong_at on a shared-memory coarse array (plain loads), the same blend order
__device__ __forceinline__ float tail_prolong_at(const Dims3& fd, const Dims3& cd, const float* wc, long long f) {
    const unsigned uf = (unsigned)f, n0 = (unsigned)fd.n0, n1 = (unsigned)fd.n1;
    const unsigned t = uf / n0;
    const int fi = (int)(uf - t * n0);
    const int fk = (int)(t / n1);
    const int fj = (int)(t - (unsigned)fk * n1);
    int I0 = fi >> 1, I1 = pclamp((fi & 1) ? I0 + 1 : I0 - 1, cd.n0);
    int J0 = fj >> 1, J1 = pclamp((fj & 1) ? J0 + 1 : J0 - 1, cd.n1);
    int K0 = fk >> 1, K1 = pclamp((fk & 1) ? K0 + 1 : K0 - 1, cd.n2);
    const unsigned sJ = (unsigned)cd.n0, sK = (unsigned)cd.n0 * (unsigned)cd.n1;
    auto row = [&](int K, int J) {
        const float* w = wc + (unsigned)K * sK + (unsigned)J * sJ;
        return 0.75f * w[I0] + 0.25f * w[I1];
    };
    float k0 = 0.75f * row(K0, J0) + 0.25f * row(K0, J1);
    float k1 = 0.75f * row(K1, J0) + 0.25f * row(K1, J1);
    return 0.75f * k0 + 0.25f * k1;
}

__global__ void __launch_bounds__(TAIL_THREADS) coarse_tail_kernel(const __grid_constant__ TailArgs a, const Scal* S) {
    if (S && S->done) return;
    extern __shared__ float tsm[];
    long long off[LEARN_MAX_LEVELS + 1];
    long long total = 0;
    for (int l = 0; l <= a.n; ++l) {
        off[l] = total;
        total += (long long)a.d[l].n0 * a.d[l].n1 * a.d[l].n2;
    }
    float* U = tsm;                    // u of levels lt-1 .. lt+n-1, packed
    float* W = tsm + total - off[1];   // w of the tail levels (the same offsets; nothing for lt-1)
    const long long n0 = off[1];
    for (long long c = threadIdx.x; c < n0; c += blockDim.x) U[c] = a.uin[c];
    __syncthreads();
    for (int l = 1; l <= a.n; ++l) {
        const Dims3 fd = a.d[l - 1], cd = a.d[l];
        const long long N = (long long)cd.n0 * cd.n1 * cd.n2;
        for (long long c = threadIdx.x; c < N; c += blockDim.x) {
            const int I = (int)(c % cd.n0), J = (int)((c / cd.n0) % cd.n1), K = (int)(c / ((long long)cd.n0 * cd.n1));
            const float v = tail_restrict_at(U + off[l - 1], fd, cd, I, J, K, a.rscale[l - 1]);
            U[off[l] + c] = v;
            a.u[l - 1][c] = v;
        }
        __syncthreads();
    }
    for (int l = a.n; l >= 1; --l) {
        const Dims3 fd = a.d[l];
        const long long N = (long long)fd.n0 * fd.n1 * fd.n2;
        for (long long c = threadIdx.x; c < N; c += blockDim.x) {
            float v = a.gain[l - 1] * 1.f * U[off[l] + c];
            if (l < a.n) v += tail_prolong_at(fd, a.d[l + 1], W + off[l + 1], c);
            W[off[l] + c] = v;
            a.w[l - 1][c] = v;
        }
        __syncthreads();
    }
}

// w_l = gain * (ydiv ? y : s y) + P w_{l+1}   (wc null on the coarsest level); with yn, the
// network term is odd: y <- (y - yn) / 2 (yn = the network applied to the negated input)
__global__ void __launch_bounds__(256) prolong_kernel(Dims3 fd, Dims3 cd, const float* wc, const float* y, const float* yn, int ydiv,
                                                      float gain, float* out, const Scal* S) {
    if (S->done) return;
    long long Nf = (long long)fd.n0 * fd.n1 * fd.n2;
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= Nf) return;
    float sy = ydiv ? 1.f : (float)S->s;
    float yv = yn ? 0.5f * (y[f] - yn[f]) : y[f];
    float v = gain * sy * yv;
    if (wc) v += prolong_at(fd, cd, wc, f);
    out[f] = v;
}

// prolong_kernel on 4 consecutive fine cells per thread (cell count a multiple of 4, 16-byte
// aligned arrays): one index division per 4 cells and each coarse row loaded once (prolong4),
// every value formed as prolong_kernel forms it
__global__ void __launch_bounds__(256) prolong4_kernel(Dims3 fd, Dims3 cd, const float* wc, const float* y, const float* yn, int ydiv,
                                                       float gain, float* out, const Scal* S) {
    if (S->done) return;
    const long long NQ = ((long long)fd.n0 * fd.n1 * fd.n2) >> 2;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= NQ) return;
    const float sy = ydiv ? 1.f : (float)S->s;
    float Y[4], PW[4] = {0.f, 0.f, 0.f, 0.f}, V[4];
    un4(ld4(y, q), Y);
    if (yn) {
        float Yn[4];
        un4(ld4(yn, q), Yn);
#pragma unroll
        for (int m = 0; m < 4; ++m) Y[m] = 0.5f * (Y[m] - Yn[m]);
    }
    if (wc) prolong4(fd, cd, wc, q, PW);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float v = gain * sy * Y[m];
        if (wc) v += PW[m];
        V[m] = v;
    }
    st4(out, q, V);
}

// z = D^-1 r + P w_1 (active), D^-1 r (ghost), 0 (inactive); partial (z, q_prev)
__global__ void __launch_bounds__(LB) precond_z_kernel(long long N, Dims3 fd, Dims3 cd, const float* r, const float* invD,
                                                       const uint8_t* st, const float* w1, float* z, const float* qprev, double* part,
                                                       const Scal* S) {
    if (S->done) return;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    double v[1] = {0.};
    for (long long q = t0; q < NQ; q += T) {
        float R[4], D[4], Z[4], Q[4];
        uint8_t F[4];
        un4(ld4(r, q), R); un4(ld4(invD, q), D); un4(ld4(qprev, q), Q); st_flags4(st, q, F);
        float PW[4] = {0.f, 0.f, 0.f, 0.f};
        if (w1) prolong4(fd, cd, w1, q, PW);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (F[m] == ST_INACTIVE) Z[m] = 0.f;
            else {
                Z[m] = D[m] * R[m];
                if (F[m] == ST_ACTIVE) Z[m] += PW[m];
            }
            v[0] += (double)Z[m] * Q[m];
        }
        st4(z, q, Z);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        float zv;
        if (is_inactive(st, c)) zv = 0.f;
        else {
            zv = __ldg(invD + c) * r[c];
            if (w1 && is_active(st, c)) zv += prolong_at(fd, cd, w1, c);
        }
        z[c] = zv;
        v[0] += (double)zv * qprev[c];
    }
    block_sums(v, 1, part);
}

__global__ void beta_kernel(const double* part, int nblk, Scal* S) {
    if (S->done) return;
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) { S->zq = t[0]; S->beta = S->pq != 0. ? t[0] / S->pq : 0.; }
}

// FP32 operator row (7-point, or the ghost row's 9 entries)
template <class X>
__device__ __forceinline__ float applyF(const OpSymF32& A, long long c, X&& x) {
    float y = __ldg(A.aP + c) * x(c) + __ldg(A.aE + c) * x(c + 1) + __ldg(A.aE + c - 1) * x(c - 1) + __ldg(A.aN + c) * x(c + A.nI)
              + __ldg(A.aN + c - A.nI) * x(c - A.nI) + __ldg(A.aT + c) * x(c + A.nIJ) + __ldg(A.aT + c - A.nIJ) * x(c - A.nIJ);
    if (A.gh.n > 0) {
        uint32_t w = __ldg(A.gh.bits + (c >> 5));
        if ((w >> (c & 31)) & 1u) {
            int lo = 0, hi = A.gh.n;
            while (lo < hi) { int mid = (lo + hi) >> 1; if (__ldg(A.gh.cell + mid) < c) lo = mid + 1; else hi = mid; }
            float s = 0.f;
            for (int m = 0; m < 9; ++m) { int col = __ldg(A.gh.col + 9 * lo + m); if (col >= 0) s += (float)__ldg(A.gh.val + 9 * lo + m) * x(col); }
            y = s;
        }
    }
    return y;
}

// p_new = z - beta p_old, q_new = A p_new (neighbours recomputed), partials (p, q), (p, r)
__global__ void __launch_bounds__(LB) direction_kernel(OpSymF32 A, long long N, const float* z, const float* pold, float* pnew, float* qnew,
                                                       const float* r, double* part, const Scal* S) {
    if (S->done) return;
    float be = (float)S->beta;
    double v[2] = {0., 0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float pc = z[c] - be * pold[c];
        float qc = applyF(A, c, [&](long long e_) { return z[e_] - be * pold[e_]; });
        pnew[c] = pc; qnew[c] = qc;
        v[0] += (double)pc * qc;
        v[1] += (double)pc * r[c];
    }
    block_sums(v, 2, part);
}

__global__ void alpha_kernel(const double* part, int nblk, Scal* S) {
    if (S->done) return;
    double t[2];
    totals(part, nblk, 2, t);
    if (threadIdx.x == 0) {
        S->pq = t[0];
        S->pr = t[1];
        S->alpha = t[0] != 0. ? t[1] / t[0] : 0.;
        if (!(t[0] != 0.) || t[0] != t[0]) S->done = 1;
    }
}

// e += alpha p, r -= alpha q, partial ||r||^2 and ||D^-1 r||^2 (next network scale)
__global__ void __launch_bounds__(LB) step_kernel(long long N, float* e, float* r, const float* p, const float* q, const float* invD,
                                                  const uint8_t* st, double* part, const Scal* S) {
    if (S->done) return;
    const float al = (float)S->alpha;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    double v[2] = {0., 0.};
    for (long long qd = t0; qd < NQ; qd += T) {
        float E[4], R[4], P4[4], Q[4], D[4];
        uint8_t F[4];
        un4(ld4(e, qd), E); un4(ld4(r, qd), R); un4(ld4(p, qd), P4); un4(ld4(q, qd), Q); un4(ld4(invD, qd), D); st_flags4(st, qd, F);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            E[m] = E[m] + al * P4[m];
            R[m] = R[m] - al * Q[m];
            v[0] += (double)R[m] * R[m];
            if (F[m] == ST_ACTIVE) { double u = (double)D[m] * R[m]; v[1] += u * u; }
        }
        st4(e, qd, E);
        st4(r, qd, R);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        e[c] = e[c] + al * p[c];
        float rn = r[c] - al * q[c];
        r[c] = rn;
        v[0] += (double)rn * rn;
        if (is_active(st, c)) { double u = (double)__ldg(invD + c) * rn; v[1] += u * u; }
    }
    block_sums(v, 2, part);
}

__global__ void step_finish_kernel(const double* part, int nblk, Scal* S, int max_iters) {
    if (S->done) return;
    double t[2];
    totals(part, nblk, 2, t);
    if (threadIdx.x == 0) {
        S->rr = t[0];
        S->iters += 1;
        S->s = S->nact > 0. ? sqrt(t[1] / S->nact) : 1.;
        if (!(S->s > 0.)) S->s = 1.;
        if (t[0] <= S->tin2 || S->iters >= max_iters || t[0] != t[0]) S->done = 1;
    }
}

// ---------------------------------------------------------------- inner flexible BiCGStab (FP32)
// For operators with immersed-boundary ghost rows (not symmetric): right-preconditioned
// BiCGStab, each half step preconditioned by the same M; x and r stay consistent for any M.
//   p = r + beta (p - omega v);  ph = M(p);  v = A ph;  alpha = rho / (rhat, v)
//   s = r - alpha v;  sh = M(s);  t = A sh;  omega = (t, s) / (t, t)
//   e += alpha ph + omega sh;  r = s - omega t;  rho' = (rhat, r);  beta = rho'/rho alpha/omega
__global__ void __launch_bounds__(LB) bs_start_kernel(long long N, const float* r, float* rh, float* e, float* p, float* v, double* part,
                                                      const Scal* S) {
    if (S->done) return;
    double a[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float rv = r[c];
        rh[c] = rv; e[c] = 0.f; p[c] = 0.f; v[c] = 0.f;
        a[0] += (double)rv * rv;
    }
    block_sums(a, 1, part);
}
__global__ void bs_start_finish(const double* part, int nblk, Scal* S, double eta, const double* nact) {
    if (S->done) return;
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) {
        S->rr0 = t[0]; S->rr = t[0];
        S->tin2 = eta * eta * t[0];
        S->nact = *nact;
        S->rho = t[0]; S->alpha = 1.; S->omega = 1.; S->beta = 0.;
        S->done = !(t[0] > 0.);
    }
}
// finishing steps of the flexible BiCGStab reductions (in a one-block kernel, or in the block
// of the producing kernel that finishes last)
__device__ __forceinline__ void fin_scale(const double* t, Scal* S) {
    double sc = S->nact > 0. ? sqrt(t[0] / S->nact) : 1.;
    S->s = sc > 0. ? sc : 1.;
}
__device__ __forceinline__ void fin_alpha(const double* t, Scal* S) {
    S->rv = t[0];
    if (t[0] != 0. && t[0] == t[0]) S->alpha = S->rho / t[0];
    else { S->alpha = 0.; S->done = 1; }
}
__device__ __forceinline__ void fin_omega(const double* t, Scal* S) {
    S->ts = t[0]; S->tt = t[1];
    S->omega = t[1] > 0. ? t[0] / t[1] : 0.;
}
__device__ __forceinline__ void fin_update(const double* t, Scal* S, int max_iters) {
    S->rr = t[0];
    S->iters += 1;
    double rho_new = t[1];
    bool breakdown = !(S->omega != 0.) || !(S->rho != 0.) || t[1] != t[1];
    S->beta = breakdown ? 0. : (rho_new / S->rho) * (S->alpha / S->omega);
    S->rho = rho_new;
    if (t[0] <= S->tin2 || S->iters >= max_iters || t[0] != t[0] || breakdown) S->done = 1;
}
// p = r + beta (p - omega v); partial sum of (D^-1 p)^2 over active cells (scale of M(p))
__global__ void __launch_bounds__(LB) bs_dir_kernel(long long N, const float* r, const float* v, const float* invD, const uint8_t* st,
                                                    float* p, double* part, Scal* S, unsigned* ctr, float* uo) {
    if (S->done) return;
    const float be = (float)S->beta, om = (float)S->omega;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    double a[1] = {0.};
    for (long long q = t0; q < NQ; q += T) {
        float R[4], V[4], P4[4], D[4];
        uint8_t F[4];
        un4(ld4(r, q), R); un4(ld4(v, q), V); un4(ld4(p, q), P4); un4(ld4(invD, q), D); st_flags4(st, q, F);
        float U[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            P4[m] = R[m] + be * (P4[m] - om * V[m]);
            U[m] = F[m] == ST_ACTIVE ? D[m] * P4[m] : 0.f;
            if (F[m] == ST_ACTIVE) { double u = (double)D[m] * P4[m]; a[0] += u * u; }
        }
        st4(p, q, P4);
        if (uo) st4(uo, q, U);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        float pv = r[c] + be * (p[c] - om * v[c]);
        p[c] = pv;
        if (is_active(st, c)) { double u = (double)__ldg(invD + c) * pv; a[0] += u * u; }
        if (uo) uo[c] = is_active(st, c) ? __ldg(invD + c) * pv : 0.f;
    }
    block_sums(a, 1, part);
    if (ctr && last_block(ctr)) {
        double t[1];
        totals_cg(part, gridDim.x, 1, t);
        if (threadIdx.x == 0) { fin_scale(t, S); *ctr = 0u; }
    }
}
__global__ void scale_finish(const double* part, int nblk, Scal* S) {
    if (S->done) return;
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) fin_scale(t, S);
}
// y = M(x) on the cell lattice: D^-1 x + P w_1 on active cells, D^-1 x on ghost rows, 0 on inactive cells
__global__ void __launch_bounds__(LB) bs_z_kernel(long long N, Dims3 fd, Dims3 cd, const float* x, const float* invD, const uint8_t* st,
                                                  const float* w1, float* y, const Scal* S) {
    if (S->done) return;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    // lattice coordinates of cell 4q, stepped with the loop (no division inside it)
    const unsigned n0 = (unsigned)fd.n0, n1 = (unsigned)fd.n1;
    const unsigned step = (unsigned)(4 * T), stepRows = step / n0, dI = step - stepRows * n0;
    const unsigned dK = stepRows / n1, dJ = stepRows - dK * n1;
    int fi, fj, fk;
    {
        const unsigned f0 = (unsigned)(4 * t0), rows = f0 / n0;
        fi = (int)(f0 - rows * n0);
        fk = (int)(rows / n1);
        fj = (int)(rows - (unsigned)fk * n1);
    }
    for (long long q = t0; q < NQ; q += T) {
        float X[4], D[4], Y[4];
        uint8_t F[4];
        un4(ld4(x, q), X); un4(ld4(invD, q), D); st_flags4(st, q, F);
        float PW[4] = {0.f, 0.f, 0.f, 0.f};
        if (w1) prolong4_ijk(fd, cd, w1, (unsigned)(4 * q), fi, fj, fk, PW);
        fi += (int)dI;
        const int carry = fi >= fd.n0;
        if (carry) fi -= fd.n0;
        fj += (int)dJ + carry;
        const int carryJ = fj >= fd.n1;
        if (carryJ) fj -= fd.n1;
        fk += (int)dK + carryJ;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (F[m] == ST_INACTIVE) Y[m] = 0.f;
            else {
                Y[m] = D[m] * X[m];
                if (F[m] == ST_ACTIVE) Y[m] += PW[m];
            }
        }
        st4(y, q, Y);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        float zv;
        if (is_inactive(st, c)) zv = 0.f;
        else {
            zv = __ldg(invD + c) * x[c];
            if (w1 && is_active(st, c)) zv += prolong_at(fd, cd, w1, c);
        }
        y[c] = zv;
    }
}
// A x for the 4 consecutive cells 4q .. 4q+3 (nI and nI*nJ multiples of 4, so every neighbouring
// group of 4 is 16-byte aligned): 14 loads for the 4 rows instead of 14 per row.  The west /
// south / bottom coefficients of a cell are the east / north / top ones of that neighbour.
__device__ __forceinline__ void spmv4(const OpSymF32& A, const float* x, long long q, float (&Y)[4]) {
    const long long c = 4 * q;
    float P[4], E[4], Nn[4], T[4], Sn[4], B[4], X[4], XN[4], XS[4], XT[4], XB[4];
    un4(ld4(A.aP, q), P); un4(ld4(A.aE, q), E); un4(ld4(A.aN, q), Nn); un4(ld4(A.aT, q), T);
    un4(ld4(A.aN, q - A.nI / 4), Sn); un4(ld4(A.aT, q - A.nIJ / 4), B);
    un4(ld4(x, q), X); un4(ld4(x, q + A.nI / 4), XN); un4(ld4(x, q - A.nI / 4), XS);
    un4(ld4(x, q + A.nIJ / 4), XT); un4(ld4(x, q - A.nIJ / 4), XB);
    const float eW = __ldg(A.aE + c - 1), xW = x[c - 1], xE = x[c + 4];
    const float W[4] = {eW, E[0], E[1], E[2]};
    const float xl[4] = {xW, X[0], X[1], X[2]};
    const float xr[4] = {X[1], X[2], X[3], xE};
#pragma unroll
    for (int m = 0; m < 4; ++m)
        Y[m] = P[m] * X[m] + E[m] * xr[m] + W[m] * xl[m] + Nn[m] * XN[m] + Sn[m] * XS[m] + T[m] * XT[m] + B[m] * XB[m];
    if (A.gh.n > 0) {
        const uint32_t bits = (__ldg(A.gh.bits + (c >> 5)) >> (c & 31)) & 0xFu;
        if (bits)
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if ((bits >> m) & 1u) Y[m] = applyF(A, c + m, [&](long long e_) { return x[e_]; });
    }
}

// out = A x; partial (a1, out), or with b2: (b2, out) and (out, out)
template <bool V4>
__global__ void __launch_bounds__(LB, 5) bs_spmv_kernel(OpSymF32 A, long long N, const float* x, float* out, const float* a1, const float* b2,
                                                     double* part, Scal* S, unsigned* ctr) {
    if (S->done) return;
    double a[2] = {0., 0.};
    long long c0 = 0;
    if (V4) {
        const long long NQ = N >> 2;
        for (long long q = blockIdx.x * (long long)LB + threadIdx.x; q < NQ; q += (long long)gridDim.x * LB) {
            float Y[4];
            spmv4(A, x, q, Y);
            st4(out, q, Y);
            if (b2) {
                float Bv[4];
                un4(ld4(b2, q), Bv);
#pragma unroll
                for (int m = 0; m < 4; ++m) { a[0] += (double)Bv[m] * Y[m]; a[1] += (double)Y[m] * Y[m]; }
            } else {
                float Av[4];
                un4(ld4(a1, q), Av);
#pragma unroll
                for (int m = 0; m < 4; ++m) a[0] += (double)Av[m] * Y[m];
            }
        }
        c0 = 4 * NQ;
    }
    for (long long c = c0 + blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float y = applyF(A, c, [&](long long e_) { return x[e_]; });
        out[c] = y;
        if (b2) { a[0] += (double)b2[c] * y; a[1] += (double)y * y; }
        else a[0] += (double)a1[c] * y;
    }
    block_sums(a, b2 ? 2 : 1, part);
    if (ctr && last_block(ctr)) {
        double t[2];
        totals_cg(part, gridDim.x, b2 ? 2 : 1, t);
        if (threadIdx.x == 0) {
            if (b2) fin_omega(t, S);
            else fin_alpha(t, S);
            *ctr = 0u;
        }
    }
}
// s = r - alpha v; partial sum of (D^-1 s)^2 over active cells
__global__ void __launch_bounds__(LB) bs_s_kernel(long long N, const float* r, const float* v, const float* invD, const uint8_t* st, float* s,
                                                  double* part, Scal* S, unsigned* ctr, float* uo) {
    if (S->done) return;
    const float al = (float)S->alpha;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    double a[1] = {0.};
    for (long long q = t0; q < NQ; q += T) {
        float R[4], V[4], D[4], O[4];
        uint8_t F[4];
        un4(ld4(r, q), R); un4(ld4(v, q), V); un4(ld4(invD, q), D); st_flags4(st, q, F);
        float U[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            O[m] = R[m] - al * V[m];
            U[m] = F[m] == ST_ACTIVE ? D[m] * O[m] : 0.f;
            if (F[m] == ST_ACTIVE) { double u = (double)D[m] * O[m]; a[0] += u * u; }
        }
        st4(s, q, O);
        if (uo) st4(uo, q, U);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        float sv = r[c] - al * v[c];
        s[c] = sv;
        if (is_active(st, c)) { double u = (double)__ldg(invD + c) * sv; a[0] += u * u; }
        if (uo) uo[c] = is_active(st, c) ? __ldg(invD + c) * sv : 0.f;
    }
    block_sums(a, 1, part);
    if (ctr && last_block(ctr)) {
        double t[1];
        totals_cg(part, gridDim.x, 1, t);
        if (threadIdx.x == 0) { fin_scale(t, S); *ctr = 0u; }
    }
}
// e += alpha ph + omega sh; r = s - omega t; partials ||r||^2, (rhat, r)
__global__ void __launch_bounds__(LB) bs_update_kernel(long long N, float* e, float* r, const float* ph, const float* sh, const float* s,
                                                       const float* t, const float* rh, double* part, Scal* S, unsigned* ctr, int max_iters) {
    if (S->done) return;
    const float al = (float)S->alpha, om = (float)S->omega;
    const long long T = (long long)gridDim.x * LB, t0 = blockIdx.x * (long long)LB + threadIdx.x, NQ = N >> 2;
    double a[2] = {0., 0.};
    for (long long q = t0; q < NQ; q += T) {
        float E[4], PH[4], SH[4], S4[4], T4[4], RH[4], RN[4];
        un4(ld4(e, q), E); un4(ld4(ph, q), PH); un4(ld4(sh, q), SH); un4(ld4(s, q), S4); un4(ld4(t, q), T4); un4(ld4(rh, q), RH);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            E[m] = E[m] + al * PH[m] + om * SH[m];
            RN[m] = S4[m] - om * T4[m];
            a[0] += (double)RN[m] * RN[m];
            a[1] += (double)RH[m] * RN[m];
        }
        st4(e, q, E);
        st4(r, q, RN);
    }
    for (long long c = 4 * NQ + t0; c < N; c += T) {
        e[c] = e[c] + al * ph[c] + om * sh[c];
        float rn = s[c] - om * t[c];
        r[c] = rn;
        a[0] += (double)rn * rn;
        a[1] += (double)rh[c] * rn;
    }
    block_sums(a, 2, part);
    if (ctr && last_block(ctr)) {
        double tt[2];
        totals_cg(part, gridDim.x, 2, tt);
        if (threadIdx.x == 0) { fin_update(tt, S, max_iters); *ctr = 0u; }
    }
}

// active-cell count (the scale of the preconditioner input is an RMS over active cells)
__global__ void __launch_bounds__(LB) count_active_kernel(long long N, const uint8_t* st, double* part) {
    double a[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) a[0] += is_active(st, c) ? 1. : 0.;
    block_sums(a, 1, part);
}
__global__ void count_finish(const double* part, int nblk, double* out) {
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) *out = t[0];
}

// ---------------------------------------------------------------- small kernels
__global__ void mean_kernel(long long N, const double* b, double* part) {
    double v[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) v[0] += b[c];
    block_sums(v, 1, part);
}
__global__ void mean_finish_kernel(const double* part, int nblk, double* out, long long N) {
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x == 0) *out = t[0] / (double)N;
}
__global__ void sub_mean_kernel(long long N, double* b, const double* mean) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) b[c] = b[c] - *mean;
}
__global__ void zero_kernel(long long N, double* x) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) x[c] = 0.;
}
__global__ void cast_kernel(OpSym A, long long N, float* aP, float* aE, float* aN, float* aT, float* invD) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    double d = A.aP[c];
    aP[c] = (float)d; aE[c] = (float)A.aE[c]; aN[c] = (float)A.aN[c]; aT[c] = (float)A.aT[c];
    invD[c] = d != 0. ? (float)(1. / d) : 1.f;
}
// the next stage of a cascade starts its own refinement passes (||b||^2 and the tolerance stay)
__global__ void reopen_kernel(Scal* S) {
    if (threadIdx.x != 0) return;
    S->odone = 0; S->done = 0; S->status = 0; S->stall = 0; S->outer = 0; S->first = 0;
}

__global__ void publish_kernel(const Scal* S, KspOut* out) {
    if (threadIdx.x != 0) return;
    out->iters[0] = S->iters;
    out->iters[1] = S->outer;
    out->relres[0] = S->bb > 0. ? sqrt(S->rr64 / S->bb) : 0.;
    out->status[0] = S->status;
}

// ---------------------------------------------------------------- inner FGMRES (FP32)
// Right-preconditioned flexible GMRES (Saad 1993): z_j = M(v_j), w = A z_j, classical
// Gram-Schmidt against v_0..v_j with FP64 dot accumulation, Givens rotations on the
// Hessenberg column, x = sum y_j z_j at the end of the cycle.  It tolerates any change of M
// between applications, the case of the BF16 network with ReLU.
constexpr int FGM = FGMRES_MAX_RESTART;
constexpr int FG_DOT_BLOCKS = 592;    // 4 x 148 SMs: cell chunks of the multi-dot kernel

struct FgScal {
    double H[(FGM + 1) * FGM];   // column-major: H[j * (FGM + 1) + i]
    double h1[FGM + 1], h2[FGM + 1];   // the two Gram-Schmidt passes of the current column
    double cs[FGM], sn[FGM], g[FGM + 1], y[FGM];
    double beta;
    int jEnd;
};

// v_0 = r / ||r|| (||r||^2 from the outer residual), e = 0
__global__ void fg_init_kernel(long long N, const float* r, float* v0, float* e, const Scal* S, FgScal* F) {
    if (S->done) return;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double beta = sqrt(S->rr64);
    if (c == 0) { F->beta = beta; F->g[0] = beta; F->jEnd = 0; }
    if (c < N) { v0[c] = (float)((double)r[c] / beta); e[c] = 0.f; }
}
__global__ void fg_start_finish(Scal* S, double eta, const double* nact) {
    if (S->done || threadIdx.x != 0) return;
    S->rr0 = S->rr64; S->rr = S->rr64;
    S->tin2 = eta * eta * S->rr64;
    S->nact = *nact;
    S->done = !(S->rr64 > 0.);
}
// partial sum of (D^-1 x)^2 over active cells (the network scale of M(x))
__global__ void __launch_bounds__(LB) scale_partial_kernel(long long N, const float* x, const float* invD, const uint8_t* st, double* part,
                                                           const Scal* S, float* uo) {
    if (S->done) return;
    double a[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        const bool act = is_active(st, c);
        if (act) { double u = (double)__ldg(invD + c) * x[c]; a[0] += u * u; }
        if (uo) uo[c] = act ? __ldg(invD + c) * x[c] : 0.f;
    }
    block_sums(a, 1, part);
}
// w = A z (FP32, with the ghost rows)
template <bool V4>
__global__ void __launch_bounds__(LB) fg_spmv_kernel(OpSymF32 A, long long N, const float* z, float* w, const Scal* S) {
    if (S->done) return;
    long long c0 = 0;
    if (V4) {
        const long long NQ = N >> 2;
        for (long long q = blockIdx.x * (long long)LB + threadIdx.x; q < NQ; q += (long long)gridDim.x * LB) {
            float Y[4];
            spmv4(A, z, q, Y);
            st4(w, q, Y);
        }
        c0 = 4 * NQ;
    }
    for (long long c = c0 + blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB)
        w[c] = applyF(A, c, [&](long long e_) { return z[e_]; });
}
// h[0..j] from the partials (block q sums entry q)
__global__ void fg_dots_finish(const double* part, int nchunk, double* h, const Scal* S) {
    if (S->done) return;
    const int i = blockIdx.x;
    __shared__ double sm[LB];
    double t = 0.;
    for (int b = threadIdx.x; b < nchunk; b += blockDim.x) t += part[(size_t)i * nchunk + b];
    sm[threadIdx.x] = t;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) h[i] = sm[0];
}
// Dot products of w with v_0 .. v_j in one sweep that reads w and every v_i once: each thread
// accumulates its cells' products per i in shared memory (FP32), then each block reduces them
// (FP64) into part[i * gridDim.x + block], the layout fg_dots_finish reads.
__global__ void __launch_bounds__(LB) fg_multidot_kernel(long long N, const float* w, const float* V, long long PS, int j, double* part,
                                                         const Scal* S) {
    if (S->done) return;
    extern __shared__ float fg_sm[];
    float* acc = fg_sm;   // [j + 1][LB]
    const int t = threadIdx.x;
    for (int i = 0; i <= j; ++i) acc[i * LB + t] = 0.f;
    for (long long c = blockIdx.x * (long long)LB + t; c < N; c += (long long)gridDim.x * LB) {
        const float wv = w[c];
        for (int i = 0; i <= j; ++i) acc[i * LB + t] += wv * V[i * PS + c];
    }
    __syncthreads();
    const int warp = t >> 5, lane = t & 31;
    for (int i = warp; i <= j; i += LB / 32) {
        double sacc = 0.;
        for (int u = lane; u < LB; u += 32) sacc += (double)acc[i * LB + u];
        for (int off = 16; off > 0; off >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, off);
        if (lane == 0) part[(size_t)i * gridDim.x + blockIdx.x] = sacc;
    }
}

// First Gram-Schmidt update fused with the second pass's dot products: w <- w - sum_i h1[i] v_i and
// the dots (w, v_i) of the updated w, reading every v_i once (each thread keeps its cell's v_i in
// shared memory between the update and the dots).  Partials as fg_multidot_kernel's.
__global__ void __launch_bounds__(LB) fg_orth_dots_kernel(long long N, float* w, const float* V, long long PS, int j, const double* h1,
                                                          double* part, const Scal* S) {
    if (S->done) return;
    extern __shared__ float fg_sm[];
    float* acc = fg_sm;                  // [j + 1][LB]
    float* vs = fg_sm + (j + 1) * LB;    // [j + 1][LB]
    __shared__ float h[FGM + 1];
    const int t = threadIdx.x;
    for (int i = t; i <= j; i += blockDim.x) h[i] = (float)h1[i];
    for (int i = 0; i <= j; ++i) acc[i * LB + t] = 0.f;
    __syncthreads();
    for (long long c = blockIdx.x * (long long)LB + t; c < N; c += (long long)gridDim.x * LB) {
        float x = w[c];
        for (int i = 0; i <= j; ++i) {
            const float v = V[i * PS + c];
            vs[i * LB + t] = v;
            x -= h[i] * v;
        }
        w[c] = x;
        for (int i = 0; i <= j; ++i) acc[i * LB + t] += x * vs[i * LB + t];
    }
    __syncthreads();
    const int warp = t >> 5, lane = t & 31;
    for (int i = warp; i <= j; i += LB / 32) {
        double sacc = 0.;
        for (int u = lane; u < LB; u += 32) sacc += (double)acc[i * LB + u];
        for (int off = 16; off > 0; off >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, off);
        if (lane == 0) part[(size_t)i * gridDim.x + blockIdx.x] = sacc;
    }
}

// w -= sum_i h[i] v_i; partial ||w||^2
__global__ void __launch_bounds__(LB) fg_orth_kernel(long long N, float* w, const float* V, long long PS, int j, const double* hc, double* part,
                                                     const Scal* S) {
    if (S->done) return;
    __shared__ float h[FGM + 1];
    for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = (float)hc[i];
    __syncthreads();
    double a[1] = {0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float x = w[c];
        for (int i = 0; i <= j; ++i) x -= h[i] * V[i * PS + c];
        w[c] = x;
        a[0] += (double)x * x;
    }
    block_sums(a, 1, part);
}
// h_{j+1,j}, rotations, residual estimate, stop test
__global__ void fg_step_finish(const double* part, int nblk, int j, int m, int max_iters, FgScal* F, Scal* S) {
    if (S->done) return;
    double t[1];
    totals(part, nblk, 1, t);
    if (threadIdx.x != 0) return;
    double* Hc = F->H + (size_t)j * (FGM + 1);
    for (int i = 0; i <= j; ++i) Hc[i] = F->h1[i] + F->h2[i];   // classical Gram-Schmidt, two passes
    double hn = sqrt(t[0]);
    Hc[j + 1] = hn;
    for (int i = 0; i < j; ++i) {
        double a = Hc[i], b = Hc[i + 1];
        Hc[i] = F->cs[i] * a + F->sn[i] * b;
        Hc[i + 1] = -F->sn[i] * a + F->cs[i] * b;
    }
    double a = Hc[j], b = Hc[j + 1];
    double r = sqrt(a * a + b * b);
    double c = r > 0. ? a / r : 1., sn = r > 0. ? b / r : 0.;
    F->cs[j] = c; F->sn[j] = sn;
    Hc[j] = r; Hc[j + 1] = 0.;
    F->g[j + 1] = -sn * F->g[j];
    F->g[j] = c * F->g[j];
    double res2 = F->g[j + 1] * F->g[j + 1];
    S->rr = res2;
    S->iters += 1;
    F->jEnd = j + 1;
    bool stop = res2 <= S->tin2 || j + 1 >= m || S->iters >= max_iters || !(hn > 0.) || res2 != res2;
    if (stop) S->done = 1;
    S->alpha = hn > 0. ? 1. / hn : 0.;   // scale of the next basis vector
}
// v_{j+1} = w / h_{j+1,j}
__global__ void fg_scale_kernel(long long N, const float* w, float* vn, const Scal* S) {
    if (S->done) return;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) vn[c] = (float)((double)w[c] * S->alpha);
}
// y = R^-1 g (upper triangular, jEnd x jEnd)
__global__ void fg_solve_kernel(FgScal* F) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = F->jEnd;
    for (int i = n - 1; i >= 0; --i) {
        double s = F->g[i];
        for (int k = i + 1; k < n; ++k) s -= F->H[(size_t)k * (FGM + 1) + i] * F->y[k];
        double d = F->H[(size_t)i * (FGM + 1) + i];
        F->y[i] = d != 0. ? s / d : 0.;
    }
}
// e = sum_i y_i z_i
__global__ void __launch_bounds__(LB) fg_combine_kernel(long long N, const float* Z, long long PS, const FgScal* F, float* e) {
    __shared__ float y[FGM];
    const int n = F->jEnd;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (float)F->y[i];
    __syncthreads();
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float a = 0.f;
        for (int i = 0; i < n; ++i) a += y[i] * Z[i * PS + c];
        e[c] = a;
    }
}

// ---------------------------------------------------------------- pyramid host side
Dims3 dims_of(const Level& l) { return Dims3{l.n[0], l.n[1], l.n[2]}; }

// Restriction chain, the network (or the identity) on every coarse level, prolongation chain
// (result in lev[1].w).  Every kernel is a no-op while S->done is set.
// ufine: optional D^-1 rfine on active cells, 0 elsewhere (written by the kernel that produced
// rfine); with it the restriction to level 1 stages one array instead of three
int apply_levels(LearnedWork& lw, const float* rfine, const uint8_t* status, int mode, Scal* S, cudaStream_t st, const float* ufine = nullptr) {
    if (mode == NET_MODE_JACOBI || lw.nLev < 2) return 0;
    auto netAt = [&](int l) { return mode == NET_MODE_NETWORK && l >= lw.netFrom && l <= lw.netTo; };
    // the coarse tail: from the first level lt >= 2 whose finer neighbour has at most TAIL_MAX_IN
    // cells and from which on no level runs the network, one kernel does the rest of the pyramid
    int lt = lw.nLev;
    long long tailCells = 0;   // u and w of the tail levels, in shared memory with the staged input
    for (int l = lw.nLev - 1; l >= 2; --l) {
        if (netAt(l) || lw.lev[l - 1].N > TAIL_MAX_IN) break;
        if ((size_t)(lw.lev[l - 1].N + 2 * (tailCells + lw.lev[l].N)) * sizeof(float) > 48 * 1024) break;
        tailCells += lw.lev[l].N;
        lt = l;
    }
    for (int l = 1; l < lt; ++l) {
        Level& c = lw.lev[l];
        const Level& f = lw.lev[l - 1];
        if (l == 1 && !netAt(1) && lw.rtErr && ufine && restrict_tma_usable(dims_of(f), ufine, nullptr, nullptr)) {
            if (launch_restrict_tma(dims_of(f), dims_of(c), ufine, nullptr, nullptr, c.rscale, c.u, lw.rtErr, S, st)) return 1;
            continue;
        }
        if (l == 1 && !netAt(1) && lw.rtErr && restrict_tma_usable(dims_of(f), rfine, lw.invD, status)) {
            if (launch_restrict_tma(dims_of(f), dims_of(c), rfine, lw.invD, status, c.rscale, c.u, lw.rtErr, S, st)) return 1;
            continue;
        }
        // deeper levels: the input is already plain values, the staged form of the restriction
        // applies where the level has tiles enough for two per SM
        if (l >= 2 && !netAt(l) && lw.rtErr && restrict_tiles(dims_of(c)) >= 2 * 148 &&
            restrict_tma_usable(dims_of(f), f.u, nullptr, nullptr)) {
            if (launch_restrict_tma(dims_of(f), dims_of(c), f.u, nullptr, nullptr, c.rscale, c.u, lw.rtErr, S, st)) return 1;
            continue;
        }
        restrict_kernel<<<restrict_grid(dims_of(c)), 256, 0, st>>>(dims_of(f), dims_of(c), l == 1 ? rfine : f.u, l == 1 ? lw.invD : nullptr,
                                                                   l == 1 ? status : nullptr, c.rscale, c.u, nullptr, 0.f,
                                                                   netAt(l) ? c.net.act[0] : nullptr, netAt(l) ? c.netNeg.act[0] : nullptr,
                                                                   c.mask, c.chan, S);
    }
    CB_CHECK_LAUNCH();
    // every network level and both signs of the odd form: one grouped launch per layer
    {
        NetBuffers* nets[2 * LEARN_MAX_LEVELS];
        int nn = 0;
        for (int l = 1; l < lw.nLev; ++l)
            if (netAt(l)) { nets[nn++] = &lw.lev[l].net; nets[nn++] = &lw.lev[l].netNeg; }
        if (nn > 0 && net_forward_group_if(nets, nn, &S->done, st)) return 1;
    }
    if (lt < lw.nLev) {
        TailArgs ta;
        std::memset(&ta, 0, sizeof(ta));
        ta.n = lw.nLev - lt;
        ta.d[0] = dims_of(lw.lev[lt - 1]);
        ta.uin = lw.lev[lt - 1].u;
        long long cells = lw.lev[lt - 1].N;
        for (int q = 0; q < ta.n; ++q) {
            Level& c = lw.lev[lt + q];
            ta.d[q + 1] = dims_of(c);
            ta.rscale[q] = c.rscale;
            ta.gain[q] = c.gain;
            ta.u[q] = c.u;
            ta.w[q] = c.w;
            cells += 2 * c.N;
        }
        coarse_tail_kernel<<<1, TAIL_THREADS, sizeof(float) * (size_t)cells, st>>>(ta, S);
        CB_CHECK_LAUNCH();
    }
    for (int l = lt - 1; l >= 1; --l) {
        Level& f = lw.lev[l];
        const bool top = l + 1 >= lw.nLev;
        const float* y = netAt(l) ? f.net.y : f.u;
        const float* yn = netAt(l) ? f.netNeg.y : nullptr;
        auto a16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
        if ((f.N & 3) == 0 && a16(y) && a16(f.w) && (!yn || a16(yn)))
            prolong4_kernel<<<grid_for(f.N / 4, 256), 256, 0, st>>>(dims_of(f), top ? dims_of(f) : dims_of(lw.lev[l + 1]),
                                                                    top ? nullptr : lw.lev[l + 1].w, y, yn, netAt(l) ? 0 : 1, f.gain,
                                                                    f.w, S);
        else
            prolong_kernel<<<grid_for(f.N, 256), 256, 0, st>>>(dims_of(f), top ? dims_of(f) : dims_of(lw.lev[l + 1]),
                                                               top ? nullptr : lw.lev[l + 1].w, y, yn, netAt(l) ? 0 : 1, f.gain, f.w, S);
    }
    CB_CHECK_LAUNCH();
    return 0;
}

const float* level_w1(const LearnedWork& lw, int mode) { return (mode == NET_MODE_JACOBI || lw.nLev < 2) ? nullptr : lw.lev[1].w; }
Dims3 level1_dims(const LearnedWork& lw) { return lw.nLev >= 2 ? dims_of(lw.lev[1]) : dims_of(lw.lev[0]); }

// masks of the coarse levels: fraction of active fine cells
int level_masks(LearnedWork& lw, const uint8_t* status, cudaStream_t st) {
    for (int l = 1; l < lw.nLev; ++l) {
        Level& c = lw.lev[l];
        const Level& f = lw.lev[l - 1];
        restrict_kernel<<<restrict_grid(dims_of(c)), 256, 0, st>>>(dims_of(f), dims_of(c), l == 1 ? nullptr : f.mask, nullptr,
                                                                   l == 1 ? status : nullptr, c.rscale, c.mask, nullptr, 0.f, nullptr,
                                                                   nullptr, nullptr, 0.f, nullptr);
    }
    CB_CHECK_LAUNCH();
    lw.masksReady = true;
    return 0;
}

OpSymF32 cast_operator(LearnedWork& lw, const OpSym& A, const Lat& L, cudaStream_t st) {
    cast_kernel<<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, lw.A[0], lw.A[1], lw.A[2], lw.A[3], lw.invD);
    OpSymF32 Af;
    Af.aP = lw.A[0]; Af.aE = lw.A[1]; Af.aN = lw.A[2]; Af.aT = lw.A[3]; Af.nI = A.nI; Af.nIJ = A.nIJ; Af.gh = A.gh;
    return Af;
}

}  // namespace

int learned_alloc(LearnedWork& lw, const Lat& L, void* (*alloc)(size_t, void*), void* ctx) {
    lw.L = L;
    lw.alloc = alloc;
    lw.allocCtx = ctx;
    auto fcell = [&]() -> float* {
        float* b = static_cast<float*>(alloc(sizeof(float) * (size_t)L.PS, ctx));
        return b ? b + L.H : nullptr;
    };
    lw.r = fcell(); lw.z = fcell(); lw.e = fcell(); lw.u1 = fcell();
    lw.p[0] = fcell(); lw.p[1] = fcell(); lw.q[0] = fcell(); lw.q[1] = fcell();
    lw.t = fcell(); lw.rh = fcell();
    lw.invD = fcell();
    for (int q = 0; q < 4; ++q) lw.A[q] = fcell();
    lw.part = static_cast<double*>(alloc(sizeof(double) * 4 * MAXP, ctx));
    lw.scal = alloc(sizeof(Scal), ctx);
    lw.mean = static_cast<double*>(alloc(sizeof(double) * 2, ctx));
    lw.rtErr = static_cast<int*>(alloc(sizeof(int) * 4, ctx));
    lw.ctr = static_cast<unsigned*>(alloc(sizeof(unsigned) * 4, ctx));
    bool ok = lw.r && lw.z && lw.e && lw.p[0] && lw.p[1] && lw.q[0] && lw.q[1] && lw.t && lw.rh && lw.invD && lw.part && lw.scal && lw.mean &&
              lw.rtErr && lw.ctr && lw.u1;
    for (int q = 0; q < 4; ++q) ok = ok && lw.A[q];
    if (!ok) { set_error("learned-solver allocation failed"); return 1; }
    if (cudaMallocHost(&lw.hostScal, sizeof(Scal)) != cudaSuccess) { set_error("pinned allocation failed"); return 1; }
    // level pyramid: halve every direction longer than one cell until about 64 cells remain
    Level& l0 = lw.lev[0];
    l0.n[0] = L.nI; l0.n[1] = L.nJ; l0.n[2] = L.nK; l0.N = L.N; l0.rscale = 1.f; l0.gain = 1.f; l0.chan = 0.f;
    lw.nLev = 1;
    while (lw.nLev < LEARN_MAX_LEVELS) {
        const Level& f = lw.lev[lw.nLev - 1];
        if (f.N <= 64 || (f.n[0] == 1 && f.n[1] == 1 && f.n[2] == 1)) break;
        Level& c = lw.lev[lw.nLev];
        int coarsened = 0;
        for (int d = 0; d < 3; ++d) {
            c.n[d] = f.n[d] > 1 ? (f.n[d] + 1) / 2 : 1;
            coarsened += f.n[d] > 1;
        }
        c.N = (long long)c.n[0] * c.n[1] * c.n[2];
        c.rscale = 1.f / (float)(1 << coarsened);
        c.gain = f.gain * 4.f;
        c.chan = (float)lw.nLev / 8.f;
        c.u = static_cast<float*>(alloc(sizeof(float) * (size_t)c.N, ctx));
        c.w = static_cast<float*>(alloc(sizeof(float) * (size_t)c.N, ctx));
        c.mask = static_cast<float*>(alloc(sizeof(float) * (size_t)c.N, ctx));
        if (!c.u || !c.w || !c.mask) { set_error("learned-solver allocation failed"); return 1; }
        Lat Lc = make_lat(c.n[0], c.n[1], c.n[2]);
        int rc = lw.nLev == 1 ? net_alloc(c.net, Lc, alloc, ctx) : net_alloc_shared(c.net, Lc, lw.lev[1].net, alloc, ctx);
        if (rc || net_alloc_shared(c.netNeg, Lc, lw.lev[1].net, alloc, ctx)) return 1;
        c.w2 = static_cast<float*>(alloc(sizeof(float) * (size_t)c.N, ctx));
        if (!c.w2) { set_error("learned-solver allocation failed"); return 1; }
        ++lw.nLev;
    }
    lw.weights = lw.nLev >= 2 ? &lw.lev[1].net : nullptr;
    lw.masksReady = false;
    return 0;
}

void learned_free_host(LearnedWork& lw) {
    if (lw.hostScal) cudaFreeHost(lw.hostScal);
    lw.hostScal = nullptr;
}

namespace {
int fg_alloc(LearnedWork& lw, int m) {
    if (lw.fgCap >= m) return 0;
    if (lw.fgCap > 0) { set_error("FGMRES restart length cannot grow after the first FGMRES solve"); return 1; }
    const Lat& L = lw.L;
    lw.fgV = static_cast<float*>(lw.alloc(sizeof(float) * (size_t)L.PS * (m + 1), lw.allocCtx));
    lw.fgZ = static_cast<float*>(lw.alloc(sizeof(float) * (size_t)L.PS * m, lw.allocCtx));
    lw.fgScal = lw.alloc(sizeof(FgScal), lw.allocCtx);
    lw.fgPart = static_cast<double*>(lw.alloc(sizeof(double) * (size_t)(FGM + 1) * FG_DOT_BLOCKS, lw.allocCtx));
    if (!lw.fgV || !lw.fgZ || !lw.fgScal || !lw.fgPart) { set_error("FGMRES workspace allocation failed"); return 1; }
    lw.fgCap = m;
    // the fused Gram-Schmidt kernels keep (m + 1) x LB floats (twice, for the update + dots one)
    const int smMax = (int)(2 * sizeof(float) * (size_t)(FGM + 1) * LB);
    if (cudaFuncSetAttribute(fg_multidot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smMax) != cudaSuccess ||
        cudaFuncSetAttribute(fg_orth_dots_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smMax) != cudaSuccess) {
        set_error("FGMRES kernels: shared-memory attribute refused");
        return 1;
    }
    return 0;
}
}  // namespace

int learned_solve(LearnedWork& lw, const OpSym& A, const uint8_t* status, const double* b, double* x, const Lat& L, double rtol, int maxit,
                  double eta, int project, int mode, KspOut* out, cudaStream_t st, double atol) {
    const long long N = L.N;
    const int nb = nblocks(N);
    const int G = grid_for(N, 256);
    Scal* S = static_cast<Scal*>(lw.scal);
    if (mode == NET_MODE_NETWORK && (!lw.haveParams || lw.nLev < 2)) mode = NET_MODE_JACOBI;
    if (mode != NET_MODE_JACOBI && !lw.masksReady && level_masks(lw, status, st)) return 1;
    OpSymF32 Af = cast_operator(lw, A, L, st);
    if (project) {
        mean_kernel<<<nb, LB, 0, st>>>(N, b, lw.part);
        mean_finish_kernel<<<1, LB, 0, st>>>(lw.part, nb, lw.mean, N);
        sub_mean_kernel<<<G, 256, 0, st>>>(N, const_cast<double*>(b), lw.mean);
    }
    zero_kernel<<<G, 256, 0, st>>>(N, x);
    Scal init;
    std::memset(&init, 0, sizeof(init));
    init.first = 1;
    CB_CUDA(cudaMemcpyAsync(S, &init, sizeof(Scal), cudaMemcpyHostToDevice, st));
    CB_CHECK_LAUNCH();
    const Dims3 fd = dims_of(lw.lev[0]), cd = level1_dims(lw);
    const bool nonsym = A.gh.n > 0;
    // 4-cell vector rows: neighbouring groups of 4 cells stay 16-byte aligned
    const bool v4 = (L.nI % 4) == 0 && (L.nIJ % 4) == 0;
    int method = lw.inner;
    if (method == LEARN_INNER_AUTO)
        method = !nonsym ? LEARN_INNER_FCG : (mode == NET_MODE_NETWORK ? LEARN_INNER_FGMRES : LEARN_INNER_BICGSTAB);
    const int m = lw.restart < 1 ? 1 : (lw.restart > FGM ? FGM : lw.restart);
    if (method == LEARN_INNER_FGMRES && fg_alloc(lw, m)) return 1;
    FgScal* F = static_cast<FgScal*>(lw.fgScal);
    const long long PS = L.PS;
    if (method != LEARN_INNER_FCG) {
        count_active_kernel<<<nb, LB, 0, st>>>(N, status, lw.part);
        count_finish<<<1, LB, 0, st>>>(lw.part, nb, lw.mean + 1);
    }
    // One stage of the solve: FP64 refinement passes around the inner method `smethod` with the
    // preconditioner form `smode`, from the current x; inner iterations are capped at iterCap
    // (counted over the whole solve).
    auto stage = [&](int smode, int smethod, int iterCap) -> int {
        const int maxit = iterCap;
        const int mode = smode;
        const float* w1 = level_w1(lw, mode);
        const bool symmetric = smethod == LEARN_INNER_FCG;
        const bool fgmres = smethod == LEARN_INNER_FGMRES;
        // FGMRES: one restart cycle per refinement pass, as many cycles as the iteration budget
        // allows, at most 100
        const int max_outer = fgmres ? std::min(100, std::max(12, maxit / m + 1)) : 12;
        const int chunk = 8;
        for (int outer = 0; outer <= max_outer; ++outer) {
            outer_residual_kernel<<<nb, LB, 0, st>>>(A, N, b, x, lw.r, lw.part, S);
            outer_check_kernel<<<1, LB, 0, st>>>(lw.part, nb, S, max_outer);
            CB_CUDA(cudaMemcpyAsync(lw.hostScal, S, sizeof(Scal), cudaMemcpyDeviceToHost, st));
            CB_CUDA(cudaStreamSynchronize(st));
            Scal* hs = static_cast<Scal*>(lw.hostScal);
            if (outer == 0) {
                // the tolerance needs ||b||^2: the first outer residual (x = 0) is b itself
                double tol2 = std::max(rtol * rtol * hs->bb, atol * atol);
                bool fin = hs->rr64 <= tol2 || !(hs->bb > 0.);
                CB_CUDA(cudaMemcpyAsync(&S->tol2, &tol2, sizeof(double), cudaMemcpyHostToDevice, st));
                if (fin) {
                    int one = 1;
                    CB_CUDA(cudaMemcpyAsync(&S->odone, &one, sizeof(int), cudaMemcpyHostToDevice, st));
                    break;
                }
            } else if (hs->odone) {
                break;
            }
            // inner target: deep first, then only the factor still missing
            double etaK = eta;
            if (hs->bb > 0. && hs->rr64 > 0.) {
                double need = 0.25 * sqrt(std::max(rtol * rtol * hs->bb, atol * atol) / hs->rr64);
                if (need > etaK) etaK = need;
            }
            if (etaK > 0.5) etaK = 0.5;
            int cur = 0;
            if (fgmres) {
                fg_init_kernel<<<G, 256, 0, st>>>(N, lw.r, lw.fgV + L.H, lw.e, S, F);
                fg_start_finish<<<1, 32, 0, st>>>(S, etaK, lw.mean + 1);
                CB_CHECK_LAUNCH();
                for (int j = 0; j < m; ++j) {
                    float* vj = lw.fgV + j * PS + L.H;
                    float* zj = lw.fgZ + j * PS + L.H;
                    scale_partial_kernel<<<nb, LB, 0, st>>>(N, vj, lw.invD, status, lw.part, S, lw.u1);
                    scale_finish<<<1, LB, 0, st>>>(lw.part, nb, S);
                    if (apply_levels(lw, vj, status, mode, S, st, lw.u1)) return 1;
                    bs_z_kernel<<<nb, LB, 0, st>>>(N, fd, cd, vj, lw.invD, status, w1, zj, S);
                    if (v4) fg_spmv_kernel<true><<<nb, LB, 0, st>>>(Af, N, zj, lw.t, S);
                    else fg_spmv_kernel<false><<<nb, LB, 0, st>>>(Af, N, zj, lw.t, S);
                    // classical Gram-Schmidt with one re-orthogonalisation (CGS2): FP32 vectors lose
                    // orthogonality in a single pass once the preconditioner is strong.  Three sweeps over
                    // the basis: the first pass's dots, its update fused with the second pass's dots, and
                    // the second pass's update (with ||w||^2).
                    {
                        const size_t sm1 = sizeof(float) * (size_t)(j + 1) * LB;
                        fg_multidot_kernel<<<FG_DOT_BLOCKS, LB, sm1, st>>>(N, lw.t, lw.fgV + L.H, PS, j, lw.fgPart, S);
                        fg_dots_finish<<<j + 1, LB, 0, st>>>(lw.fgPart, FG_DOT_BLOCKS, F->h1, S);
                        fg_orth_dots_kernel<<<FG_DOT_BLOCKS, LB, 2 * sm1, st>>>(N, lw.t, lw.fgV + L.H, PS, j, F->h1, lw.fgPart, S);
                        fg_dots_finish<<<j + 1, LB, 0, st>>>(lw.fgPart, FG_DOT_BLOCKS, F->h2, S);
                        fg_orth_kernel<<<nb, LB, 0, st>>>(N, lw.t, lw.fgV + L.H, PS, j, F->h2, lw.part, S);
                    }
                    fg_step_finish<<<1, LB, 0, st>>>(lw.part, nb, j, m, maxit, F, S);
                    fg_scale_kernel<<<G, 256, 0, st>>>(N, lw.t, lw.fgV + (j + 1) * PS + L.H, S);
                    // no host wait inside a cycle: once the cycle's `done` is set on the device, the
                    // remaining iterations' kernels return at once
                }
                fg_solve_kernel<<<1, 32, 0, st>>>(F);
                fg_combine_kernel<<<nb, LB, 0, st>>>(N, lw.fgZ + L.H, PS, F, lw.e);
                CB_CHECK_LAUNCH();
                outer_update_kernel<<<G, 256, 0, st>>>(N, x, lw.e, S);
                int zero = 0;
                CB_CUDA(cudaMemcpyAsync(&S->done, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
                continue;
            }
            if (symmetric) {
                inner_start_kernel<<<nb, LB, 0, st>>>(N, lw.r, lw.invD, status, lw.e, lw.p[0], lw.q[0], lw.part, S);
                inner_start_finish_kernel<<<1, LB, 0, st>>>(lw.part, nb, S, etaK);
            } else {
                bs_start_kernel<<<nb, LB, 0, st>>>(N, lw.r, lw.rh, lw.e, lw.p[0], lw.q[0], lw.part, S);
                bs_start_finish<<<1, LB, 0, st>>>(lw.part, nb, S, etaK, lw.mean + 1);
            }
            bool innerDone = false;
            while (!innerDone) {
                for (int it = 0; it < chunk; ++it) {
                    if (symmetric) {
                        if (apply_levels(lw, lw.r, status, mode, S, st)) return 1;
                        precond_z_kernel<<<nb, LB, 0, st>>>(N, fd, cd, lw.r, lw.invD, status, w1, lw.z, lw.q[cur], lw.part, S);
                        beta_kernel<<<1, LB, 0, st>>>(lw.part, nb, S);
                        direction_kernel<<<nb, LB, 0, st>>>(Af, N, lw.z, lw.p[cur], lw.p[cur ^ 1], lw.q[cur ^ 1], lw.r, lw.part, S);
                        alpha_kernel<<<1, LB, 0, st>>>(lw.part, nb, S);
                        step_kernel<<<nb, LB, 0, st>>>(N, lw.e, lw.r, lw.p[cur ^ 1], lw.q[cur ^ 1], lw.invD, status, lw.part, S);
                        step_finish_kernel<<<1, LB, 0, st>>>(lw.part, nb, S, maxit);
                        cur ^= 1;
                    } else {
                        // p = p[0], v = q[0], ph = p[1], sh = q[1], s = z, t = t
                        bs_dir_kernel<<<nb, LB, 0, st>>>(N, lw.r, lw.q[0], lw.invD, status, lw.p[0], lw.part, S, lw.ctr, lw.u1);
                        if (apply_levels(lw, lw.p[0], status, mode, S, st, lw.u1)) return 1;
                        bs_z_kernel<<<nb, LB, 0, st>>>(N, fd, cd, lw.p[0], lw.invD, status, w1, lw.p[1], S);
                        if (v4) bs_spmv_kernel<true><<<nb, LB, 0, st>>>(Af, N, lw.p[1], lw.q[0], lw.rh, nullptr, lw.part, S, lw.ctr);
                        else bs_spmv_kernel<false><<<nb, LB, 0, st>>>(Af, N, lw.p[1], lw.q[0], lw.rh, nullptr, lw.part, S, lw.ctr);
                        bs_s_kernel<<<nb, LB, 0, st>>>(N, lw.r, lw.q[0], lw.invD, status, lw.z, lw.part, S, lw.ctr, lw.u1);
                        if (apply_levels(lw, lw.z, status, mode, S, st, lw.u1)) return 1;
                        bs_z_kernel<<<nb, LB, 0, st>>>(N, fd, cd, lw.z, lw.invD, status, w1, lw.q[1], S);
                        if (v4) bs_spmv_kernel<true><<<nb, LB, 0, st>>>(Af, N, lw.q[1], lw.t, nullptr, lw.z, lw.part, S, lw.ctr);
                        else bs_spmv_kernel<false><<<nb, LB, 0, st>>>(Af, N, lw.q[1], lw.t, nullptr, lw.z, lw.part, S, lw.ctr);
                        bs_update_kernel<<<nb, LB, 0, st>>>(N, lw.e, lw.r, lw.p[1], lw.q[1], lw.z, lw.t, lw.rh, lw.part, S, lw.ctr, maxit);
                    }
                }
                CB_CHECK_LAUNCH();
                CB_CUDA(cudaMemcpyAsync(lw.hostScal, S, sizeof(Scal), cudaMemcpyDeviceToHost, st));
                CB_CUDA(cudaStreamSynchronize(st));
                Scal* h2 = static_cast<Scal*>(lw.hostScal);
                innerDone = h2->done != 0;
                if (h2->iters >= maxit) break;
            }
            outer_update_kernel<<<G, 256, 0, st>>>(N, x, lw.e, S);
            // the next outer pass re-opens the inner solve
            int zero = 0;
            CB_CUDA(cudaMemcpyAsync(&S->done, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
        }
        return 0;
    };
    if (stage(mode, method, maxit)) return 1;
    // Cascade: a solve whose network stage stalled (three refinement passes in a row that each
    // leave more than 90% of the true residual) or ran out of passes continues, from the iterate
    // it reached, with the same pyramid and an identity in place of the network (a fixed linear
    // preconditioner, so BiCGStab or flexible CG apply); only a solve that misses the tolerance
    // there too leaves status != 0 for the plain FP64 re-solve.
    int cascades = 0, netIters = 0;
    {
        Scal* hs = static_cast<Scal*>(lw.hostScal);
        if (mode == NET_MODE_NETWORK) netIters = hs->iters;
        if (mode == NET_MODE_NETWORK && (hs->status == 1 || hs->status == 2)) {
            const int itersSoFar = hs->iters;
            reopen_kernel<<<1, 32, 0, st>>>(S);
            CB_CHECK_LAUNCH();
            cascades = 1;
            if (stage(NET_MODE_LEVELS, nonsym ? LEARN_INNER_BICGSTAB : LEARN_INNER_FCG, itersSoFar + maxit)) return 1;
        }
    }
    CB_CUDA(cudaMemcpyAsync(&out->cascades, &cascades, sizeof(int), cudaMemcpyHostToDevice, st));
    CB_CUDA(cudaMemcpyAsync(&out->net_iters, &netIters, sizeof(int), cudaMemcpyHostToDevice, st));
    publish_kernel<<<1, 32, 0, st>>>(S, out);
    CB_CHECK_LAUNCH();
    CB_CUDA(cudaMemcpyAsync(lw.hostScal, S, sizeof(Scal), cudaMemcpyDeviceToHost, st));
    int rtErr = 0;
    if (lw.rtErr) CB_CUDA(cudaMemcpyAsync(&rtErr, lw.rtErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
    if (rtErr) { set_error("a TMA load of the staged restriction did not complete"); return 1; }
    lw.lastIters = static_cast<Scal*>(lw.hostScal)->iters;
    lw.lastOuter = static_cast<Scal*>(lw.hostScal)->outer;
    return 0;
}

// ---------------------------------------------------------------- training pairs
namespace {

// Pair of an intermediate iterate x_k of a plain solve: residual r_k = b - A x_k (FP64, then
// rounded) and correction e_k = x* - x_k, so that A e_k = r_k.
__global__ void __launch_bounds__(LB) snapshot_pair_kernel(OpSym A, long long N, const double* b, const double* xs, const double* xk, float* pb,
                                                           float* px) {
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        double y = __ldg(A.aP + c) * xk[c] + __ldg(A.aE + c) * xk[c + 1] + __ldg(A.aE + c - 1) * xk[c - 1]
                   + __ldg(A.aN + c) * xk[c + A.nI] + __ldg(A.aN + c - A.nI) * xk[c - A.nI]
                   + __ldg(A.aT + c) * xk[c + A.nIJ] + __ldg(A.aT + c - A.nIJ) * xk[c - A.nIJ];
        if (A.gh.n > 0) {
            uint32_t w = __ldg(A.gh.bits + (c >> 5));
            if ((w >> (c & 31)) & 1u) {
                int lo = 0, hi = A.gh.n;
                while (lo < hi) { int mid = (lo + hi) >> 1; if (__ldg(A.gh.cell + mid) < c) lo = mid + 1; else hi = mid; }
                double s = 0.;
                for (int m = 0; m < 9; ++m) { int col = __ldg(A.gh.col + 9 * lo + m); if (col >= 0) s += __ldg(A.gh.val + 9 * lo + m) * xk[col]; }
                y = s;
            }
        }
        pb[c] = (float)(b[c] - y);
        px[c] = (float)(xs[c] - xk[c]);
    }
}

}  // namespace

int learned_snapshot_pair(const OpSym& A, const Lat& L, const double* b, const double* xstar, const double* xk, float* pb, float* px,
                          cudaStream_t st) {
    snapshot_pair_kernel<<<nblocks(L.N), LB, 0, st>>>(A, L.N, b, xstar, xk, pb, px);
    CB_CHECK_LAUNCH();
    return 0;
}

// ---------------------------------------------------------------- random multi-scale pairs
namespace {

// uniform in [-1, 1) from a 64-bit integer hash (splitmix64 finaliser) of (seed, pair, cell)
__device__ __forceinline__ float hash_uniform(unsigned seed, unsigned q, unsigned long long c) {
    unsigned long long x = c + 0x9E3779B97F4A7C15ull * (((unsigned long long)seed << 32) ^ (unsigned long long)(q + 1));
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    return (float)((double)(x >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
}
__global__ void rand_fill_kernel(long long n, unsigned seed, unsigned q, float* out) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < n) out[c] = hash_uniform(seed, q, (unsigned long long)c);
}
// out = P wc on the finer level fd (mask: zero on non-active cells of the cell lattice)
__global__ void prolong_only_kernel(Dims3 fd, Dims3 cd, const float* wc, const uint8_t* st, float* out) {
    long long Nf = (long long)fd.n0 * fd.n1 * fd.n2;
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= Nf) return;
    out[f] = (st && st[f] != ST_ACTIVE) ? 0.f : prolong_at(fd, cd, wc, f);
}
__global__ void mask_active_kernel(long long N, const uint8_t* st, float* x) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N && st && st[c] != ST_ACTIVE) x[c] = 0.f;
}
__global__ void __launch_bounds__(LB) apply_f32_kernel(OpSymF32 A, long long N, const float* x, float* y) {
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB)
        y[c] = applyF(A, c, [&](long long e_) { return x[e_]; });
}

}  // namespace

int learned_random_pairs(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, int nPairs, unsigned seed, float* pairsB,
                         float* pairsX, cudaStream_t st) {
    OpSymF32 Af = cast_operator(lw, A, L, st);
    const long long N = L.N;
    for (int q = 0; q < nPairs; ++q) {
        float* b = pairsB + (size_t)q * L.PS + L.H;
        float* e = pairsX + (size_t)q * L.PS + L.H;
        const int l = lw.nLev > 1 ? q % lw.nLev : 0;
        if (l == 0) {
            rand_fill_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, seed, (unsigned)q, e);
            mask_active_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, status, e);
        } else {
            rand_fill_kernel<<<grid_for(lw.lev[l].N, 256), 256, 0, st>>>(lw.lev[l].N, seed, (unsigned)q, lw.lev[l].w);
            for (int k = l - 1; k >= 1; --k)
                prolong_only_kernel<<<grid_for(lw.lev[k].N, 256), 256, 0, st>>>(dims_of(lw.lev[k]), dims_of(lw.lev[k + 1]), lw.lev[k + 1].w,
                                                                               nullptr, lw.lev[k].w);
            prolong_only_kernel<<<grid_for(N, 256), 256, 0, st>>>(dims_of(lw.lev[0]), dims_of(lw.lev[1]), lw.lev[1].w, status, e);
        }
        apply_f32_kernel<<<nblocks(N), LB, 0, st>>>(Af, N, e, b);
        CB_CHECK_LAUNCH();
    }
    return 0;
}

// ---------------------------------------------------------------- training
namespace {

struct TrainScal {
    double s, coef, loss, loss_sum;
};

__global__ void half_split_kernel(long long n, float* a, float* b) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < n) { float v = 0.5f * a[c]; a[c] = v; b[c] = -v; }
}

__global__ void __launch_bounds__(LB) train_scale_kernel(long long N, const float* b, const float* invD, const uint8_t* st, double* part) {
    double v[2] = {0., 0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        if (!is_active(st, c)) continue;
        double u = (double)__ldg(invD + c) * b[c];
        v[0] += u * u; v[1] += 1.;
    }
    block_sums(v, 2, part);
}
__global__ void train_scale_finish(const double* part, int nblk, TrainScal* T, Scal* S) {
    double t[2];
    totals(part, nblk, 2, t);
    if (threadIdx.x == 0) {
        double sc = t[1] > 0. ? sqrt(t[0] / t[1]) : 1.;
        if (!(sc > 0.)) sc = 1.;
        T->s = sc; S->s = sc; S->done = 0;
    }
}
// err = M(b) - x*
__global__ void __launch_bounds__(LB) train_err_kernel(long long N, Dims3 fd, Dims3 cd, const float* b, const float* invD, const uint8_t* st,
                                                       const float* w1, const float* xs, float* err) {
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float zv;
        if (is_inactive(st, c)) zv = 0.f;
        else {
            zv = __ldg(invD + c) * b[c];
            if (w1 && is_active(st, c)) zv += prolong_at(fd, cd, w1, c);
        }
        err[c] = zv - xs[c];
    }
}
// 7-point product restricted to the active cells (values elsewhere taken as zero): the
// symmetric block of the p' matrix whose energy norm the training loss uses
__device__ __forceinline__ float apply_active(const OpSymF32& A, const uint8_t* st, long long N, long long c, const float* x) {
    auto xv = [&](long long e_) { return (e_ >= 0 && e_ < N && st[e_] == ST_ACTIVE) ? x[e_] : 0.f; };
    return __ldg(A.aP + c) * xv(c) + __ldg(A.aE + c) * xv(c + 1) + __ldg(A.aE + c - 1) * xv(c - 1) + __ldg(A.aN + c) * xv(c + A.nI)
           + __ldg(A.aN + c - A.nI) * xv(c - A.nI) + __ldg(A.aT + c) * xv(c + A.nIJ) + __ldg(A.aT + c - A.nIJ) * xv(c - A.nIJ);
}
// g = -(A err), h = -(A x*): partial err.g and x*.h (energy norms of the error and of x*);
// with immersed-boundary cells, on the active block only
__global__ void __launch_bounds__(LB) train_energy_kernel(OpSymF32 A, long long N, const uint8_t* st, const float* err, const float* xs, float* g,
                                                          double* part) {
    double v[2] = {0., 0.};
    for (long long c = blockIdx.x * (long long)LB + threadIdx.x; c < N; c += (long long)gridDim.x * LB) {
        float ge, hx;
        if (st == nullptr) {
            ge = -applyF(A, c, [&](long long e_) { return err[e_]; });
            hx = -applyF(A, c, [&](long long e_) { return xs[e_]; });
        } else if (st[c] == ST_ACTIVE) {
            ge = -apply_active(A, st, N, c, err);
            hx = -apply_active(A, st, N, c, xs);
        } else {
            ge = 0.f; hx = 0.f;
        }
        g[c] = ge;
        v[0] += (double)err[c] * ge;
        v[1] += (double)xs[c] * hx;
    }
    block_sums(v, 2, part);
}
__global__ void train_energy_finish(const double* part, int nblk, TrainScal* T, float* lossOut) {
    double t[2];
    totals(part, nblk, 2, t);
    if (threadIdx.x == 0) {
        double den = t[1] > 0. ? t[1] : 1.;
        T->coef = 2. / den;
        T->loss = t[0] / den;
        T->loss_sum += t[0] / den;
        if (lossOut) *lossOut = (float)(t[0] / den);
    }
}
// dL/dz on the cells where z carries the prolonged term
__global__ void train_dz_kernel(long long N, const float* g, const uint8_t* st, const TrainScal* T, float inv_batch, float* dz) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    dz[c] = is_active(st, c) ? (float)T->coef * g[c] * inv_batch : 0.f;
}
__global__ void adam_kernel(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, int t) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float gq = g[q];
    float mq = b1 * m[q] + (1.f - b1) * gq;
    float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq; v[q] = vq;
    float mh = mq / (1.f - powf(b1, (float)t)), vh = vq / (1.f - powf(b2, (float)t));
    p[q] = p[q] - lr * mh / (sqrtf(vh) + eps);
}
__global__ void loss_out_kernel(TrainScal* T, float* hist, int step, float inv_batch) {
    if (threadIdx.x == 0) { hist[step] = (float)(T->loss_sum * inv_batch); T->loss_sum = 0.; }
}

// one application M(b) for pair (b, x*): error in lw.z, energy loss, g = -(A err) in lw.e
int pair_forward(LearnedWork& lw, const OpSymF32& Af, const uint8_t* status, const Lat& L, const float* b, const float* xs, int mode,
                 TrainScal* T, float* lossOut, cudaStream_t st) {
    const long long N = L.N;
    const int nb = nblocks(N);
    Scal* S = static_cast<Scal*>(lw.scal);
    train_scale_kernel<<<nb, LB, 0, st>>>(N, b, lw.invD, status, lw.part);
    train_scale_finish<<<1, LB, 0, st>>>(lw.part, nb, T, S);
    if (apply_levels(lw, b, status, mode, S, st)) return 1;
    train_err_kernel<<<nb, LB, 0, st>>>(N, dims_of(lw.lev[0]), level1_dims(lw), b, lw.invD, status, level_w1(lw, mode), xs, lw.z);
    train_energy_kernel<<<nb, LB, 0, st>>>(Af, N, status, lw.z, xs, lw.e, lw.part);
    train_energy_finish<<<1, LB, 0, st>>>(lw.part, nb, T, lossOut);
    CB_CHECK_LAUNCH();
    return 0;
}

int check_net_error(LearnedWork& lw) {
    if (!lw.weights) return 0;
    int herr = 0;
    CB_CUDA(cudaMemcpy(&herr, lw.weights->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) { set_error("tensor-core convolution: an MMA completion wait timed out"); return 1; }
    return 0;
}

}  // namespace

int learned_eval(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, const float* pairsB, const float* pairsX, int nPairs,
                 int mode, float* lossHost, cudaStream_t st) {
    if (mode == NET_MODE_NETWORK && (!lw.haveParams || lw.nLev < 2)) { set_error("no network parameters on this handle"); return 1; }
    if (mode != NET_MODE_JACOBI && !lw.masksReady && level_masks(lw, status, st)) return 1;
    OpSymF32 Af = cast_operator(lw, A, L, st);
    TrainScal* T = nullptr;
    float* dl = nullptr;
    CB_CUDA(cudaMallocAsync(&T, sizeof(TrainScal), st));
    CB_CUDA(cudaMallocAsync(&dl, sizeof(float) * (nPairs > 0 ? nPairs : 1), st));
    CB_CUDA(cudaMemsetAsync(T, 0, sizeof(TrainScal), st));
    int rc = 0;
    for (int q = 0; q < nPairs && !rc; ++q)
        rc = pair_forward(lw, Af, status, L, pairsB + (size_t)q * L.PS + L.H, pairsX + (size_t)q * L.PS + L.H, mode, T, dl + q, st);
    if (!rc && nPairs > 0 && lossHost) rc = cudaMemcpyAsync(lossHost, dl, sizeof(float) * nPairs, cudaMemcpyDeviceToHost, st) != cudaSuccess;
    cudaStreamSynchronize(st);
    cudaFreeAsync(T, st); cudaFreeAsync(dl, st);
    CB_CUDA(cudaStreamSynchronize(st));
    if (rc) { set_error("evaluation failed"); return 1; }
    return check_net_error(lw);
}

int learned_train(LearnedWork& lw, const OpSym& A, const uint8_t* status, const Lat& L, const float* pairsB, const float* pairsX,
                  int nPairs, int steps, int batch, float lr, unsigned seed, float* lossHost, cudaStream_t st) {
    if (lw.nLev < 2 || !lw.weights) { set_error("lattice too small for the level pyramid of the learned preconditioner"); return 1; }
    const long long N = L.N;
    const int G = grid_for(N, 256);
    if (!lw.masksReady && level_masks(lw, status, st)) return 1;
    OpSymF32 Af = cast_operator(lw, A, L, st);
    NetBuffers& W = *lw.weights;
    TrainScal* T = nullptr;
    float *mom = nullptr, *vel = nullptr, *hist = nullptr;
    CB_CUDA(cudaMallocAsync(&T, sizeof(TrainScal), st));
    CB_CUDA(cudaMallocAsync(&mom, sizeof(float) * NET_PARAMS, st));
    CB_CUDA(cudaMallocAsync(&vel, sizeof(float) * NET_PARAMS, st));
    CB_CUDA(cudaMallocAsync(&hist, sizeof(float) * (steps > 0 ? steps : 1), st));
    CB_CUDA(cudaMemsetAsync(T, 0, sizeof(TrainScal), st));
    CB_CUDA(cudaMemsetAsync(mom, 0, sizeof(float) * NET_PARAMS, st));
    CB_CUDA(cudaMemsetAsync(vel, 0, sizeof(float) * NET_PARAMS, st));
    unsigned long long rs = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto next = [&]() { rs = rs * 6364136223846793005ull + 1442695040888963407ull; return (unsigned)(rs >> 33); };
    const float inv_batch = 1.f / (float)batch;
    const Scal* S = static_cast<const Scal*>(lw.scal);
    for (int step = 0; step < steps; ++step) {
        CB_CUDA(cudaMemsetAsync(W.grad, 0, sizeof(float) * NET_PARAMS, st));
        if (net_pack_weights(W, st)) return 1;
        for (int q = 0; q < batch; ++q) {
            int idx = (int)(next() % (unsigned)nPairs);
            const float* b = pairsB + (size_t)idx * L.PS + L.H;
            const float* xs = pairsX + (size_t)idx * L.PS + L.H;
            if (pair_forward(lw, Af, status, L, b, xs, NET_MODE_NETWORK, T, nullptr, st)) return 1;
            train_dz_kernel<<<G, 256, 0, st>>>(N, lw.e, status, T, inv_batch, lw.r);
            // adjoint chain: dL/dw_l = P_l^T dL/dw_(l-1) (into u_l), dL/dy_l = gain_l s dL/dw_l (into w_l)
            for (int l = 1; l < lw.nLev; ++l) {
                Level& c = lw.lev[l];
                const Level& f = lw.lev[l - 1];
                restrict_kernel<<<restrict_grid(dims_of(c)), 256, 0, st>>>(dims_of(f), dims_of(c), l == 1 ? lw.r : f.u, nullptr, nullptr, 1.f,
                                                                           c.u, c.w, c.gain, nullptr, nullptr, nullptr, 0.f, S);
                if (l >= lw.netFrom && l <= lw.netTo) {
                    // y = (net(x) - net(-x)) / 2: the two evaluations get dL/dy / 2 and -dL/dy / 2
                    half_split_kernel<<<grid_for(c.N, 256), 256, 0, st>>>(c.N, c.w, c.w2);
                    if (net_backward(c.net, c.w, st) || net_backward(c.netNeg, c.w2, st)) return 1;
                }
            }
        }
        loss_out_kernel<<<1, 32, 0, st>>>(T, hist, step, inv_batch);
        adam_kernel<<<grid_for(NET_PARAMS, 256), 256, 0, st>>>(NET_PARAMS, W.params, W.grad, mom, vel, lr, 0.9f, 0.999f, 1e-8f, step + 1);
        CB_CHECK_LAUNCH();
    }
    if (net_pack_weights(W, st)) return 1;
    if (lossHost && steps > 0) CB_CUDA(cudaMemcpyAsync(lossHost, hist, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
    cudaFreeAsync(T, st); cudaFreeAsync(mom, st); cudaFreeAsync(vel, st); cudaFreeAsync(hist, st);
    CB_CUDA(cudaStreamSynchronize(st));
    if (check_net_error(lw)) return 1;
    lw.haveParams = true;
    return 0;
}

}  // namespace cb
