// Phases of a distributed Krylov solve on one slab of a k-slab decomposition (slab.cuh).
//
// Each phase is one grid-stride sweep over the slab's owned cells; a phase that reduces
// writes per-block partial sums and a one-block launch adds them in block order, so a
// slab's sums do not depend on scheduling.  The sweeps are bandwidth-bound like the
// persistent solvers' (the same bytes per cell per iteration, plus the D^-1 p and D^-1 s
// vectors that are stored here because their halo planes are exchanged).
#include "slab.cuh"
#include "stencil.cuh"

namespace cb {

namespace {

constexpr int SB = 256;   // threads per block
constexpr int SP = 8;     // partial slots per block

template <int K>
__device__ void slab_block_partials(double (&v)[K], double* part) {
    __shared__ double sm[SP][SB / 32];
#pragma unroll
    for (int q = 0; q < K; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) sm[q][w] = v[q];
    __syncthreads();
    if (threadIdx.x < K) {
        double t = 0.;
        for (int i = 0; i < SB / 32; ++i) t += sm[threadIdx.x][i];
        part[(long long)blockIdx.x * SP + threadIdx.x] = t;
    }
}

// red[q] = sum over blocks (in block order) of part[g*SP + q]
__global__ void slab_finish_kernel(const double* part, int nblocks, int K, double* red) {
    __shared__ double sm[SB];
    for (int q = 0; q < K; ++q) {
        double t = 0.;
        for (int g = threadIdx.x; g < nblocks; g += SB) t += part[(long long)g * SP + q];
        sm[threadIdx.x] = t;
        __syncthreads();
        for (int s = SB / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) red[q] = sm[0];
        __syncthreads();
    }
}

template <int NR, class Op, int PH>
__global__ void __launch_bounds__(SB) slab_kernel(Op A, SlabKsp k, SlabScal s) {
    constexpr int K = PH == SB_INIT || PH == SB_V || PH == SB_TRUE ? NR
                    : PH == SB_T || PH == SB_X                    ? 2 * NR
                    : PH == SC_W                                   ? 3
                    : PH == SC_TRUE || PH == SS_SUM_B || PH == SS_SUM_X ? 1
                                                                   : 0;
    const long long PS = k.L.PS;
    const long long T = (long long)gridDim.x * blockDim.x;
    long long lo = k.o0, hi = k.o1;
    if constexpr (PH == SS_SUB_X) {   // the halo planes too, so they need no exchange afterwards
        lo = lo - k.L.nIJ > 0 ? lo - k.L.nIJ : 0;
        hi = hi + k.L.nIJ < k.L.N ? hi + k.L.nIJ : k.L.N;
    }
    double acc[K > 0 ? K : 1];
#pragma unroll
    for (int q = 0; q < (K > 0 ? K : 1); ++q) acc[q] = 0.;
    const double* invD = k.w.invD;
    for (long long c = lo + blockIdx.x * (long long)blockDim.x + threadIdx.x; c < hi; c += T) {
        if constexpr (PH == SB_INIT || PH == SC_INIT) {
            double dg = diag_of(A, c);
            double id = dg != 0. ? 1. / dg : 1.;
            k.w.invD[c] = id;
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                double bv = k.b[q * PS + c];
                k.x[q * PS + c] = 0.;
                k.w.r[q * PS + c] = bv;
                if constexpr (PH == SB_INIT) {
                    k.w.rp[q * PS + c] = bv;
                    acc[q] += bv * bv;
                } else {
                    k.ph[c] = id * bv;
                    k.w.p[0][c] = 0.;
                    k.w.t[c] = 0.;
                }
            }
        } else if constexpr (PH == SB_P) {
            double id = invD[c];
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!(s.flags[q] & SF_RUN)) continue;
                double rv = k.w.r[q * PS + c];
                double pv;
                if (s.flags[q] & SF_FRESH) { pv = rv; k.w.rp[q * PS + c] = rv; }
                else pv = rv + s.beta[q] * (k.w.p[0][q * PS + c] - s.omega[q] * k.w.v[0][q * PS + c]);
                k.w.p[0][q * PS + c] = pv;
                k.ph[q * PS + c] = id * pv;
            }
        } else if constexpr (PH == SB_V) {
            double y[NR];
            apply<NR>(A, c, [&](int q, long long e) { return k.ph[q * PS + e]; }, y);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!(s.flags[q] & SF_RUN)) continue;
                k.w.v[0][q * PS + c] = y[q];
                acc[q] += k.w.rp[q * PS + c] * y[q];
            }
        } else if constexpr (PH == SB_S) {
            double id = invD[c];
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!(s.flags[q] & SF_RUN)) continue;
                k.sh[q * PS + c] = id * (k.w.r[q * PS + c] - s.alpha[q] * k.w.v[0][q * PS + c]);
            }
        } else if constexpr (PH == SB_T) {
            double y[NR];
            apply<NR>(A, c, [&](int q, long long e) { return k.sh[q * PS + e]; }, y);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!(s.flags[q] & SF_RUN)) continue;
                double sv = k.w.r[q * PS + c] - s.alpha[q] * k.w.v[0][q * PS + c];
                k.w.t[q * PS + c] = y[q];
                acc[2 * q] += y[q] * sv;
                acc[2 * q + 1] += y[q] * y[q];
            }
        } else if constexpr (PH == SB_X) {
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!(s.flags[q] & SF_RUN)) continue;
                double sv = k.w.r[q * PS + c] - s.alpha[q] * k.w.v[0][q * PS + c];
                k.x[q * PS + c] = k.x[q * PS + c] + (s.alpha[q] * k.ph[q * PS + c] + s.omega[q] * k.sh[q * PS + c]);
                double rn = sv - s.omega[q] * k.w.t[q * PS + c];
                k.w.r[q * PS + c] = rn;
                acc[2 * q] += rn * k.w.rp[q * PS + c];
                acc[2 * q + 1] += rn * rn;
            }
        } else if constexpr (PH == SB_TRUE || PH == SC_TRUE) {
            double y[NR];
            apply<NR>(A, c, [&](int q, long long e) { return k.x[q * PS + e]; }, y);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (PH == SB_TRUE && !(s.flags[q] & SF_TRUE)) continue;
                double rt = k.b[q * PS + c] - y[q];
                k.w.r[q * PS + c] = rt;
                acc[q] += rt * rt;
            }
        } else if constexpr (PH == SC_W) {
            double y[1];
            apply<1>(A, c, [&](int, long long e) { return k.ph[e]; }, y);
            double uv = k.ph[c];
            double rv = k.w.r[c];
            k.w.v[0][c] = y[0];
            acc[0] += rv * uv;
            acc[1] += y[0] * uv;
            acc[2] += rv * rv;
        } else if constexpr (PH == SC_UPD) {
            double si = k.w.v[0][c] + s.beta[0] * k.w.p[0][c];
            double pi = k.ph[c] + s.beta[0] * k.w.t[c];
            k.x[c] = k.x[c] + s.alpha[0] * pi;
            double rn = k.w.r[c] - s.alpha[0] * si;
            k.w.p[0][c] = si;
            k.w.t[c] = pi;
            k.w.r[c] = rn;
            k.ph[c] = invD[c] * rn;
        } else if constexpr (PH == SC_RESTART) {
            k.ph[c] = invD[c] * k.w.r[c];
            k.w.p[0][c] = 0.;
            k.w.t[c] = 0.;
        } else if constexpr (PH == SS_SUM_B) {
            acc[0] += k.b[c];
        } else if constexpr (PH == SS_SUB_B) {
            k.b[c] = k.b[c] - s.alpha[0];
        } else if constexpr (PH == SS_SUM_X) {
            acc[0] += k.x[c];
        } else if constexpr (PH == SS_SUB_X) {
            k.x[c] = k.x[c] - s.alpha[0];
        }
    }
    if constexpr (K > 0) slab_block_partials<K>(acc, k.part);
}

template <int NR, class Op, int PH>
int run_phase(const Op& A, const SlabKsp& k, const SlabScal& s, cudaStream_t st, int smCount) {
    constexpr int K = PH == SB_INIT || PH == SB_V || PH == SB_TRUE ? NR
                    : PH == SB_T || PH == SB_X                    ? 2 * NR
                    : PH == SC_W                                   ? 3
                    : PH == SC_TRUE || PH == SS_SUM_B || PH == SS_SUM_X ? 1
                                                                   : 0;
    long long n = k.o1 - k.o0 + 2 * k.L.nIJ;
    long long want = (n + SB - 1) / SB;
    int cap = 8 * smCount < SLAB_MAX_BLOCKS ? 8 * smCount : SLAB_MAX_BLOCKS;
    int G = (int)(want < cap ? want : cap);
    if (G < 1) G = 1;
    slab_kernel<NR, Op, PH><<<G, SB, 0, st>>>(A, k, s);
    CB_CHECK_LAUNCH();
    if constexpr (K > 0) {
        slab_finish_kernel<<<1, SB, 0, st>>>(k.part, G, K, k.red);
        CB_CHECK_LAUNCH();
    }
    return K;
}

int sm_count_cached() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
    }
    return n;
}

template <int NR, class Op>
int dispatch(const Op& A, int phase, const SlabKsp& k, const SlabScal& s, cudaStream_t st) {
    if (k.o0 < 0 || k.o1 > k.L.N || k.o0 >= k.o1) { set_error("slab: empty or out-of-range owned cells"); return -1; }
    const int sm = sm_count_cached();
    switch (phase) {
        case SB_INIT: return run_phase<NR, Op, SB_INIT>(A, k, s, st, sm);
        case SB_P: return run_phase<NR, Op, SB_P>(A, k, s, st, sm);
        case SB_V: return run_phase<NR, Op, SB_V>(A, k, s, st, sm);
        case SB_S: return run_phase<NR, Op, SB_S>(A, k, s, st, sm);
        case SB_T: return run_phase<NR, Op, SB_T>(A, k, s, st, sm);
        case SB_X: return run_phase<NR, Op, SB_X>(A, k, s, st, sm);
        case SB_TRUE: return run_phase<NR, Op, SB_TRUE>(A, k, s, st, sm);
        default: break;
    }
    if (NR == 1) {
        switch (phase) {
            case SC_INIT: return run_phase<1, Op, SC_INIT>(A, k, s, st, sm);
            case SC_W: return run_phase<1, Op, SC_W>(A, k, s, st, sm);
            case SC_UPD: return run_phase<1, Op, SC_UPD>(A, k, s, st, sm);
            case SC_TRUE: return run_phase<1, Op, SC_TRUE>(A, k, s, st, sm);
            case SC_RESTART: return run_phase<1, Op, SC_RESTART>(A, k, s, st, sm);
            case SS_SUM_B: return run_phase<1, Op, SS_SUM_B>(A, k, s, st, sm);
            case SS_SUB_B: return run_phase<1, Op, SS_SUB_B>(A, k, s, st, sm);
            case SS_SUM_X: return run_phase<1, Op, SS_SUM_X>(A, k, s, st, sm);
            case SS_SUB_X: return run_phase<1, Op, SS_SUB_X>(A, k, s, st, sm);
            default: break;
        }
    }
    set_error("slab: unknown Krylov phase " + std::to_string(phase) + " for " + std::to_string(NR) + " right-hand side(s)");
    return -1;
}

}  // namespace

int slab_ksp_phase(const Op7& A, int nr, int phase, const SlabKsp& k, const SlabScal& s, cudaStream_t st) {
    if (nr == 3) return dispatch<3>(A, phase, k, s, st);
    if (nr == 1) return dispatch<1>(A, phase, k, s, st);
    set_error("slab: 1 or 3 right-hand sides");
    return -1;
}

int slab_ksp_phase(const OpSym& A, int nr, int phase, const SlabKsp& k, const SlabScal& s, cudaStream_t st) {
    if (nr == 1) return dispatch<1>(A, phase, k, s, st);
    set_error("slab: the pressure-correction operator takes one right-hand side");
    return -1;
}

}  // namespace cb
