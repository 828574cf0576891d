// Krylov solvers as persistent cooperative kernels.
//
// The reference calls PETSc (KSPBCGS + PCSOR, src/Math/SparseMatrix.cpp:86-106) once
// per system, from a zero initial guess, and returns the iteration count.  PETSc's
// lexicographic SOR sweep is sequential, so the device solvers use Jacobi
// preconditioning (the plain FP64 device path) with the published algorithms:
//   * BiCGStab (van der Vorst 1992), right-preconditioned, for the momentum system
//     (three right-hand sides sharing one operator sweep) and for non-symmetric
//     pressure-correction systems (immersed-boundary ghost rows);
//   * CG (Hestenes-Stiefel; Chronopoulos-Gear single-reduction form), for the symmetric
//     pressure-correction system.
// Every solve is one kernel launch: all blocks stay resident (cooperative launch) and
// meet at grid barriers between the phases of an iteration; the dot products are summed
// per block and then, in every block, over the block partials in a fixed order, so all
// blocks take the same convergence decision and the result is bit-reproducible.  The
// loop ends on the true residual ||b - A x|| <= rtol ||b|| (checked when the recursive
// residual meets it; the iteration restarts from the true residual otherwise) or at
// maxit, so no launch can run unbounded.
//
// Values written earlier in the same launch by other blocks are read with ordinary loads
// after the grid barrier (whose device-scope fence orders them), never through the
// read-only (non-coherent) path; only never-written inputs use __ldg.  Vectors that can be formed
// from others are not stored: CG's search direction p = z + beta p_old and BiCGStab's
// p = r + beta (p_old - omega v) and s = r - alpha v are recomputed at the stencil
// neighbours instead of costing an extra pass and barrier.
#include <cooperative_groups.h>
#include <cstring>
#include "krylov.cuh"
#include "stencil.cuh"

#define CAFFE_KSP_CG_JACOBI_INT 2   // caffe_ksp value of Jacobi-CG (include/caffe_b200.h)

namespace cg = cooperative_groups;

namespace cb {

constexpr int KB = 256;   // threads per block
constexpr int KP = 8;     // partial slots per block

__device__ __forceinline__ double ldcg(const double* p) { return *p; }   // coherent load after a grid barrier

template <int K>
__device__ __forceinline__ void warp_sum(double (&v)[K]) {
#pragma unroll
    for (int q = 0; q < K; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
}

// block sums of v[0..K) into partials[blockIdx.x*KP + q]
template <int K>
__device__ void block_partials(double (&v)[K], double* partials) {
    __shared__ double sm[KP][32];
    warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) sm[q][w] = v[q];
    __syncthreads();
    if (w == 0) {
        double t[K];
#pragma unroll
        for (int q = 0; q < K; ++q) t[q] = lane < nw ? sm[q][lane] : 0.;
        warp_sum(t);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < K; ++q) partials[blockIdx.x * KP + q] = t[q];
    }
    __syncthreads();
}

// sum of all blocks' partials, computed identically in every block
template <int K>
__device__ void grid_totals(const double* partials, double (&out)[K]) {
    __shared__ double sm[KP][32];
    double v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = 0.;
    for (int g = threadIdx.x; g < (int)gridDim.x; g += blockDim.x)
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] += ldcg(partials + (long long)g * KP + q);
    warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) sm[q][w] = v[q];
    __syncthreads();
    if (w == 0) {
        double t[K];
#pragma unroll
        for (int q = 0; q < K; ++q) t[q] = lane < nw ? sm[q][lane] : 0.;
        warp_sum(t);
        __syncwarp();
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < K; ++q) sm[q][0] = t[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = sm[q][0];
    __syncthreads();
}

// Block partials, grid barrier, totals.  Partials alternate between two buffers: a block
// that races ahead to the next reduction cannot overwrite a slot another block is still
// summing, because it must first pass the barrier of the reduction in between.
template <int K>
__device__ __forceinline__ void grid_reduce(cg::grid_group& grid, double (&v)[K], double* partials, int& parity, double (&out)[K]) {
    double* buf = partials + (long long)(parity & 1) * gridDim.x * KP;
    block_partials<K>(v, buf);
    grid.sync();
    grid_totals<K>(buf, out);
    ++parity;
}


template <class Op>
__global__ void inv_diag_kernel(Op A, long long N, double* invD) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    double dg = diag_of(A, c);
    invD[c] = dg != 0. ? 1. / dg : 1.;
}

struct KArgs {
    const double* b;
    double* x;
    double* r;
    double* rp;
    double* p[2];
    double* v[2];
    double* t;
    const double* invD;
    double* partials;
    KspOut* out;
    long long N, PS;
    double rtol;
    double atol;   // absolute floor: converged when ||b - A x|| <= max(rtol ||b||, atol)
    int maxit;
    int project;   // remove the mean of b first (singular all-Neumann pressure systems)
    // fallback mode: when skip_if_ok is set the launch returns at once unless the status
    // it points to (the previous solve's) is non-zero; fallbacks counts the launches that ran
    const int* skip_if_ok;
    int* fallbacks;
};

// Remove the mean of b (one plane), in place; every block computes the same mean.
__device__ __forceinline__ void project_mean(cg::grid_group& grid, double* b, long long N, long long t0, long long T,
                                             double* partials, int& par) {
    double s[1] = {0.};
    for (long long c = t0; c < N; c += T) s[0] += b[c];
    double tot[1];
    grid_reduce<1>(grid, s, partials, par, tot);
    double mean = tot[0] / (double)N;
    for (long long c = t0; c < N; c += T) b[c] = b[c] - mean;
    // the projected b is read at stencil neighbours owned by other blocks right after this
    // (CG forms w = A D^-1 b): every block's subtraction must be visible first
    grid.sync();
}

// ------------------------------------------------------------------ BiCGStab
template <int NR, class Op>
__global__ void __launch_bounds__(KB) bicgstab_kernel(Op A, KArgs a) {
    if (a.skip_if_ok && *a.skip_if_ok == 0) return;   // uniform across the grid: no barrier is reached
    if (a.skip_if_ok && blockIdx.x == 0 && threadIdx.x == 0 && a.fallbacks) atomicAdd(a.fallbacks, 1);
    cg::grid_group grid = cg::this_grid();
    const long long N = a.N, PS = a.PS;
    const long long T = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const double* invD = a.invD;

    double acc[2 * NR];
    int par = 0;
    if (NR == 1 && a.project) project_mean(grid, const_cast<double*>(a.b), N, t0, T, a.partials, par);
    // ---- initial state: x = 0, r = rp = b
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = 0.;
    for (long long c = t0; c < N; c += T) {
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            double bv = a.b[q * PS + c];
            a.x[q * PS + c] = 0.;
            a.r[q * PS + c] = bv;
            a.rp[q * PS + c] = bv;
            acc[q] += bv * bv;
        }
    }
    double bb[NR];
    {
        double tmp[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) tmp[q] = acc[q];
        grid_reduce<NR>(grid, tmp, a.partials, par, bb);
    }

    double rho[NR], rho_old[NR], alpha[NR], omega[NR], tol2[NR];
    int it[NR], status[NR];
    bool done[NR], fresh[NR], needT[NR];
    double relres[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
        rho[q] = bb[q]; rho_old[q] = 1.; alpha[q] = 1.; omega[q] = 1.;
        tol2[q] = fmax(a.rtol * a.rtol * bb[q], a.atol * a.atol);
        it[q] = 0; fresh[q] = true; needT[q] = false; relres[q] = 0.;
        // x = 0 already meets the absolute floor: nothing to do (relative residual 1)
        done[q] = !(bb[q] > 0.) || bb[q] <= tol2[q];
        if (bb[q] > 0. && done[q]) relres[q] = 1.;
        if (bb[q] != bb[q]) status[q] = 3; else status[q] = 0;
    }
    int cur = 0;
    while (true) {
        bool run[NR], any = false;
#pragma unroll
        for (int q = 0; q < NR; ++q) { run[q] = !done[q]; any |= run[q]; }
        if (!any) break;
        double beta[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) beta[q] = fresh[q] ? 0. : (rho[q] / rho_old[q]) * (alpha[q] / omega[q]);
        const double* po = a.p[cur];
        const double* vo = a.v[cur];
        double* pn = a.p[cur ^ 1];
        double* vn = a.v[cur ^ 1];
        // ---- phase 1: p = r + beta (p_old - omega v_old);  v = A D^-1 p;  (rp, v)
#pragma unroll
        for (int q = 0; q < NR; ++q) acc[q] = 0.;
        for (long long c = t0; c < N; c += T) {
            auto pnew = [&](int q, long long e) -> double {
                double rv = ldcg(a.r + q * PS + e);
                if (fresh[q]) return rv;
                return rv + beta[q] * (ldcg(po + q * PS + e) - omega[q] * ldcg(vo + q * PS + e));
            };
            double y[NR];
            apply<NR>(A, c, [&](int q, long long e) { return __ldg(invD + e) * pnew(q, e); }, y);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!run[q]) continue;
                double pc = pnew(q, c);
                pn[q * PS + c] = pc;
                vn[q * PS + c] = y[q];
                double rpv;
                if (fresh[q]) { rpv = ldcg(a.r + q * PS + c); a.rp[q * PS + c] = rpv; }
                else rpv = a.rp[q * PS + c];
                acc[q] += rpv * y[q];
            }
        }
        double rv[NR];
        {
            double tmp[NR];
#pragma unroll
            for (int q = 0; q < NR; ++q) tmp[q] = acc[q];
            grid_reduce<NR>(grid, tmp, a.partials, par, rv);
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            if (!run[q]) continue;
            if (rv[q] == 0. || rv[q] != rv[q]) { needT[q] = true; run[q] = false; }
            else alpha[q] = rho[q] / rv[q];
        }
        // ---- phase 2: s = r - alpha v;  t = A D^-1 s;  (t, s), (t, t)
#pragma unroll
        for (int q = 0; q < 2 * NR; ++q) acc[q] = 0.;
        for (long long c = t0; c < N; c += T) {
            double y[NR];
            apply<NR>(A, c, [&](int q, long long e) {
                return __ldg(invD + e) * (ldcg(a.r + q * PS + e) - alpha[q] * ldcg(vn + q * PS + e));
            }, y);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!run[q]) continue;
                double s = ldcg(a.r + q * PS + c) - alpha[q] * ldcg(vn + q * PS + c);
                a.t[q * PS + c] = y[q];
                acc[2 * q] += y[q] * s;
                acc[2 * q + 1] += y[q] * y[q];
            }
        }
        double tot[2 * NR];
        {
            double tmp[2 * NR];
#pragma unroll
            for (int q = 0; q < 2 * NR; ++q) tmp[q] = acc[q];
            grid_reduce<2 * NR>(grid, tmp, a.partials, par, tot);
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            if (!run[q]) continue;
            omega[q] = tot[2 * q + 1] == 0. ? 0. : tot[2 * q] / tot[2 * q + 1];
        }
        // ---- phase 3: x += alpha D^-1 p + omega D^-1 s;  r = s - omega t;  (r, rp), (r, r)
#pragma unroll
        for (int q = 0; q < 2 * NR; ++q) acc[q] = 0.;
        for (long long c = t0; c < N; c += T) {
            double id = __ldg(invD + c);
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!run[q]) continue;
                double s = ldcg(a.r + q * PS + c) - alpha[q] * ldcg(vn + q * PS + c);
                double ph = id * ldcg(pn + q * PS + c);
                double sh = id * s;
                a.x[q * PS + c] = a.x[q * PS + c] + (alpha[q] * ph + omega[q] * sh);
                double rn = s - omega[q] * ldcg(a.t + q * PS + c);
                a.r[q * PS + c] = rn;
                acc[2 * q] += rn * a.rp[q * PS + c];
                acc[2 * q + 1] += rn * rn;
            }
        }
        {
            double tmp[2 * NR];
#pragma unroll
            for (int q = 0; q < 2 * NR; ++q) tmp[q] = acc[q];
            grid_reduce<2 * NR>(grid, tmp, a.partials, par, tot);
        }
        bool anyT = false;
#pragma unroll
        for (int q = 0; q < NR; ++q) {
            if (run[q]) {
                it[q] += 1;
                fresh[q] = false;
                rho_old[q] = rho[q];
                rho[q] = tot[2 * q];
                double rr = tot[2 * q + 1];
                if (rr <= tol2[q] || omega[q] == 0. || it[q] >= a.maxit || rr != rr) needT[q] = true;
            }
            anyT |= needT[q];
        }
        cur ^= 1;
        if (anyT) {
            // ---- true residual r = b - A x for the components being checked
#pragma unroll
            for (int q = 0; q < NR; ++q) acc[q] = 0.;
            for (long long c = t0; c < N; c += T) {
                double y[NR];
                apply<NR>(A, c, [&](int q, long long e) { return ldcg(a.x + q * PS + e); }, y);
#pragma unroll
                for (int q = 0; q < NR; ++q) {
                    if (!needT[q]) continue;
                    double rt = a.b[q * PS + c] - y[q];
                    a.r[q * PS + c] = rt;
                    acc[q] += rt * rt;
                }
            }
            double rrT[NR];
            {
                double tmp[NR];
#pragma unroll
                for (int q = 0; q < NR; ++q) tmp[q] = acc[q];
                grid_reduce<NR>(grid, tmp, a.partials, par, rrT);
            }
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                if (!needT[q]) continue;
                needT[q] = false;
                relres[q] = sqrt(rrT[q] / bb[q]);
                if (rrT[q] <= tol2[q]) { done[q] = true; status[q] = 0; }
                else if (rrT[q] != rrT[q]) { done[q] = true; status[q] = 3; }
                else if (it[q] >= a.maxit) { done[q] = true; status[q] = 1; }
                else { fresh[q] = true; rho[q] = rrT[q]; rho_old[q] = 1.; alpha[q] = 1.; omega[q] = 1.; }
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int q = 0; q < NR; ++q) { a.out->iters[q] = it[q]; a.out->relres[q] = relres[q]; a.out->status[q] = status[q]; }
    }
}

// ------------------------------------------------------------------ CG, one reduction per iteration
// Chronopoulos & Gear (1989) form of preconditioned CG: with u = M^-1 r and w = A u the two
// inner products (r, u) and (w, u) are taken together, so an iteration is one sweep and one
// grid barrier:
//   s_i = w_i + beta_i s_{i-1};  p_i = u_i + beta_i p_{i-1};  x += alpha_i p_i;
//   r_{i+1} = r_i - alpha_i s_i;  u_{i+1} = M^-1 r_{i+1};  w_{i+1} = A u_{i+1};
//   gamma = (r_{i+1}, u_{i+1}), delta = (w_{i+1}, u_{i+1});
//   beta_{i+1} = gamma_{i+1} / gamma_i;  alpha_{i+1} = gamma_{i+1} / (delta - beta_{i+1} gamma_{i+1} / alpha_i).
// u_{i+1} at the stencil neighbours is recomputed from r_i, w_i and s_{i-1}, which are
// double-buffered (the sweep writes the other buffer).
template <class Op>
__global__ void __launch_bounds__(KB, 4) cg1_kernel(Op A, KArgs a) {
    if (a.skip_if_ok && *a.skip_if_ok == 0) return;   // uniform across the grid: no barrier is reached
    if (a.skip_if_ok && blockIdx.x == 0 && threadIdx.x == 0 && a.fallbacks) atomicAdd(a.fallbacks, 1);
    cg::grid_group grid = cg::this_grid();
    const long long N = a.N, PS = a.PS;
    const long long T = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const double* invD = a.invD;
    // current (read) and next (written) buffers, swapped after every sweep
    double *rC = a.r, *rN = a.r + PS, *wC = a.v[0], *wN = a.v[1], *sC = a.p[0], *sN = a.p[1];
    double* p = a.t;       // u = M^-1 r is not stored: it is recomputed from r where needed
    int par = 0;
    if (a.project) project_mean(grid, const_cast<double*>(a.b), N, t0, T, a.partials, par);
    // ---- start: x = 0, r = b, u = M^-1 b, w = A u, s_-1 = p_-1 = 0
    double acc[3] = {0., 0., 0.};
    for (long long c = t0; c < N; c += T) {
        double bv = a.b[c];
        double uv = __ldg(invD + c) * bv;
        double y[1];
        apply<1>(A, c, [&](int, long long e) { return __ldg(invD + e) * a.b[e]; }, y);
        a.x[c] = 0.;
        rC[c] = bv; wC[c] = y[0]; sC[c] = 0.; p[c] = 0.;
        acc[0] += bv * uv; acc[1] += y[0] * uv; acc[2] += bv * bv;
    }
    double tot[3];
    grid_reduce<3>(grid, acc, a.partials, par, tot);
    double gamma = tot[0], bb = tot[2];
    double tol2 = fmax(a.rtol * a.rtol * bb, a.atol * a.atol);
    double alpha = tot[1] != 0. ? gamma / tot[1] : 0., beta = 0.;
    int it = 0, status = 0;
    double relres = 0.;
    bool done = !(bb > 0.) || bb <= tol2;   // x = 0 already meets the absolute floor
    if (bb > 0. && done) relres = 1.;
    if (bb != bb) status = 3;
    while (!done) {
        const double* r0 = rC;
        const double* w0 = wC;
        const double* s0 = sC;
        double* r1 = rN;
        double* w1 = wN;
        double* s1 = sN;
        acc[0] = acc[1] = acc[2] = 0.;
        for (long long c = t0; c < N; c += T) {
            double idc = __ldg(invD + c);
            double r0c = r0[c];
            double si = w0[c] + beta * s0[c];
            double pi = idc * r0c + beta * p[c];
            a.x[c] = a.x[c] + alpha * pi;
            double rn = r0c - alpha * si;
            double un = idc * rn;
            double y[1];
            apply<1>(A, c, [&](int, long long e) {
                return __ldg(invD + e) * (r0[e] - alpha * (w0[e] + beta * s0[e]));
            }, y);
            s1[c] = si; p[c] = pi; r1[c] = rn; w1[c] = y[0];
            acc[0] += rn * un; acc[1] += y[0] * un; acc[2] += rn * rn;
        }
        grid_reduce<3>(grid, acc, a.partials, par, tot);
        it += 1;
        { double* t_ = rC; rC = rN; rN = t_; t_ = wC; wC = wN; wN = t_; t_ = sC; sC = sN; sN = t_; }
        double gn = tot[0], dn = tot[1], rr = tot[2];
        bool check = rr <= tol2 || it >= a.maxit || rr != rr;
        double bn = gn / gamma;
        double den = dn - bn * gn / alpha;
        if (den == 0. || den != den || gamma == 0.) check = true;
        beta = bn; alpha = gn / den; gamma = gn;
        if (check) {
            // ---- true residual r = b - A x (into the current buffer)
            double* rc = rC;
            double a2[1] = {0.};
            for (long long c = t0; c < N; c += T) {
                double y[1];
                apply<1>(A, c, [&](int, long long e) { return a.x[e]; }, y);
                double rt = a.b[c] - y[0];
                rc[c] = rt;
                a2[0] += rt * rt;
            }
            double t1[1];
            grid_reduce<1>(grid, a2, a.partials, par, t1);
            relres = sqrt(t1[0] / bb);
            if (t1[0] <= tol2) { done = true; status = 0; }
            else if (t1[0] != t1[0]) { done = true; status = 3; }
            else if (it >= a.maxit) { done = true; status = 1; }
            else {
                // restart from the true residual: u = M^-1 r, w = A u, s = p = 0
                double a3[2] = {0., 0.};
                double* wc = wC;
                double* sc = sC;
                for (long long c = t0; c < N; c += T) {
                    double uv = __ldg(invD + c) * rc[c];
                    double y[1];
                    apply<1>(A, c, [&](int, long long e) { return __ldg(invD + e) * rc[e]; }, y);
                    wc[c] = y[0]; sc[c] = 0.; p[c] = 0.;
                    a3[0] += rc[c] * uv; a3[1] += y[0] * uv;
                }
                double t2[2];
                grid_reduce<2>(grid, a3, a.partials, par, t2);
                gamma = t2[0];
                alpha = t2[1] != 0. ? gamma / t2[1] : 0.;
                beta = 0.;
                if (gamma == 0.) { done = true; status = 2; }
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { a.out->iters[0] = it; a.out->relres[0] = relres; a.out->status[0] = status; }
}

// ------------------------------------------------------------------ mixed precision
// FP64 iterative refinement around FP32 inner solves (the precision form of the pressure
// correction): the true residual r = b - A x, the update x += e, and every dot product and
// norm stay FP64; the matrix copy, the Jacobi preconditioner, the inner Krylov vectors and
// the inner operator sweeps are FP32.  One launch runs the whole solve:
//   repeat: r = b - A x (FP64, reduced) -> stop at ||r|| <= rtol ||b||;
//           A32 e = float(r) by FP32 CG or BiCGStab to inner_rtol (relative);  x += e.
struct OpSymF {
    const float* aP;
    const float* aE;
    const float* aN;
    const float* aT;
    long long nI, nIJ;
    GhostRows gh;
};

template <class X>
__device__ __forceinline__ float applyf(const OpSymF& A, long long c, X&& x) {
    float aP = __ldg(A.aP + c), aE = __ldg(A.aE + c), aW = __ldg(A.aE + c - 1), aN = __ldg(A.aN + c);
    float aS = __ldg(A.aN + c - A.nI), aT = __ldg(A.aT + c), aB = __ldg(A.aT + c - A.nIJ);
    float y = aP * x(c) + aE * x(c + 1) + aW * x(c - 1) + aN * x(c + A.nI) + aS * x(c - A.nI) + aT * x(c + A.nIJ)
              + aB * x(c - A.nIJ);
    if (A.gh.n > 0) {
        uint32_t wbits = __ldg(A.gh.bits + (c >> 5));
        if ((wbits >> (c & 31)) & 1u) {
            int g = ghost_index(A.gh, c);
            float sum = 0.f;
            for (int m = 0; m < 9; ++m) {
                int col = __ldg(A.gh.col + 9 * g + m);
                if (col >= 0) sum += (float)__ldg(A.gh.val + 9 * g + m) * x((long long)col);
            }
            y = sum;
        }
    }
    return y;
}

__global__ void cast_sym_kernel(OpSym A, long long N, float* aP, float* aE, float* aN, float* aT, float* invD) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    double d = A.aP[c];
    aP[c] = (float)d; aE[c] = (float)A.aE[c]; aN[c] = (float)A.aN[c]; aT[c] = (float)A.aT[c];
    invD[c] = d != 0. ? (float)(1. / d) : 1.f;
}

struct MxArgs {
    const double* b;
    double* x;
    float* r[2];
    float* w[2];
    float* s[2];
    float* p;
    float* e;
    float* v[2];
    float* t;
    const float* invD;
    double* partials;
    KspOut* out;
    long long N;
    double rtol;
    double atol;
    int maxit;
    double eta;
    int project;
    int inner_max;
};

template <class Op64, int INNER_BICG>
__global__ void __launch_bounds__(KB, 4) mixed_kernel(Op64 A, OpSymF Af, MxArgs a) {
    cg::grid_group grid = cg::this_grid();
    const long long N = a.N;
    const long long T = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const float* invD = a.invD;
    int par = 0;
    if (a.project) project_mean(grid, const_cast<double*>(a.b), N, t0, T, a.partials, par);
    double acc1[1] = {0.};
    for (long long c = t0; c < N; c += T) {
        double bv = a.b[c];
        a.x[c] = 0.;
        acc1[0] += bv * bv;
    }
    double tot1[1];
    grid_reduce<1>(grid, acc1, a.partials, par, tot1);
    double bb = tot1[0], tol2 = fmax(a.rtol * a.rtol * bb, a.atol * a.atol);
    int status = 0, inner_total = 0, outer = 0;
    double relres = 0.;
    bool done = !(bb > 0.);
    if (bb != bb) { status = 3; done = true; }
    float* rC = a.r[0];
    float* rN = a.r[1];
    while (!done) {
        // ---- FP64 true residual, handed to the inner solver in FP32
        acc1[0] = 0.;
        for (long long c = t0; c < N; c += T) {
            double y[1];
            apply<1>(A, c, [&](int, long long e_) { return a.x[e_]; }, y);
            double rt = a.b[c] - y[0];
            rC[c] = (float)rt;
            acc1[0] += rt * rt;
        }
        grid_reduce<1>(grid, acc1, a.partials, par, tot1);
        double rr = tot1[0];
        relres = sqrt(rr / bb);
        if (rr <= tol2) { status = 0; break; }
        if (rr != rr) { status = 3; break; }
        if (inner_total >= a.maxit) { status = 1; break; }
        ++outer;
        // inner target: as deep as FP32 allows on the first pass, then only the factor still
        // missing to the outer tolerance (with a safety margin)
        double eta = 0.25 * sqrt(tol2 / rr);
        if (eta < a.eta) eta = a.eta;
        if (eta > 0.5) eta = 0.5;
        // ---- FP32 inner solve A32 e = r (e from zero), dots and norms in FP64
        int inner = 0;
        if (!INNER_BICG) {
            // Chronopoulos-Gear CG, as cg1_kernel, in FP32 storage
            float* wC = a.w[0]; float* wN = a.w[1]; float* sC = a.s[0]; float* sN = a.s[1];
            double acc[3] = {0., 0., 0.};
            for (long long c = t0; c < N; c += T) {
                float r0 = rC[c];
                float u0 = __ldg(invD + c) * r0;
                float y = applyf(Af, c, [&](long long e_) { return __ldg(invD + e_) * rC[e_]; });
                a.e[c] = 0.f; wC[c] = y; sC[c] = 0.f; a.p[c] = 0.f;
                acc[0] += (double)r0 * u0; acc[1] += (double)y * u0; acc[2] += (double)r0 * r0;
            }
            double tot[3];
            grid_reduce<3>(grid, acc, a.partials, par, tot);
            double gamma = tot[0], rr0 = tot[2];
            double alpha = tot[1] != 0. ? gamma / tot[1] : 0., beta = 0.;
            double tin2 = eta * eta * rr0;
            bool stop = !(gamma != 0.);
            while (!stop) {
                float al = (float)alpha, be = (float)beta;
                acc[0] = acc[1] = acc[2] = 0.;
                for (long long c = t0; c < N; c += T) {
                    float idc = __ldg(invD + c);
                    float r0 = rC[c];
                    float si = wC[c] + be * sC[c];
                    float pi = idc * r0 + be * a.p[c];
                    a.e[c] = a.e[c] + al * pi;
                    float rn = r0 - al * si;
                    float un = idc * rn;
                    float y = applyf(Af, c, [&](long long e_) { return __ldg(invD + e_) * (rC[e_] - al * (wC[e_] + be * sC[e_])); });
                    sN[c] = si; a.p[c] = pi; rN[c] = rn; wN[c] = y;
                    acc[0] += (double)rn * un; acc[1] += (double)y * un; acc[2] += (double)rn * rn;
                }
                grid_reduce<3>(grid, acc, a.partials, par, tot);
                ++inner;
                { float* t_ = rC; rC = rN; rN = t_; t_ = wC; wC = wN; wN = t_; t_ = sC; sC = sN; sN = t_; }
                double gn = tot[0], dn = tot[1], rri = tot[2];
                double bn = gn / gamma;
                double den = dn - bn * gn / alpha;
                if (rri <= tin2 || inner >= a.inner_max || inner_total + inner >= a.maxit || den == 0. || den != den || gn == 0.) stop = true;
                beta = bn; alpha = gn / den; gamma = gn;
            }
        } else {
            // BiCGStab, right-preconditioned with Jacobi, in FP32 storage
            float* rp = a.s[0];
            float* pO = a.p;  float* pNn = a.s[1];
            float* vO = a.v[0]; float* vNn = a.v[1];
            double acc[1] = {0.};
            for (long long c = t0; c < N; c += T) {
                float r0 = rC[c];
                a.e[c] = 0.f; rp[c] = r0; pO[c] = 0.f; vO[c] = 0.f;
                acc[0] += (double)r0 * r0;
            }
            double tot[1];
            grid_reduce<1>(grid, acc, a.partials, par, tot);
            double rr0 = tot[0], tin2 = eta * eta * rr0;
            double rho = rr0, rho_old = 1., alpha = 1., omega = 1.;
            bool fresh = true, stop = !(rr0 > 0.);
            float* rcur = rC;
            while (!stop) {
                double beta = fresh ? 0. : (rho / rho_old) * (alpha / omega);
                float be = (float)beta, om = (float)omega;
                double a1[1] = {0.};
                for (long long c = t0; c < N; c += T) {
                    auto pn_at = [&](long long e_) -> float {
                        float rv = rcur[e_];
                        return fresh ? rv : rv + be * (pO[e_] - om * vO[e_]);
                    };
                    float y = applyf(Af, c, [&](long long e_) { return __ldg(invD + e_) * pn_at(e_); });
                    pNn[c] = pn_at(c); vNn[c] = y;
                    a1[0] += (double)rp[c] * y;
                }
                double t1[1];
                grid_reduce<1>(grid, a1, a.partials, par, t1);
                if (t1[0] == 0. || t1[0] != t1[0]) break;
                alpha = rho / t1[0];
                float al = (float)alpha;
                double a2[2] = {0., 0.};
                for (long long c = t0; c < N; c += T) {
                    float y = applyf(Af, c, [&](long long e_) { return __ldg(invD + e_) * (rcur[e_] - al * vNn[e_]); });
                    float sv = rcur[c] - al * vNn[c];
                    a.t[c] = y;
                    a2[0] += (double)y * sv; a2[1] += (double)y * y;
                }
                double t2[2];
                grid_reduce<2>(grid, a2, a.partials, par, t2);
                omega = t2[1] == 0. ? 0. : t2[0] / t2[1];
                om = (float)omega;
                double a3[2] = {0., 0.};
                for (long long c = t0; c < N; c += T) {
                    float idc = __ldg(invD + c);
                    float sv = rcur[c] - al * vNn[c];
                    a.e[c] = a.e[c] + (al * (idc * pNn[c]) + om * (idc * sv));
                    float rn = sv - om * a.t[c];
                    rcur[c] = rn;
                    a3[0] += (double)rn * rp[c]; a3[1] += (double)rn * rn;
                }
                double t3[2];
                grid_reduce<2>(grid, a3, a.partials, par, t3);
                ++inner;
                fresh = false;
                rho_old = rho; rho = t3[0];
                { float* t_ = pO; pO = pNn; pNn = t_; t_ = vO; vO = vNn; vNn = t_; }
                if (t3[1] <= tin2 || omega == 0. || inner >= a.inner_max || inner_total + inner >= a.maxit || t3[1] != t3[1]) stop = true;
            }
            rC = rcur;
        }
        inner_total += inner;
        // ---- x += e (FP64); the next residual reads x at the neighbours
        for (long long c = t0; c < N; c += T) a.x[c] = a.x[c] + (double)a.e[c];
        grid.sync();
        if (outer > 60) { status = 1; break; }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out->iters[0] = inner_total; a.out->iters[1] = outer; a.out->relres[0] = relres; a.out->status[0] = status;
    }
}

// ------------------------------------------------------------------ host side
static int g_numSM = 0;

static int sm_count() {
    if (g_numSM == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_numSM, cudaDevAttrMultiProcessorCount, dev);
    }
    return g_numSM;
}

template <class K>
static int coop_grid(K kernel) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, KB, 0) != cudaSuccess || nb < 1) nb = 1;
    if (nb > 4) nb = 4;
    return nb * sm_count();
}

template <class K>
static int launch_coop(K kernel, int grid, KArgs& args, const void* op, cudaStream_t st) {
    void* params[2] = {const_cast<void*>(op), &args};
    CB_CUDA(cudaLaunchCooperativeKernel((const void*)kernel, dim3(grid), dim3(KB), params, 0, st));
    return 0;
}

static KArgs make_args(const Lat& L, const KspWork& w, const double* b, double* x, double rtol, int maxit, double atol) {
    KArgs a;
    a.b = b; a.x = x; a.r = w.r; a.rp = w.rp;
    a.p[0] = w.p[0]; a.p[1] = w.p[1]; a.v[0] = w.v[0]; a.v[1] = w.v[1];
    a.t = w.t; a.invD = w.invD; a.partials = w.partials; a.out = w.out;
    a.N = L.N; a.PS = L.PS; a.rtol = rtol; a.atol = atol; a.maxit = maxit;
    a.project = 0;
    a.skip_if_ok = nullptr;
    a.fallbacks = nullptr;
    return a;
}

int ksp_bicgstab(const Op7& A, int nr, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                 cudaStream_t st, double atol) {
    inv_diag_kernel<Op7><<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.invD);
    CB_CHECK_LAUNCH();
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    if (nr == 3) {
        static int G = 0;
        if (!G) G = coop_grid(bicgstab_kernel<3, Op7>);
        return launch_coop(bicgstab_kernel<3, Op7>, G, a, &A, st);
    }
    static int G1 = 0;
    if (!G1) G1 = coop_grid(bicgstab_kernel<1, Op7>);
    return launch_coop(bicgstab_kernel<1, Op7>, G1, a, &A, st);
}

int ksp_bicgstab_sym(const OpSym& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                     cudaStream_t st, int project, double atol) {
    inv_diag_kernel<OpSym><<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.invD);
    CB_CHECK_LAUNCH();
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    a.project = project;
    static int G = 0;
    if (!G) G = coop_grid(bicgstab_kernel<1, OpSym>);
    return launch_coop(bicgstab_kernel<1, OpSym>, G, a, &A, st);
}

int ksp_cg(const OpSym& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit, cudaStream_t st,
           int project, double atol) {
    inv_diag_kernel<OpSym><<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.invD);
    CB_CHECK_LAUNCH();
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    a.project = project;
    static int G = 0;
    if (!G) G = coop_grid(cg1_kernel<OpSym>);
    return launch_coop(cg1_kernel<OpSym>, G, a, &A, st);
}

int ksp_cg7(const Op7& A, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit, cudaStream_t st,
            double atol) {
    inv_diag_kernel<Op7><<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.invD);
    CB_CHECK_LAUNCH();
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    static int G = 0;
    if (!G) G = coop_grid(cg1_kernel<Op7>);
    return launch_coop(cg1_kernel<Op7>, G, a, &A, st);
}

int ksp_csr(const OpCSR& A, int method, long long n, const double* b, double* x, const KspWork& w, double rtol, int maxit,
            cudaStream_t st, double atol) {
    inv_diag_kernel<OpCSR><<<grid_for(n, 256), 256, 0, st>>>(A, n, w.invD);
    CB_CHECK_LAUNCH();
    Lat L;
    std::memset(&L, 0, sizeof(L));
    L.nI = (int)n; L.nJ = 1; L.nK = 1; L.N = n; L.nIJ = n; L.H = 0; L.PS = n;   // unpadded vectors
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    if (method == CAFFE_KSP_CG_JACOBI_INT) {
        static int G = 0;
        if (!G) G = coop_grid(cg1_kernel<OpCSR>);
        return launch_coop(cg1_kernel<OpCSR>, G, a, &A, st);
    }
    static int G = 0;
    if (!G) G = coop_grid(bicgstab_kernel<1, OpCSR>);
    return launch_coop(bicgstab_kernel<1, OpCSR>, G, a, &A, st);
}

int krylov_grid_size(int which) {
    switch (which) {
        case 0: return coop_grid(bicgstab_kernel<3, Op7>);
        case 1: return coop_grid(bicgstab_kernel<1, OpSym>);
        case 2: return coop_grid(cg1_kernel<OpSym>);
        case 4: return coop_grid(cg1_kernel<Op7>);
        case 5: return coop_grid(bicgstab_kernel<1, OpCSR>);
        case 6: return coop_grid(cg1_kernel<OpCSR>);
        default: return coop_grid(bicgstab_kernel<1, Op7>);
    }
}


int ksp_mixed_sym(const OpSym& A, int method, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                  double inner_rtol, cudaStream_t st, int project, double atol) {
    cast_sym_kernel<<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.fA[0], w.fA[1], w.fA[2], w.fA[3], w.finvD);
    CB_CHECK_LAUNCH();
    OpSymF Af;
    Af.aP = w.fA[0]; Af.aE = w.fA[1]; Af.aN = w.fA[2]; Af.aT = w.fA[3];
    Af.nI = A.nI; Af.nIJ = A.nIJ; Af.gh = A.gh;
    MxArgs m;
    m.b = b; m.x = x;
    m.r[0] = w.fr[0]; m.r[1] = w.fr[1]; m.w[0] = w.fw[0]; m.w[1] = w.fw[1]; m.s[0] = w.fs[0]; m.s[1] = w.fs[1];
    m.p = w.fp; m.e = w.fe; m.v[0] = w.fv[0]; m.v[1] = w.fv[1]; m.t = w.ft; m.invD = w.finvD;
    m.partials = w.partials; m.out = w.out; m.N = L.N; m.rtol = rtol; m.atol = atol; m.maxit = maxit; m.eta = inner_rtol;
    m.project = project; m.inner_max = 100000;
    void* params[3] = {const_cast<OpSym*>(&A), &Af, &m};
    if (method == CAFFE_KSP_CG_JACOBI_INT) {
        static int G = 0;
        if (!G) { int nb = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mixed_kernel<OpSym, 0>, KB, 0); G = (nb < 1 ? 1 : (nb > 4 ? 4 : nb)) * sm_count(); }
        CB_CUDA(cudaLaunchCooperativeKernel((const void*)mixed_kernel<OpSym, 0>, dim3(G), dim3(KB), params, 0, st));
    } else {
        static int G = 0;
        if (!G) { int nb = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mixed_kernel<OpSym, 1>, KB, 0); G = (nb < 1 ? 1 : (nb > 4 ? 4 : nb)) * sm_count(); }
        CB_CUDA(cudaLaunchCooperativeKernel((const void*)mixed_kernel<OpSym, 1>, dim3(G), dim3(KB), params, 0, st));
    }
    return 0;
}

int ksp_fallback_sym(const OpSym& A, int method, const double* b, double* x, const Lat& L, const KspWork& w, double rtol, int maxit,
                     cudaStream_t st, int project, const int* status, int* fallbacks, double atol) {
    // plain FP64 re-solve from zero, executed only when *status (the previous solve's) is non-zero
    inv_diag_kernel<OpSym><<<grid_for(L.N, 256), 256, 0, st>>>(A, L.N, w.invD);
    CB_CHECK_LAUNCH();
    KArgs a = make_args(L, w, b, x, rtol, maxit, atol);
    a.project = project;
    a.skip_if_ok = status;
    a.fallbacks = fallbacks;
    if (method == CAFFE_KSP_CG_JACOBI_INT) {
        static int G = 0;
        if (!G) G = coop_grid(cg1_kernel<OpSym>);
        return launch_coop(cg1_kernel<OpSym>, G, a, &A, st);
    }
    static int G = 0;
    if (!G) G = coop_grid(bicgstab_kernel<1, OpSym>);
    return launch_coop(bicgstab_kernel<1, OpSym>, G, a, &A, st);
}

}  // namespace cb
