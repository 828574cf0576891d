// C ABI of the device library (include/caffe_b200.h): the handle owns the mesh metrics,
// the solver fields, both linear systems and the Krylov workspace in HBM, and one stream.
// One time step of Simple / Piso / IbPiso is a fixed sequence of kernel launches on that
// stream with no host synchronisation inside it.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "flow.cuh"
#include "krylov.cuh"
#include "ib.cuh"
#include "cnn.cuh"
#include "learned.cuh"
#include "slab.cuh"

namespace cb {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
void clear_error() { g_err.clear(); }
std::string cuda_msg(cudaError_t e, const char* what, const char* file, int line) {
    return std::string(what) + " failed: " + cudaGetErrorString(e) + " (" + file + ":" + std::to_string(line) + ")";
}

// Per-step accumulation of solver statistics on the device (read back once per step).
struct StepAcc {
    int mom_iters[3];
    int p_iters_last;
    int p_iters_total;
    int p_solves;
    int status;
    int fallbacks;
    int cascades;
    int net_iters;
    double p_res_max;
    double mom_res_max;
    double continuity;
    unsigned long long courant_bits;
};

// one training pair (b, x) of a p' solve, rounded to FP32
__global__ void pair_cast_kernel(long long N, const double* b, const double* x, float* pb, float* px) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) { pb[c] = (float)b[c]; px[c] = (float)x[c]; }
}

// zero-mean gauge of a singular p' solution: block partial sums, mean, subtraction
__global__ void __launch_bounds__(256) gauge_partial_kernel(const double* x, long long N, double* part) {
    __shared__ double sm[256];
    double s = 0.;
    for (long long c = blockIdx.x * 256ll + threadIdx.x; c < N; c += (long long)gridDim.x * 256) s += x[c];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}
__global__ void __launch_bounds__(256) gauge_mean_kernel(double* part, int nblk, long long N) {
    __shared__ double sm[256];
    double s = 0.;
    for (int b = threadIdx.x; b < nblk; b += 256) s += part[b];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[nblk] = sm[0] / (double)N;
}
__global__ void gauge_apply_kernel(double* x, long long N, const double* mean) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < N) x[c] = x[c] - *mean;
}

__global__ void acc_kernel(const KspOut* o, StepAcc* acc, int kind, int nr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int q = 0; q < nr; ++q) {
        int s = o->status[q];
        if (s > acc->status) acc->status = s;
        double rr = o->relres[q];
        if (kind == 0) {
            acc->mom_iters[q] = o->iters[q];
            if (rr > acc->mom_res_max) acc->mom_res_max = rr;
        } else {
            if (kind == 2) { acc->cascades += o->cascades; acc->net_iters += o->net_iters; }
            acc->p_iters_last = o->iters[q];
            acc->p_iters_total += o->iters[q];
            acc->p_solves += 1;
            if (rr > acc->p_res_max) acc->p_res_max = rr;
        }
    }
}

__global__ void copy_planes_kernel(const double* src, double* dst, long long N, long long PS, int planes) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    for (int q = 0; q < planes; ++q) dst[c + q * PS] = src[c + q * PS];
}

__global__ void fill_planes_kernel(double* dst, long long N, long long PS, double v0, double v1, double v2, int planes) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    dst[c] = v0;
    if (planes > 1) dst[c + PS] = v1;
    if (planes > 2) dst[c + 2 * PS] = v2;
}

}  // namespace cb

using namespace cb;

struct caffe_dev {
    int device = 0;
    cudaStream_t st = nullptr;
    Lat L;
    caffe_case cs;
    Bc bc;
    FlowParams P;
    bool ib = false;
    // raw allocations
    std::vector<void*> allocs;
    // metrics
    double* vol = nullptr;
    double* cc = nullptr;
    double* S[3] = {};
    double* fc[3] = {};
    double* D[3] = {};
    double* cv[3] = {};
    // fields
    double* u = nullptr;
    double* u0buf = nullptr;
    double* gradP = nullptr;
    double* gradPC = nullptr;
    double* gradU = nullptr;
    double* p = nullptr;
    double* pc = nullptr;
    double* d = nullptr;
    double* mfc = nullptr;
    double* F[3] = {};
    double* Fb[3] = {};
    double* pPatch[6] = {};
    long long patchN[6] = {};
    uint8_t* status = nullptr;
    // systems
    double* ma[7] = {};
    double* mb = nullptr;
    double* paP = nullptr;
    double* paE = nullptr;
    double* paN = nullptr;
    double* paT = nullptr;
    double* pb = nullptr;
    KspWork kw;
    IbState ibs;
    // learned preconditioner of the p' solve
    LearnedWork lw;
    bool haveLearned = false;
    int netMode = NET_MODE_NETWORK;
    // training pairs (b, x) of p' solves, FP32 halo-padded planes
    float* pairB = nullptr;
    float* pairX = nullptr;
    int pairCap = 0, pairCount = 0;
    int pairSnapshots = 0;       // intermediate-iterate pairs per recorded solve
    double* snapX = nullptr;     // iterate of a truncated re-solve (one FP64 cell plane)
    double* gaugePart = nullptr; // partial sums of the zero-mean gauge (1024 + 1 doubles)
    bool recording = false;
    // reductions and statistics
    double* chunkMax = nullptr;
    StepAcc* acc = nullptr;
    StepAcc* accHost = nullptr;   // pinned
    caffe_step_stats last;
    cudaEvent_t ev[6] = {};
    bool stepTimed = false;
    // event pairs around every linear solve of a step (device time of each solve)
    std::vector<cudaEvent_t> evP, evM;
    int nPTimed = 0, nMTimed = 0;
    // k-slab decomposition: the owned cells [o0, o1) and the vectors of the distributed
    // Krylov phases (set by caffe_slab_set_owned)
    bool slab = false;
    long long o0 = 0, o1 = 0;
    double* slabPh = nullptr;
    double* slabSh = nullptr;
    double* slabPart = nullptr;
    bool ownStream = true;   // false once the caller has handed in its own stream

    template <class T>
    T* dalloc(size_t count) {
        void* ptr = nullptr;
        if (cudaMalloc(&ptr, count * sizeof(T) + 256) != cudaSuccess) return nullptr;
        cudaMemsetAsync(ptr, 0, count * sizeof(T) + 256, st);
        allocs.push_back(ptr);
        return static_cast<T*>(ptr);
    }
    // halo-padded cell array of `planes` planes; returns the pointer to element 0 of plane 0
    double* cell(int planes) {
        double* b = dalloc<double>((size_t)L.PS * planes);
        return b ? b + L.H : nullptr;
    }
    static void* alloc_cb(size_t bytes, void* ctx) { return static_cast<caffe_dev*>(ctx)->dalloc<char>(bytes); }
    int ensure_learned() {
        if (haveLearned) return 0;
        if (learned_alloc(lw, L, &caffe_dev::alloc_cb, this)) return 1;
        haveLearned = true;
        return 0;
    }
    int ensure_pairs(int cap) {
        if (cap <= pairCap) return 0;
        size_t plane = (size_t)L.PS;
        float *nb = nullptr, *nx = nullptr;
        if (cudaMalloc(&nb, sizeof(float) * plane * cap) != cudaSuccess || cudaMalloc(&nx, sizeof(float) * plane * cap) != cudaSuccess) {
            cudaFree(nb); cudaFree(nx);
            set_error("training-pair allocation failed");
            return 1;
        }
        cudaMemsetAsync(nb, 0, sizeof(float) * plane * cap, st);
        cudaMemsetAsync(nx, 0, sizeof(float) * plane * cap, st);
        if (pairCount > 0) {
            cudaMemcpyAsync(nb, pairB, sizeof(float) * plane * pairCount, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(nx, pairX, sizeof(float) * plane * pairCount, cudaMemcpyDeviceToDevice, st);
        }
        cudaStreamSynchronize(st);
        cudaFree(pairB); cudaFree(pairX);
        pairB = nb; pairX = nx; pairCap = cap;
        return 0;
    }
    float* fcell() {
        float* b = dalloc<float>((size_t)L.PS);
        return b ? b + L.H : nullptr;
    }
    FlowFields fields(bool forCorrect = false) {
        FlowFields f;
        f.u = u;
        f.u0 = u0buf ? u0buf : u;
        f.gradP = gradP; f.gradPC = gradPC; f.gradU = gradU;
        f.p = p; f.pc = pc; f.d = d; f.mfc = mfc;
        for (int q = 0; q < 3; ++q) { f.F[q] = F[q]; f.Fout[q] = Fb[q]; }
        for (int q = 0; q < 6; ++q) f.pPatch[q] = pPatch[q];
        f.status = ib ? status : nullptr;
        f.nonorth = cs.nonorth;
        (void)forCorrect;
        return f;
    }
    Geo geo() const {
        Geo g;
        g.L = L; g.vol = vol; g.cc = cc;
        for (int q = 0; q < 3; ++q) { g.S[q] = S[q]; g.fc[q] = fc[q]; g.D[q] = D[q]; g.cv[q] = cv[q]; }
        return g;
    }
    GhostRows ghosts(int which) const {
        GhostRows gh;
        gh.n = ib ? ibs.nGhost : 0;
        gh.cell = ibs.gCell;
        gh.col = ibs.gCol;
        gh.val = which == 0 ? ibs.gValMom : ibs.gValP;
        gh.bits = ibs.bits;
        return gh;
    }
    Op7 momOp() const {
        Op7 A;
        for (int q = 0; q < 7; ++q) A.a[q] = ma[q];
        A.nI = L.nI; A.nIJ = L.nIJ;
        A.gh = ghosts(0);
        return A;
    }
    OpSym pOp() const {
        OpSym A;
        A.aP = paP; A.aE = paE; A.aN = paN; A.aT = paT;
        A.nI = L.nI; A.nIJ = L.nIJ;
        A.gh = ghosts(1);
        return A;
    }
    ~caffe_dev() {
        if (st) cudaStreamSynchronize(st);
        for (void* a : allocs) cudaFree(a);
        for (auto& e : ev) if (e) cudaEventDestroy(e);
        for (auto& e : evP) if (e) cudaEventDestroy(e);
        for (auto& e : evM) if (e) cudaEventDestroy(e);
        learned_free_host(lw);
        cudaFree(pairB); cudaFree(pairX);
        if (accHost) cudaFreeHost(accHost);
        if (st && ownStream) cudaStreamDestroy(st);
    }
};

namespace {

int setup_bcs(caffe_dev* h) {
    const caffe_case& c = h->cs;
    for (int f = 0; f < 6; ++f) {
        int t = c.bc_type[f];
        h->bc.flow[f] = t;
        switch (t) {  // FlowBoundaryConditions.cpp:44-71
            case CAFFE_INLET: case CAFFE_WALL: h->bc.uType[f] = P_FIXED; h->bc.pType[f] = P_ZERO_GRADIENT; break;
            case CAFFE_OUTLET: h->bc.uType[f] = P_ZERO_GRADIENT; h->bc.pType[f] = P_FIXED; break;
            case CAFFE_EMPTY: h->bc.uType[f] = P_EMPTY; h->bc.pType[f] = P_EMPTY; break;
            case CAFFE_ZERO_GRADIENT: h->bc.uType[f] = P_ZERO_GRADIENT; h->bc.pType[f] = P_ZERO_GRADIENT; break;
            default: set_error("invalid boundary type " + std::to_string(t) + " on face " + std::to_string(f)); return 1;
        }
        for (int q = 0; q < 3; ++q) h->bc.uRef[f][q] = c.ref_vec[f][q];
        h->bc.pRef[f] = c.ref_val[f];
    }
    return 0;
}

// The reference preconditions with PETSc's lexicographic symmetric SOR sweep
// (src/Math/SparseMatrix.cpp:95-100), which is sequential row by row; the device does not
// substitute another preconditioner for it silently.
const char* const SGS_UNAVAILABLE =
    "BiCGStab with symmetric Gauss-Seidel (the reference's PETSc PCSOR) is a sequential sweep and is not "
    "implemented on the device: choose CAFFE_KSP_BICGSTAB_JACOBI or CAFFE_KSP_CG_JACOBI";

int validate_case(const caffe_case* c) {
    if (!c) { set_error("case is NULL"); return 1; }
    if (c->kind < 0 || c->kind > 2) { set_error("invalid solver kind"); return 1; }
    if (c->omega_u <= 0. || c->omega_p <= 0.) { set_error("relaxation factors must be positive"); return 1; }
    if (c->n_inner < 1 && c->time_accurate) { set_error("numberOfInnerIterations must be >= 1"); return 1; }
    if (c->n_pcorr < 1 && c->kind != CAFFE_SIMPLE) { set_error("numberOfPressureCorrections must be >= 1"); return 1; }
    if (c->convection < 0 || c->convection > 1) { set_error("invalid convection scheme"); return 1; }
    if (c->mom_method == CAFFE_KSP_CG_JACOBI) { set_error("the momentum matrix is not symmetric: CG cannot solve it"); return 1; }
    if (c->mom_method == CAFFE_KSP_BICGSTAB_SGS || c->p_method == CAFFE_KSP_BICGSTAB_SGS) {
        set_error(SGS_UNAVAILABLE);
        return 1;
    }
    if (c->mom_method < 0 || c->mom_method > CAFFE_KSP_CG_JACOBI || c->p_method < 0 || c->p_method > CAFFE_KSP_CG_JACOBI) {
        set_error("invalid Krylov method");
        return 1;
    }
    if (!(c->mom_atol >= 0.) || !(c->p_atol >= 0.)) { set_error("absolute tolerances must be >= 0"); return 1; }
    if (c->maxit < 1) { set_error("maxit must be >= 1"); return 1; }
    if (c->kind == CAFFE_IBPISO && !(c->ib_radius > 0.)) { set_error("IbPiso needs a sphere radius > 0"); return 1; }
    if (c->p_form < 0 || c->p_form > 3) { set_error("invalid pressure-solve form"); return 1; }
    return 0;
}

// Initial boundary patches of p: PrimitiveBoundaryCondition::changeType on a FIXED face
// copies every face's current reference value into every patch (PrimitiveBoundaryCondition.tpp:
// 257-294); faces configured later keep the zero of a fresh field until refreshed.
int init_p_patches(caffe_dev* h) {
    double refs[6] = {0, 0, 0, 0, 0, 0}, patch[6] = {0, 0, 0, 0, 0, 0};
    for (int f = 0; f < 6; ++f) {
        refs[f] = h->cs.ref_val[f];
        if (h->bc.pType[f] == P_FIXED)
            for (int m = 0; m < 6; ++m) patch[m] = refs[m];
    }
    for (int f = 0; f < 6; ++f) {
        std::vector<double> v((size_t)h->patchN[f], patch[f]);
        CB_CUDA(cudaMemcpyAsync(h->pPatch[f], v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
        CB_CUDA(cudaStreamSynchronize(h->st));
    }
    return 0;
}

int fill(caffe_dev* h, double* dst, int planes, double a, double b = 0., double c = 0.) {
    fill_planes_kernel<<<grid_for(h->L.N, 256), 256, 0, h->st>>>(dst, h->L.N, h->L.PS, a, b, c, planes);
    CB_CHECK_LAUNCH();
    return 0;
}

// With no fixed-pressure face and no immersed boundary the p' matrix is singular (the
// constant vector is its null space) and its right-hand side carries a round-off
// component along it that no Krylov method can remove; the solver then projects the
// right-hand side onto the range first (the CPU oracle does the same).
// deepest relative residual reduction an FP32 inner solve of the mixed-precision form aims for
// (later inner solves only aim for the factor still missing)
constexpr double MIXED_INNER_RTOL = 1e-6;
constexpr double LEARNED_INNER_RTOL = 1e-5;

int p_singular(const caffe_dev* h) {
    if (h->ib) return 0;
    for (int f = 0; f < 6; ++f) if (h->bc.pType[f] == P_FIXED) return 0;
    return 1;
}

// ------------------------------------------------------------------ phases
int ph_save_u0(caffe_dev* h) {
    if (!h->u0buf) return 0;
    copy_planes_kernel<<<grid_for(h->L.N, 256), 256, 0, h->st>>>(h->u, h->u0buf, h->L.N, h->L.PS, 3);
    CB_CHECK_LAUNCH();
    return 0;
}
int ph_assemble_momentum(caffe_dev* h, double dt) {
    MomSys m;
    for (int q = 0; q < 7; ++q) m.a[q] = h->ma[q];
    m.b = h->mb;
    return launch_momentum_assemble(h->geo(), h->bc, h->fields(), m, h->P, dt, h->st);
}
int ph_solve_momentum(caffe_dev* h) {
    if (ksp_bicgstab(h->momOp(), 3, h->mb, h->u, h->L, h->kw, h->cs.mom_rtol, h->cs.maxit, h->st, h->cs.mom_atol)) return 1;
    acc_kernel<<<1, 32, 0, h->st>>>(h->kw.out, h->acc, 0, 3);
    CB_CHECK_LAUNCH();
    return 0;
}
int ph_momentum_post(caffe_dev* h) { return launch_rhie_chow(h->geo(), h->bc, h->fields(), h->P, h->st); }
int ph_assemble_pcorr(caffe_dev* h) {
    PcSys s;
    s.aP = h->paP; s.aE = h->paE; s.aN = h->paN; s.aT = h->paT; s.b = h->pb;
    return launch_pcorr_assemble(h->geo(), h->bc, h->fields(), s, h->P, h->st);
}
int ph_solve_pcorr(caffe_dev* h) {
    int rc;
    OpSym A = h->pOp();
    bool sym = !(h->ib && h->ibs.nGhost > 0);
    int method = h->cs.p_method;
    if (method == CAFFE_KSP_CG_JACOBI && !sym) method = CAFFE_KSP_BICGSTAB_JACOBI;   // ghost rows are not symmetric
    int project = p_singular(h);
    const bool learned = h->cs.p_form == CAFFE_P_LEARNED || h->cs.p_form == CAFFE_P_LEARNED_MIXED;
    if (learned) {
        // FP64 refinement around an FP32 flexible Krylov solve preconditioned through the level
        // pyramid and the network; the plain FP64 solve re-runs on the device if it does not
        // reach the tolerance
        if (h->ensure_learned()) return 1;
        rc = learned_solve(h->lw, A, h->ib ? h->status : nullptr, h->pb, h->pc, h->L, h->cs.p_rtol, h->cs.maxit, LEARNED_INNER_RTOL,
                           project, h->netMode, h->kw.out, h->st, h->cs.p_atol);
        if (!rc) rc = ksp_fallback_sym(A, method, h->pb, h->pc, h->L, h->kw, h->cs.p_rtol, h->cs.maxit, h->st, 0,
                                       &h->kw.out->status[0], &h->acc->fallbacks, h->cs.p_atol);
    } else if (h->cs.p_form == CAFFE_P_MIXED) {
        // FP32 inner solves inside FP64 refinement; the plain FP64 solve re-runs on the device
        // when the refinement does not reach the tolerance
        rc = ksp_mixed_sym(A, method, h->pb, h->pc, h->L, h->kw, h->cs.p_rtol, h->cs.maxit, MIXED_INNER_RTOL, h->st, project,
                           h->cs.p_atol);
        if (!rc) rc = ksp_fallback_sym(A, method, h->pb, h->pc, h->L, h->kw, h->cs.p_rtol, h->cs.maxit, h->st, 0,
                                       &h->kw.out->status[0], &h->acc->fallbacks, h->cs.p_atol);
    } else if (method == CAFFE_KSP_CG_JACOBI) {
        rc = ksp_cg(A, h->pb, h->pc, h->L, h->kw, h->cs.p_rtol, h->cs.maxit, h->st, project, h->cs.p_atol);
    } else {
        rc = ksp_bicgstab_sym(A, h->pb, h->pc, h->L, h->kw, h->cs.p_rtol, h->cs.maxit, h->st, project, h->cs.p_atol);
    }
    if (rc) return rc;
    if (project) {
        // singular system: the solution's constant is fixed to zero mean (the discrete gradient
        // on meshes with non-planar faces is not blind to it), whichever Krylov method ran
        if (!h->gaugePart && !(h->gaugePart = h->dalloc<double>(1025))) { set_error("allocation failed"); return 1; }
        int nb = (int)std::min<long long>(1024, (h->L.N + 255) / 256);
        gauge_partial_kernel<<<nb, 256, 0, h->st>>>(h->pc, h->L.N, h->gaugePart);
        gauge_mean_kernel<<<1, 256, 0, h->st>>>(h->gaugePart, nb, h->L.N);
        gauge_apply_kernel<<<grid_for(h->L.N, 256), 256, 0, h->st>>>(h->pc, h->L.N, h->gaugePart + nb);
        CB_CHECK_LAUNCH();
    }
    acc_kernel<<<1, 32, 0, h->st>>>(h->kw.out, h->acc, learned ? 2 : 1, 1);
    CB_CHECK_LAUNCH();
    if (h->recording && h->pairCount < h->pairCap) {
        // (b, x*) of this solve, then (b - A x_k, x* - x_k) for iterates x_k of truncated plain
        // re-solves after 8, 32, 128, ... iterations
        size_t slot = (size_t)h->pairCount * h->L.PS + h->L.H;
        pair_cast_kernel<<<grid_for(h->L.N, 256), 256, 0, h->st>>>(h->L.N, h->pb, h->pc, h->pairB + slot, h->pairX + slot);
        CB_CHECK_LAUNCH();
        ++h->pairCount;
        int kIt = 8;
        for (int q = 0; q < h->pairSnapshots && h->pairCount < h->pairCap; ++q, kIt *= 4) {
            if (!h->snapX && !(h->snapX = h->cell(1))) { set_error("allocation failed"); return 1; }
            rc = method == CAFFE_KSP_CG_JACOBI ? ksp_cg(A, h->pb, h->snapX, h->L, h->kw, 0., kIt, h->st, 0)
                                               : ksp_bicgstab_sym(A, h->pb, h->snapX, h->L, h->kw, 0., kIt, h->st, 0);
            if (rc) return rc;
            slot = (size_t)h->pairCount * h->L.PS + h->L.H;
            if (learned_snapshot_pair(A, h->L, h->pb, h->pc, h->snapX, h->pairB + slot, h->pairX + slot, h->st)) return 1;
            ++h->pairCount;
        }
    }
    return 0;
}
int ph_correct(caffe_dev* h) {
    if (launch_correct(h->geo(), h->bc, h->fields(), h->P, h->st)) return 1;
    for (int q = 0; q < 3; ++q) std::swap(h->F[q], h->Fb[q]);
    // a slab forms grad u separately, after its u halo planes are exchanged
    return launch_correct_post(h->geo(), h->bc, h->fields(), h->st, !h->slab);
}
int ph_continuity(caffe_dev* h) {
    return launch_continuity(h->L, h->mfc, h->vol, h->ib ? h->status : nullptr, h->chunkMax, &h->acc->continuity, h->st);
}
int ph_courant(caffe_dev* h, double dt) { return launch_courant(h->geo(), h->fields(), dt, &h->acc->courant_bits, h->st); }
int ph_ib_field(caffe_dev* h) {
    if (!h->ib) { set_error("ib_field: the handle has no immersed boundary"); return 1; }
    return ib_compute_field(h->ibs, h->geo(), h->cs, h->u, h->p, h->status, h->st);
}
int ph_ib_coeffs(caffe_dev* h) {
    if (!h->ib) { set_error("ib_coeffs: the handle has no immersed boundary"); return 1; }
    return ib_compute_coeffs(h->ibs, h->geo(), h->cs, h->status, h->ma[0], h->paP, h->st);
}

int ensure_events(std::vector<cudaEvent_t>& v, size_t n) {
    while (v.size() < n) {
        cudaEvent_t e;
        CB_CUDA(cudaEventCreate(&e));
        v.push_back(e);
    }
    return 0;
}

int do_step(caffe_dev* h, double dt) {
    const caffe_case& c = h->cs;
    CB_CUDA(cudaMemsetAsync(h->acc, 0, sizeof(StepAcc), h->st));
    CB_CUDA(cudaEventRecord(h->ev[0], h->st));
    int nIn = c.time_accurate ? c.n_inner : 1;
    int nPC = c.kind == CAFFE_SIMPLE ? 1 : c.n_pcorr;
    if (ensure_events(h->evP, (size_t)2 * nIn * nPC) || ensure_events(h->evM, (size_t)2 * nIn)) return 1;
    h->nPTimed = 0; h->nMTimed = 0;
    if (ph_save_u0(h)) return 1;                        // uField0_ = uField_
    if (c.kind == CAFFE_IBPISO && ph_ib_field(h)) return 1;
    for (int it = 0; it < nIn; ++it) {
        if (c.kind == CAFFE_IBPISO && ph_ib_coeffs(h)) return 1;
        if (ph_assemble_momentum(h, dt)) return 1;
        CB_CUDA(cudaEventRecord(h->evM[2 * h->nMTimed], h->st));
        if (ph_solve_momentum(h)) return 1;
        CB_CUDA(cudaEventRecord(h->evM[2 * h->nMTimed + 1], h->st));
        ++h->nMTimed;
        if (ph_momentum_post(h)) return 1;
        for (int q = 0; q < nPC; ++q) {
            if (ph_assemble_pcorr(h)) return 1;
            CB_CUDA(cudaEventRecord(h->evP[2 * h->nPTimed], h->st));
            if (ph_solve_pcorr(h)) return 1;
            CB_CUDA(cudaEventRecord(h->evP[2 * h->nPTimed + 1], h->st));
            ++h->nPTimed;
            if (ph_correct(h)) return 1;
        }
    }
    CB_CUDA(cudaEventRecord(h->ev[3], h->st));
    if (c.kind != CAFFE_IBPISO && ph_courant(h, dt)) return 1;
    if (ph_continuity(h)) return 1;
    CB_CUDA(cudaEventRecord(h->ev[4], h->st));
    CB_CUDA(cudaMemcpyAsync(h->accHost, h->acc, sizeof(StepAcc), cudaMemcpyDeviceToHost, h->st));
    h->stepTimed = true;
    return 0;
}

int read_stats(caffe_dev* h, caffe_step_stats* s) {
    CB_CUDA(cudaStreamSynchronize(h->st));
    const StepAcc& a = *h->accHost;
    caffe_step_stats o;
    std::memset(&o, 0, sizeof(o));
    o.continuity = a.continuity;
    double co;
    std::memcpy(&co, &a.courant_bits, sizeof(double));
    o.courant = co;
    for (int q = 0; q < 3; ++q) o.mom_iters[q] = a.mom_iters[q];
    o.p_iters_last = a.p_iters_last;
    o.p_iters_total = a.p_iters_total;
    o.p_solves = a.p_solves;
    o.p_res_max = a.p_res_max;
    o.mom_res_max = a.mom_res_max;
    o.status = a.status;
    o.fallbacks = a.fallbacks;
    o.cascades = a.cascades;
    o.net_iters = a.net_iters;
    o.n_ghost = h->ib ? h->ibs.nGhostHost : 0;
    o.n_rows = (int)(h->L.N - (h->ib ? h->ibs.nInactiveHost : 0));
    float ms = 0.f;
    if (h->stepTimed) {
        if (cudaEventElapsedTime(&ms, h->ev[0], h->ev[4]) == cudaSuccess) o.step_ms = ms;
        for (int q = 0; q < h->nPTimed; ++q)
            if (cudaEventElapsedTime(&ms, h->evP[2 * q], h->evP[2 * q + 1]) == cudaSuccess) o.p_ms += ms;
        for (int q = 0; q < h->nMTimed; ++q)
            if (cudaEventElapsedTime(&ms, h->evM[2 * q], h->evM[2 * q + 1]) == cudaSuccess) o.mom_ms += ms;
    }
    h->last = o;
    if (s) *s = o;
    return 0;
}

// named arrays --------------------------------------------------------------
struct ArrDesc {
    double* base;     // device pointer to element 0 of plane 0
    long long n;      // elements per plane
    long long stride; // plane stride on the device
    int planes;
    int kind;         // 0 plain planes, 1 momentum coefficients, 2 p' coefficients
    bool writable;
};

bool find_array(caffe_dev* h, const std::string& nm, ArrDesc& a) {
    const Lat& L = h->L;
    a.kind = 0; a.writable = true;
    auto cellv = [&](double* b, int planes) { a.base = b; a.n = L.N; a.stride = L.PS; a.planes = planes; return b != nullptr; };
    auto face = [&](double* b, long long n, int planes) { a.base = b; a.n = n; a.stride = n; a.planes = planes; return b != nullptr; };
    if (nm == "u") return cellv(h->u, 3);
    if (nm == "u0") return cellv(h->u0buf ? h->u0buf : h->u, 3);
    if (nm == "gradP") return cellv(h->gradP, 3);
    if (nm == "gradPCorr") return cellv(h->gradPC, 3);
    if (nm == "gradU") return cellv(h->gradU, 9);
    if (nm == "p") return cellv(h->p, 1);
    if (nm == "pCorr") return cellv(h->pc, 1);
    if (nm == "d") return cellv(h->d, 1);
    if (nm == "massFlow") return cellv(h->mfc, 1);
    if (nm == "vol") { a.writable = false; return cellv(h->vol, 1); }
    if (nm == "cc") { a.writable = false; return cellv(h->cc, 3); }
    if (nm == "momB") return cellv(h->mb, 3);
    if (nm == "pcB") return cellv(h->pb, 1);
    if (nm == "massFlowI") return face(h->F[0], L.nFI, 1);
    if (nm == "massFlowJ") return face(h->F[1], L.nFJ, 1);
    if (nm == "massFlowK") return face(h->F[2], L.nFK, 1);
    const char* dn[3] = {"I", "J", "K"};
    long long nf[3] = {L.nFI, L.nFJ, L.nFK};
    for (int q = 0; q < 3; ++q) {
        if (nm == std::string("S") + dn[q]) { a.writable = false; return face(h->S[q], nf[q], 3); }
        if (nm == std::string("fc") + dn[q]) { a.writable = false; return face(h->fc[q], nf[q], 3); }
        if (nm == std::string("D") + dn[q]) { a.writable = false; return face(h->D[q], nf[q], 1); }
        if (nm == std::string("cv") + dn[q]) { a.writable = false; return face(h->cv[q], nf[q], 3); }
    }
    if (nm.size() == 7 && nm.compare(0, 6, "pPatch") == 0) {
        int f = nm[6] - '0';
        if (f < 0 || f > 5) return false;
        return face(h->pPatch[f], h->patchN[f], 1);
    }
    if (nm == "status") { a.kind = 3; a.n = L.N; a.planes = 1; a.stride = L.N; a.base = nullptr; a.writable = false; return h->ib; }
    if (nm == "ibCell" || nm == "ibCol" || nm == "ibValMom" || nm == "ibValP") {
        if (!h->ib) return false;
        a.kind = nm == "ibCell" ? 4 : (nm == "ibCol" ? 5 : (nm == "ibValMom" ? 6 : 7));
        a.n = (nm == "ibCell" ? 1 : 9) * (long long)h->ibs.nGhost; a.planes = 1; a.stride = a.n; a.base = nullptr; a.writable = false;
        return true;
    }
    if (nm == "momA") { a.kind = 1; a.n = L.N; a.planes = 7; a.stride = L.PS; a.base = h->ma[0]; a.writable = false; return true; }
    if (nm == "pcA") { a.kind = 2; a.n = L.N; a.planes = 7; a.stride = L.PS; a.base = h->paP; a.writable = false; return true; }
    return false;
}

}  // namespace

extern "C" {

const char* caffe_last_error(void) { return g_err.c_str(); }

int caffe_dev_create(const double* nodes, int nNI, int nNJ, int nNK, const caffe_case* cs, int device, caffe_dev** out) {
    g_err.clear();
    if (!out) { set_error("out is NULL"); return 1; }
    *out = nullptr;
    if (!nodes) { set_error("nodes is NULL"); return 1; }
    if (nNI < 2 || nNJ < 2 || nNK < 2) { set_error("a mesh needs at least 2 nodes per direction"); return 1; }
    if (validate_case(cs)) return 1;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device available"); return 1; }
    if (device < 0 || device >= ndev) { set_error("device ordinal out of range"); return 1; }
    CB_CUDA(cudaSetDevice(device));
    caffe_dev* h = new caffe_dev();
    h->device = device;
    h->cs = *cs;
    h->ib = cs->kind == CAFFE_IBPISO;
    h->L = make_lat(nNI - 1, nNJ - 1, nNK - 1);
    const Lat& L = h->L;
    auto fail = [&]() { delete h; return 1; };
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { set_error("stream creation failed"); return fail(); }
    if (setup_bcs(h)) return fail();
    h->P.rho = cs->rho; h->P.mu = cs->mu; h->P.omega_u = cs->omega_u; h->P.omega_p = cs->omega_p;
    h->P.unsteady = cs->time_accurate ? 1 : 0; h->P.convection = cs->convection;
    // metrics
    h->vol = h->cell(1); h->cc = h->cell(3);
    long long nf[3] = {L.nFI, L.nFJ, L.nFK};
    for (int q = 0; q < 3; ++q) {
        h->S[q] = h->dalloc<double>(3 * nf[q]);
        h->fc[q] = h->dalloc<double>(3 * nf[q]);
        h->D[q] = h->dalloc<double>(nf[q]);
        if (cs->nonorth) h->cv[q] = h->dalloc<double>(3 * nf[q]);
    }
    // fields
    h->u = h->cell(3);
    int nIn = cs->time_accurate ? cs->n_inner : 1;
    if (nIn > 1) h->u0buf = h->cell(3);
    h->gradP = h->cell(3); h->gradPC = h->cell(3);
    if (cs->nonorth) h->gradU = h->cell(9);
    h->p = h->cell(1); h->pc = h->cell(1); h->d = h->cell(1); h->mfc = h->cell(1);
    for (int q = 0; q < 3; ++q) { h->F[q] = h->dalloc<double>(nf[q]); h->Fb[q] = h->dalloc<double>(nf[q]); }
    h->patchN[0] = h->patchN[1] = (long long)L.nJ * L.nK;
    h->patchN[2] = h->patchN[3] = (long long)L.nI * L.nK;
    h->patchN[4] = h->patchN[5] = (long long)L.nI * L.nJ;
    for (int f = 0; f < 6; ++f) h->pPatch[f] = h->dalloc<double>(h->patchN[f]);
    // systems
    for (int q = 0; q < 7; ++q) h->ma[q] = h->cell(1);
    h->mb = h->cell(3);
    h->paP = h->cell(1); h->paE = h->cell(1); h->paN = h->cell(1); h->paT = h->cell(1); h->pb = h->cell(1);
    // Krylov workspace
    h->kw.r = h->cell(3); h->kw.rp = h->cell(3);
    h->kw.p[0] = h->cell(3); h->kw.p[1] = h->cell(3);
    h->kw.v[0] = h->cell(3); h->kw.v[1] = h->cell(3);
    h->kw.t = h->cell(3); h->kw.invD = h->cell(1);
    if (cs->p_form == CAFFE_P_MIXED || cs->p_form == CAFFE_P_LEARNED_MIXED) {
        for (int q = 0; q < 2; ++q) { h->kw.fr[q] = h->fcell(); h->kw.fw[q] = h->fcell(); h->kw.fs[q] = h->fcell(); h->kw.fv[q] = h->fcell(); }
        h->kw.fp = h->fcell(); h->kw.fe = h->fcell(); h->kw.ft = h->fcell(); h->kw.finvD = h->fcell();
        for (int q = 0; q < 4; ++q) h->kw.fA[q] = h->fcell();
        bool ok = h->kw.fp && h->kw.fe && h->kw.ft && h->kw.finvD;
        for (int q = 0; q < 2; ++q) ok = ok && h->kw.fr[q] && h->kw.fw[q] && h->kw.fs[q] && h->kw.fv[q];
        for (int q = 0; q < 4; ++q) ok = ok && h->kw.fA[q];
        if (!ok) { set_error("device allocation failed (mixed-precision workspace)"); return fail(); }
    }
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    h->kw.partials = h->dalloc<double>((size_t)2 * 8 * 8 * (nsm > 0 ? nsm : 256));
    h->kw.out = h->dalloc<KspOut>(1);
    h->chunkMax = h->dalloc<double>((size_t)(L.N / 1024 + 2));
    h->acc = h->dalloc<StepAcc>(1);
    if (cudaMallocHost(&h->accHost, sizeof(StepAcc)) != cudaSuccess) { set_error("pinned allocation failed"); return fail(); }
    std::memset(h->accHost, 0, sizeof(StepAcc));
    for (void* a : h->allocs) if (!a) { set_error("device allocation failed"); return fail(); }
    bool anyNull = !h->vol || !h->cc || !h->u || !h->gradP || !h->gradPC || !h->p || !h->pc || !h->d || !h->mfc || !h->mb ||
                   !h->paP || !h->paE || !h->paN || !h->paT || !h->pb || !h->kw.r || !h->kw.rp || !h->kw.t || !h->kw.invD ||
                   !h->kw.partials || !h->kw.out || !h->chunkMax || !h->acc;
    for (int q = 0; q < 3; ++q) anyNull = anyNull || !h->S[q] || !h->fc[q] || !h->D[q] || !h->F[q] || !h->Fb[q];
    for (int q = 0; q < 7; ++q) anyNull = anyNull || !h->ma[q];
    if (anyNull) { set_error("device allocation failed (out of memory?)"); return fail(); }
    for (auto& e : h->ev) if (cudaEventCreate(&e) != cudaSuccess) { set_error("event creation failed"); return fail(); }
    // mesh metrics from the nodes
    size_t nn = (size_t)nNI * nNJ * nNK * 3;
    double* dxyz = nullptr;
    if (cudaMalloc(&dxyz, nn * sizeof(double)) != cudaSuccess) { set_error("node upload allocation failed"); return fail(); }
    int rc = cudaMemcpyAsync(dxyz, nodes, nn * sizeof(double), cudaMemcpyHostToDevice, h->st) != cudaSuccess;
    if (rc) set_error("node upload failed");
    if (!rc) rc = compute_metrics(L, dxyz, h->vol, h->cc, h->S, h->fc, h->D, h->cv, h->st);
    if (!rc && h->ib) {
        Alloc al = [h](size_t bytes) { return h->dalloc<char>(bytes); };
        rc = ib_create(h->ibs, L, h->status, al, h->st);
        if (!rc) rc = ib_setup(h->ibs, h->geo(), h->cs, dxyz, h->status, al, h->st);
    }
    cudaStreamSynchronize(h->st);
    cudaFree(dxyz);
    if (rc) { if (g_err.empty()) set_error("metric computation failed"); return fail(); }
    // initial state (InitialConditions uniform: cells only)
    if (fill(h, h->u, 3, cs->u_init[0], cs->u_init[1], cs->u_init[2])) return fail();
    if (fill(h, h->p, 1, cs->p_init)) return fail();
    if (init_p_patches(h)) return fail();
    if (cudaStreamSynchronize(h->st) != cudaSuccess) { set_error(std::string("initialisation: ") + cudaGetErrorString(cudaGetLastError())); return fail(); }
    std::memset(&h->last, 0, sizeof(h->last));
    *out = h;
    return 0;
}

int caffe_dev_destroy(caffe_dev* h) {
    if (!h) return 0;
    cudaSetDevice(h->device);
    delete h;
    return 0;
}

int caffe_dev_solve(caffe_dev* h, double dt, caffe_step_stats* stats) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (h->slab) {
        // a slab's step needs its halo planes exchanged between phases and its solves summed over
        // the slabs: the caller runs it through caffe_slab_phase / caffe_slab_ksp / caffe_slab_halo
        set_error("the handle is one slab of a decomposition: its step runs through the caffe_slab_* phases");
        return 1;
    }
    if (!(dt > 0.) && h->cs.time_accurate) { set_error("time step must be positive"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (do_step(h, dt)) return 1;
    if (stats) {
        if (read_stats(h, stats)) return 1;
        if (stats->status == 3) { set_error("non-finite residual in a linear solve"); return 3; }
    }
    return 0;
}

int caffe_dev_stats(caffe_dev* h, caffe_step_stats* stats) {
    if (!h || !stats) { set_error("NULL argument"); return 1; }
    return read_stats(h, stats);
}

int caffe_dev_phase(caffe_dev* h, const char* name, double dt) {
    g_err.clear();
    if (!h || !name) { set_error("NULL argument"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    std::string n(name);
    int rc;
    if (n == "save_u0") rc = ph_save_u0(h);
    else if (n == "assemble_momentum") rc = ph_assemble_momentum(h, dt);
    else if (n == "solve_momentum") { CB_CUDA(cudaMemsetAsync(h->acc, 0, sizeof(StepAcc), h->st)); rc = ph_solve_momentum(h); }
    else if (n == "momentum_post") rc = ph_momentum_post(h);
    else if (n == "assemble_pcorr") rc = ph_assemble_pcorr(h);
    else if (n == "solve_pcorr") { CB_CUDA(cudaMemsetAsync(h->acc, 0, sizeof(StepAcc), h->st)); rc = ph_solve_pcorr(h); }
    else if (n == "correct") rc = ph_correct(h);
    else if (n == "continuity") { CB_CUDA(cudaMemsetAsync(h->acc, 0, sizeof(StepAcc), h->st)); rc = ph_continuity(h); }
    else if (n == "courant") { CB_CUDA(cudaMemsetAsync(h->acc, 0, sizeof(StepAcc), h->st)); rc = ph_courant(h, dt); }
    else if (n == "ib_field") rc = ph_ib_field(h);
    else if (n == "ib_coeffs") rc = ph_ib_coeffs(h);
    else { set_error("unknown phase " + n); return 2; }
    if (rc) return rc;
    CB_CUDA(cudaMemcpyAsync(h->accHost, h->acc, sizeof(StepAcc), cudaMemcpyDeviceToHost, h->st));
    CB_CUDA(cudaStreamSynchronize(h->st));
    h->stepTimed = false;
    return 0;
}

long caffe_dev_array(caffe_dev* h, const char* name, double* host, long count, int dir) {
    g_err.clear();
    if (!h || !name) { set_error("NULL argument"); return -1; }
    ArrDesc a;
    if (!find_array(h, name, a)) { set_error(std::string("unknown array ") + name); return -1; }
    long need = (long)(a.n * a.planes);
    if (!host) return need;
    if (count < need) { set_error("host buffer too small"); return -1; }
    bool planar = (dir & 2) != 0;
    bool toDev = (dir & 1) != 0;
    if (toDev && (!a.writable || a.kind != 0)) { set_error(std::string("array is read-only: ") + name); return -1; }
    if (cudaSetDevice(h->device) != cudaSuccess) { set_error("cudaSetDevice failed"); return -1; }
    if (cudaStreamSynchronize(h->st) != cudaSuccess) { set_error(std::string("stream: ") + cudaGetErrorString(cudaGetLastError())); return -1; }
    if (a.kind >= 3) {
        // cell status (uint8) and immersed-boundary ghost rows, converted to doubles
        if (a.kind == 3) {
            std::vector<uint8_t> v((size_t)a.n);
            if (cudaMemcpy(v.data(), h->status, a.n, cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
            for (long long q = 0; q < a.n; ++q) host[q] = v[q];
        } else if (a.kind == 4 || a.kind == 5) {
            std::vector<int> v((size_t)a.n);
            const int* src = a.kind == 4 ? h->ibs.gCell : h->ibs.gCol;
            if (a.n && cudaMemcpy(v.data(), src, a.n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
            for (long long q = 0; q < a.n; ++q) host[q] = v[q];
        } else {
            const double* src = a.kind == 6 ? h->ibs.gValMom : h->ibs.gValP;
            if (a.n && cudaMemcpy(host, src, a.n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
        }
        return need;
    }
    if (a.kind != 0) {
        // coefficient matrices: host layout [N][7] in the order aP aE aW aN aS aT aB
        std::vector<double> planes((size_t)7 * a.n);
        const Lat& L = h->L;
        if (a.kind == 1) {
            for (int q = 0; q < 7; ++q)
                if (cudaMemcpy(planes.data() + q * a.n, h->ma[q], a.n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
        } else {
            std::vector<double> aP(a.n), aE(a.n + L.H), aN(a.n + L.H), aT(a.n + L.H);
            if (cudaMemcpy(aP.data(), h->paP, a.n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(aE.data(), h->paE - L.H, (a.n + L.H) * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(aN.data(), h->paN - L.H, (a.n + L.H) * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(aT.data(), h->paT - L.H, (a.n + L.H) * 8, cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
            long long H = L.H;
            for (long long c = 0; c < a.n; ++c) {
                planes[c] = aP[c];
                planes[a.n + c] = aE[H + c];
                planes[2 * a.n + c] = aE[H + c - 1];
                planes[3 * a.n + c] = aN[H + c];
                planes[4 * a.n + c] = aN[H + c - L.nI];
                planes[5 * a.n + c] = aT[H + c];
                planes[6 * a.n + c] = aT[H + c - L.nIJ];
            }
        }
        for (long long c = 0; c < a.n; ++c)
            for (int q = 0; q < 7; ++q) host[c * 7 + q] = planes[q * a.n + c];
        return need;
    }
    if (planar || a.planes == 1) {
        for (int q = 0; q < a.planes; ++q) {
            cudaError_t e = toDev ? cudaMemcpyAsync(a.base + q * a.stride, host + q * a.n, a.n * sizeof(double), cudaMemcpyHostToDevice, h->st)
                                  : cudaMemcpyAsync(host + q * a.n, a.base + q * a.stride, a.n * sizeof(double), cudaMemcpyDeviceToHost, h->st);
            if (e != cudaSuccess) { set_error(std::string("copy failed: ") + cudaGetErrorString(e)); return -1; }
        }
        if (cudaStreamSynchronize(h->st) != cudaSuccess) { set_error("copy sync failed"); return -1; }
        return need;
    }
    std::vector<double> tmp((size_t)a.n * a.planes);
    if (toDev) {
        for (long long c = 0; c < a.n; ++c)
            for (int q = 0; q < a.planes; ++q) tmp[q * a.n + c] = host[c * a.planes + q];
    }
    for (int q = 0; q < a.planes; ++q) {
        cudaError_t e = toDev ? cudaMemcpy(a.base + q * a.stride, tmp.data() + q * a.n, a.n * sizeof(double), cudaMemcpyHostToDevice)
                              : cudaMemcpy(tmp.data() + q * a.n, a.base + q * a.stride, a.n * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { set_error(std::string("copy failed: ") + cudaGetErrorString(e)); return -1; }
    }
    if (!toDev) {
        for (long long c = 0; c < a.n; ++c)
            for (int q = 0; q < a.planes; ++q) host[c * a.planes + q] = tmp[q * a.n + c];
    }
    return need;
}

void* caffe_dev_stream(caffe_dev* h) { return h ? (void*)h->st : nullptr; }

int caffe_dev_synchronize(caffe_dev* h) {
    if (!h) { set_error("handle is NULL"); return 1; }
    CB_CUDA(cudaStreamSynchronize(h->st));
    return 0;
}

int caffe_dev_set_stream(caffe_dev* h, void* stream) {
    g_err.clear();
    if (!h || !stream) { set_error("NULL argument"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    CB_CUDA(cudaStreamSynchronize(h->st));
    if (h->ownStream) CB_CUDA(cudaStreamDestroy(h->st));
    h->st = static_cast<cudaStream_t>(stream);
    h->ownStream = false;
    return 0;
}

// ------------------------------------------------------------------ k-slab decomposition
int caffe_slab_set_owned(caffe_dev* h, int k0, int k1) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (h->ib) { set_error("slab: the immersed-boundary solver is not decomposed"); return 1; }
    if (h->cs.p_form != CAFFE_P_FP64) { set_error("slab: only the plain FP64 pressure-correction solve is decomposed"); return 1; }
    if (k0 < 0 || k1 > h->L.nK || k0 >= k1) { set_error("slab: owned planes must satisfy 0 <= k0 < k1 <= nK"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (!h->slabPh && !(h->slabPh = h->cell(3))) { set_error("allocation failed"); return 1; }
    if (!h->slabSh && !(h->slabSh = h->cell(3))) { set_error("allocation failed"); return 1; }
    if (!h->slabPart && !(h->slabPart = h->dalloc<double>((size_t)SLAB_MAX_BLOCKS * 8))) { set_error("allocation failed"); return 1; }
    h->slab = true;
    h->o0 = (long long)k0 * h->L.nIJ;
    h->o1 = (long long)k1 * h->L.nIJ;
    return 0;
}

namespace {
int slab_array(caffe_dev* h, const std::string& n, double** base, int* planes) {
    *base = nullptr; *planes = 0;
    if (n == "u") { *base = h->u; *planes = 3; }
    else if (n == "p") { *base = h->p; *planes = 1; }
    else if (n == "pCorr") { *base = h->pc; *planes = 1; }
    else if (n == "d") { *base = h->d; *planes = 1; }
    else if (n == "gradP") { *base = h->gradP; *planes = 3; }
    else if (n == "gradPCorr") { *base = h->gradPC; *planes = 3; }
    else if (n == "gradU" && h->gradU) { *base = h->gradU; *planes = 9; }
    else if (n == "kspPh") { *base = h->slabPh; *planes = 3; }
    else if (n == "kspSh") { *base = h->slabSh; *planes = 3; }
    return *base ? 0 : 1;
}
}  // namespace

long caffe_slab_halo(caffe_dev* h, const char* name, int planes, int side, int dir, double* buf) {
    g_err.clear();
    if (!h || !name) { set_error("NULL argument"); return -1; }
    if (!h->slab) { set_error("slab: caffe_slab_set_owned has not been called"); return -1; }
    double* base;
    int np;
    if (slab_array(h, name, &base, &np)) { set_error(std::string("slab: no halo exchange for array ") + name); return -1; }
    if (planes <= 0) planes = np;
    if (planes > np) { set_error("slab: more planes than the array has"); return -1; }
    const long long nIJ = h->L.nIJ;
    const int k0 = (int)(h->o0 / nIJ), k1 = (int)(h->o1 / nIJ);
    int own, halo;
    if (side == 0) {
        if (k0 == 0) { set_error("slab: no halo below the first plane of the lattice"); return -1; }
        own = k0; halo = k0 - 1;
    } else if (side == 1) {
        if (k1 == h->L.nK) { set_error("slab: no halo above the last plane of the lattice"); return -1; }
        own = k1 - 1; halo = k1;
    } else {
        set_error("slab: side is 0 (below) or 1 (above)");
        return -1;
    }
    const long count = (long)planes * (long)nIJ;
    if (!buf) return count;
    CB_CUDA(cudaSetDevice(h->device));
    const size_t row = (size_t)nIJ * sizeof(double), pitch = (size_t)h->L.PS * sizeof(double);
    if (dir == 0) {
        if (cudaMemcpy2DAsync(buf, row, base + (long long)own * nIJ, pitch, row, planes, cudaMemcpyDeviceToDevice, h->st) != cudaSuccess) {
            set_error("slab: halo pack failed"); return -1;
        }
    } else if (dir == 1) {
        if (cudaMemcpy2DAsync(base + (long long)halo * nIJ, pitch, buf, row, row, planes, cudaMemcpyDeviceToDevice, h->st) != cudaSuccess) {
            set_error("slab: halo unpack failed"); return -1;
        }
    } else {
        set_error("slab: dir is 0 (pack the owned plane) or 1 (unpack into the halo plane)");
        return -1;
    }
    return count;
}

int caffe_slab_ksp(caffe_dev* h, int sys, int phase, const double* scal, double* red) {
    g_err.clear();
    if (!h || !red) { set_error("NULL argument"); return -1; }
    if (!h->slab) { set_error("slab: caffe_slab_set_owned has not been called"); return -1; }
    CB_CUDA(cudaSetDevice(h->device));
    SlabKsp k;
    k.L = h->L; k.o0 = h->o0; k.o1 = h->o1;
    k.w = h->kw; k.ph = h->slabPh; k.sh = h->slabSh; k.part = h->slabPart; k.red = red;
    SlabScal s;
    for (int q = 0; q < 3; ++q) {
        s.alpha[q] = scal ? scal[4 * q] : 0.;
        s.beta[q] = scal ? scal[4 * q + 1] : 0.;
        s.omega[q] = scal ? scal[4 * q + 2] : 0.;
        s.flags[q] = scal ? (int)scal[4 * q + 3] : 0;
    }
    if (sys == 0) { k.b = h->mb; k.x = h->u; return slab_ksp_phase(h->momOp(), 3, phase, k, s, h->st); }
    if (sys == 1) { k.b = h->pb; k.x = h->pc; return slab_ksp_phase(h->pOp(), 1, phase, k, s, h->st); }
    set_error("slab: system 0 (momentum) or 1 (pressure correction)");
    return -1;
}

int caffe_slab_phase(caffe_dev* h, const char* name, double dt) {
    g_err.clear();
    if (!h || !name) { set_error("NULL argument"); return 1; }
    if (!h->slab) { set_error("slab: caffe_slab_set_owned has not been called"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    std::string n(name);
    if (n == "save_u0") return ph_save_u0(h);
    if (n == "assemble_momentum") return ph_assemble_momentum(h, dt);
    if (n == "momentum_post") return ph_momentum_post(h);
    if (n == "assemble_pcorr") return ph_assemble_pcorr(h);
    if (n == "correct") return ph_correct(h);
    if (n == "grad_u") return launch_grad_u(h->geo(), h->bc, h->fields(), h->st);
    set_error("slab: unknown phase " + n);
    return 1;
}

int caffe_slab_reduce(caffe_dev* h, const char* what, double dt, double* red) {
    g_err.clear();
    if (!h || !what || !red) { set_error("NULL argument"); return 1; }
    if (!h->slab) { set_error("slab: caffe_slab_set_owned has not been called"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    std::string n(what);
    if (n == "continuity") {
        // Simple.cpp:358-380 on this slab's cells, in their k-j-i order
        Lat Lo = h->L;
        Lo.N = h->o1 - h->o0;
        return launch_continuity(Lo, h->mfc + h->o0, h->vol + h->o0, nullptr, h->chunkMax, red, h->st);
    }
    if (n == "courant") return launch_courant(h->geo(), h->fields(), dt, reinterpret_cast<unsigned long long*>(red), h->st, h->o0, h->o1);
    set_error("slab: unknown reduction " + n);
    return 1;
}

int caffe_dev_set_precond(caffe_dev* h, const float* params) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned()) return 1;
    if (!params) { h->lw.haveParams = false; return 0; }
    if (!h->lw.weights) { set_error("lattice too small for the level pyramid of the learned preconditioner"); return 1; }
    CB_CUDA(cudaMemcpyAsync(h->lw.weights->params, params, sizeof(float) * NET_PARAMS, cudaMemcpyHostToDevice, h->st));
    if (net_pack_weights(*h->lw.weights, h->st)) return 1;
    CB_CUDA(cudaStreamSynchronize(h->st));
    h->lw.haveParams = true;
    return 0;
}

int caffe_dev_get_precond(caffe_dev* h, float* params) {
    g_err.clear();
    if (!h || !params) { set_error("NULL argument"); return 1; }
    if (!h->haveLearned || !h->lw.haveParams || !h->lw.weights) { set_error("no preconditioner parameters on this handle"); return 1; }
    CB_CUDA(cudaMemcpyAsync(params, h->lw.weights->params, sizeof(float) * NET_PARAMS, cudaMemcpyDeviceToHost, h->st));
    CB_CUDA(cudaStreamSynchronize(h->st));
    return 0;
}

int caffe_dev_set_precond_mode(caffe_dev* h, int mode) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (mode < NET_MODE_JACOBI || mode > NET_MODE_LEVELS) { set_error("unknown preconditioner mode"); return 1; }
    h->netMode = mode;
    return 0;
}

int caffe_dev_set_precond_options(caffe_dev* h, int inner_method, int net_from_level, int restart) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (inner_method < LEARN_INNER_AUTO || inner_method > LEARN_INNER_FGMRES || net_from_level < 1 || restart < 1 ||
        restart > FGMRES_MAX_RESTART) {
        set_error("invalid options");
        return 1;
    }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned()) return 1;
    if (h->lw.fgCap > 0 && restart > h->lw.fgCap) { set_error("the FGMRES restart length cannot grow after the first FGMRES solve"); return 1; }
    h->lw.inner = inner_method;
    h->lw.netFrom = net_from_level;
    h->lw.restart = restart;
    return 0;
}

int caffe_dev_set_precond_net_levels(caffe_dev* h, int first_level, int last_level) {
    g_err.clear();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (first_level < 1 || (last_level >= 0 && last_level < first_level)) { set_error("invalid network levels"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned()) return 1;
    h->lw.netFrom = first_level;
    h->lw.netTo = last_level < 0 ? (1 << 20) : last_level;
    return 0;
}

int caffe_dev_record_pairs(caffe_dev* h, int capacity, int snapshots) {
    g_err.clear();
    if (!h || capacity < 0 || snapshots < 0 || snapshots > 8) { set_error("invalid arguments"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    h->pairSnapshots = snapshots;
    if (capacity == 0) { h->recording = false; return 0; }
    if (h->ensure_pairs(capacity)) return 1;
    h->recording = true;
    return 0;
}

int caffe_dev_pair_count(caffe_dev* h) {
    if (!h) { set_error("handle is NULL"); return -1; }
    return h->pairCount;
}

int caffe_dev_add_pairs(caffe_dev* h, const float* b_pairs, const float* x_pairs, int n_pairs) {
    g_err.clear();
    if (!h || !b_pairs || !x_pairs || n_pairs < 0) { set_error("invalid arguments"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_pairs(h->pairCount + n_pairs)) return 1;
    const Lat& L = h->L;
    for (int q = 0; q < n_pairs; ++q) {
        size_t slot = (size_t)h->pairCount * L.PS + L.H;
        CB_CUDA(cudaMemcpyAsync(h->pairB + slot, b_pairs + (size_t)q * L.N, sizeof(float) * L.N, cudaMemcpyHostToDevice, h->st));
        CB_CUDA(cudaMemcpyAsync(h->pairX + slot, x_pairs + (size_t)q * L.N, sizeof(float) * L.N, cudaMemcpyHostToDevice, h->st));
        ++h->pairCount;
    }
    CB_CUDA(cudaStreamSynchronize(h->st));
    return 0;
}

int caffe_dev_add_random_pairs(caffe_dev* h, int n_pairs, unsigned seed) {
    g_err.clear();
    if (!h || n_pairs < 0) { set_error("invalid arguments"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned() || h->ensure_pairs(h->pairCount + n_pairs)) return 1;
    size_t off = (size_t)h->pairCount * h->L.PS;
    if (learned_random_pairs(h->lw, h->pOp(), h->ib ? h->status : nullptr, h->L, n_pairs, seed, h->pairB + off, h->pairX + off, h->st))
        return 1;
    CB_CUDA(cudaStreamSynchronize(h->st));
    h->pairCount += n_pairs;
    return 0;
}

int caffe_dev_copy_pairs(caffe_dev* dst, caffe_dev* src) {
    g_err.clear();
    if (!dst || !src) { set_error("handle is NULL"); return 1; }
    if (dst->device != src->device || dst->L.nI != src->L.nI || dst->L.nJ != src->L.nJ || dst->L.nK != src->L.nK) {
        set_error("pairs can only be copied between handles with the same lattice on the same device");
        return 1;
    }
    if (src->pairCount == 0) return 0;
    CB_CUDA(cudaSetDevice(dst->device));
    CB_CUDA(cudaStreamSynchronize(src->st));
    if (dst->ensure_pairs(dst->pairCount + src->pairCount)) return 1;
    size_t plane = (size_t)dst->L.PS;
    CB_CUDA(cudaMemcpyAsync(dst->pairB + (size_t)dst->pairCount * plane, src->pairB, sizeof(float) * plane * src->pairCount,
                            cudaMemcpyDeviceToDevice, dst->st));
    CB_CUDA(cudaMemcpyAsync(dst->pairX + (size_t)dst->pairCount * plane, src->pairX, sizeof(float) * plane * src->pairCount,
                            cudaMemcpyDeviceToDevice, dst->st));
    CB_CUDA(cudaStreamSynchronize(dst->st));
    dst->pairCount += src->pairCount;
    return 0;
}

int caffe_dev_train_precond(caffe_dev* h, int steps, int batch, float lr, unsigned seed, float* params_inout, float* loss_hist) {
    g_err.clear();
    if (!h || !params_inout || steps < 0 || batch < 1) { set_error("invalid arguments"); return 1; }
    if (h->pairCount < 1) { set_error("no training pairs on this handle"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned()) return 1;
    if (!h->lw.weights) { set_error("lattice too small for the level pyramid of the learned preconditioner"); return 1; }
    CB_CUDA(cudaMemcpyAsync(h->lw.weights->params, params_inout, sizeof(float) * NET_PARAMS, cudaMemcpyHostToDevice, h->st));
    int rc = learned_train(h->lw, h->pOp(), h->ib ? h->status : nullptr, h->L, h->pairB, h->pairX, h->pairCount, steps, batch, lr, seed,
                           loss_hist, h->st);
    if (rc) return rc;
    CB_CUDA(cudaMemcpy(params_inout, h->lw.weights->params, sizeof(float) * NET_PARAMS, cudaMemcpyDeviceToHost));
    return 0;
}

int caffe_dev_eval_precond(caffe_dev* h, int mode, float* loss) {
    g_err.clear();
    if (!h || !loss) { set_error("NULL argument"); return 1; }
    if (mode < NET_MODE_JACOBI || mode > NET_MODE_LEVELS) { set_error("unknown preconditioner mode"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (h->ensure_learned()) return 1;
    return learned_eval(h->lw, h->pOp(), h->ib ? h->status : nullptr, h->L, h->pairB, h->pairX, h->pairCount, mode, loss, h->st);
}

int caffe_ksp7_solve_device(int nI, int nJ, int nK, const double* d_coef7, const double* d_b, double* d_x, int method, double rtol,
                            int maxit, void* stream, int* iters, double* rel_res) {
    g_err.clear();
    if (nI < 1 || nJ < 1 || nK < 1 || !d_coef7 || !d_b || !d_x) { set_error("invalid arguments"); return 1; }
    if (maxit < 1) { set_error("maxit must be >= 1"); return 1; }
    if (method == CAFFE_KSP_BICGSTAB_SGS) { set_error(SGS_UNAVAILABLE); return 1; }
    if (method != CAFFE_KSP_BICGSTAB_JACOBI && method != CAFFE_KSP_CG_JACOBI) { set_error("invalid Krylov method"); return 1; }
    cudaStream_t st = (cudaStream_t)stream;
    Lat L = make_lat(nI, nJ, nK);
    std::vector<void*> tmp;
    auto cellbuf = [&](int planes) -> double* {
        void* p = nullptr;
        if (cudaMalloc(&p, (size_t)L.PS * planes * sizeof(double)) != cudaSuccess) return nullptr;
        cudaMemsetAsync(p, 0, (size_t)L.PS * planes * sizeof(double), st);
        tmp.push_back(p);
        return static_cast<double*>(p) + L.H;
    };
    auto cleanup = [&]() { cudaStreamSynchronize(st); for (void* p : tmp) cudaFree(p); };
    Op7 A;
    double* a7[7];
    for (int q = 0; q < 7; ++q) a7[q] = cellbuf(1);
    double* b = cellbuf(1);
    double* x = cellbuf(1);
    KspWork w;
    std::memset(&w, 0, sizeof(w));
    // same shape as a handle's workspace: every vector has 3 planes (the CG kernel uses
    // the second plane of r as its double buffer)
    w.r = cellbuf(3); w.rp = cellbuf(3); w.p[0] = cellbuf(3); w.p[1] = cellbuf(3);
    w.v[0] = cellbuf(3); w.v[1] = cellbuf(3); w.t = cellbuf(3); w.invD = cellbuf(1);
    void* part = nullptr;
    void* outp = nullptr;
    bool ok = cudaMalloc(&part, 2 * 8 * 8 * 1024 * sizeof(double)) == cudaSuccess && cudaMalloc(&outp, sizeof(KspOut)) == cudaSuccess;
    if (part) tmp.push_back(part);
    if (outp) tmp.push_back(outp);
    for (int q = 0; q < 7; ++q) ok = ok && a7[q];
    ok = ok && b && x && w.r && w.rp && w.p[0] && w.p[1] && w.v[0] && w.v[1] && w.t && w.invD;
    if (!ok) { cleanup(); set_error("workspace allocation failed"); return 1; }
    w.partials = static_cast<double*>(part);
    w.out = static_cast<KspOut*>(outp);
    for (int q = 0; q < 7; ++q) {
        if (cudaMemcpyAsync(a7[q], d_coef7 + (size_t)q * L.N, L.N * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            cleanup(); set_error("coefficient copy failed"); return 1;
        }
        A.a[q] = a7[q];
    }
    if (cudaMemcpyAsync(b, d_b, L.N * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) { cleanup(); set_error("rhs copy failed"); return 1; }
    A.nI = L.nI; A.nIJ = L.nIJ;
    A.gh.n = 0; A.gh.cell = nullptr; A.gh.col = nullptr; A.gh.val = nullptr; A.gh.bits = nullptr;
    int rc;
    if (method == CAFFE_KSP_CG_JACOBI) rc = ksp_cg7(A, b, x, L, w, rtol, maxit, st);
    else rc = ksp_bicgstab(A, 1, b, x, L, w, rtol, maxit, st);
    if (rc) { cleanup(); return rc; }
    KspOut o;
    if (cudaMemcpyAsync(d_x, x, L.N * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(&o, w.out, sizeof(KspOut), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        std::string m = std::string("solve failed: ") + cudaGetErrorString(cudaGetLastError());
        cleanup(); set_error(m); return 1;
    }
    cleanup();
    if (iters) *iters = o.iters[0];
    if (rel_res) *rel_res = o.relres[0];
    return o.status[0];
}

int caffe_ksp7_solve(int nI, int nJ, int nK, const double* coef7, const double* b, double* x, int method, double rtol, int maxit,
                     int* iters, double* rel_res) {
    g_err.clear();
    if (nI < 1 || nJ < 1 || nK < 1 || !coef7 || !b || !x) { set_error("invalid arguments"); return 1; }
    size_t N = (size_t)nI * nJ * nK;
    double *dc = nullptr, *db = nullptr, *dx = nullptr;
    if (cudaMalloc(&dc, 7 * N * sizeof(double)) != cudaSuccess || cudaMalloc(&db, N * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dx, N * sizeof(double)) != cudaSuccess) {
        cudaFree(dc); cudaFree(db); cudaFree(dx);
        set_error("allocation failed");
        return 1;
    }
    int rc = 1;
    if (cudaMemcpy(dc, coef7, 7 * N * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(db, b, N * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess) {
        rc = caffe_ksp7_solve_device(nI, nJ, nK, dc, db, dx, method, rtol, maxit, nullptr, iters, rel_res);
        if (rc != 1 && cudaMemcpy(x, dx, N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy back failed"); rc = 1; }
    } else {
        set_error("upload failed");
    }
    cudaFree(dc); cudaFree(db); cudaFree(dx);
    return rc;
}

}  // extern "C"
