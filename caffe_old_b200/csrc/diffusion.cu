// Device path of the reference's Diffusion solver (src/Solvers/Diffusion.cpp:35-131): scalar
// diffusion with unit diffusivity on one block of the structured mesh.  One solve() is
//   assemble  a_nb = +D_f, a_P = -sum_f D_f + V/dt, b = (V/dt) phi0 (Diffusion.cpp:73-85, the
//             coefficients as the reference writes them), boundary folding as
//             PrimitiveBoundaryCondition::setImplicit (PrimitiveBoundaryCondition.tpp:145-255);
//   solve     the 7-point system on the persistent Jacobi-preconditioned Krylov kernels;
//   post      phi = x, zero-gradient patches refreshed, interior faces volume-weighted, cell
//             gradients by the divergence theorem, interior faces re-extrapolated from both cells'
//             gradients and clamped to the range of the lower cell and its neighbours
//             (FvScalarScheme::extrapolateInteriorFaces, FvScalarScheme.cpp:70-156), gradients
//             again, and ||A x - b||_inf (Diffusion.cpp:127-130).
// Built with --fmad=false and the operand order of the reference, so every step outside the Krylov
// solve is bit for bit the CPU restatement's.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "krylov.cuh"

namespace cb {
int compute_metrics(const Lat& L, const double* d_xyz, double* vol, double* cc, double* S[3], double* fc[3], double* D[3], double* cv[3],
                    cudaStream_t st);
}

using namespace cb;

struct caffe_diffusion {
    int device = 0;
    cudaStream_t st = nullptr;
    Lat L;
    int types[6] = {0, 0, 0, 0, 0, 0};
    double refs[6] = {0, 0, 0, 0, 0, 0};
    int unsteady = 0, method = 1, maxit = 10000;
    double rtol = 1e-8;
    std::vector<void*> allocs;
    double* vol = nullptr;
    double* cc = nullptr;
    double* S[3] = {};
    double* fc[3] = {};
    double* D[3] = {};
    double* phi = nullptr;
    double* face[3] = {};
    double* patch[6] = {};
    long long patchN[6] = {};
    double* grad = nullptr;
    double* a[7] = {};
    double* b = nullptr;
    double* x = nullptr;
    double* resMax = nullptr;
    KspWork kw;
    int iters = 0;
    double relres = 0.;

    template <class T>
    T* dalloc(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, count * sizeof(T) + 256) != cudaSuccess) return nullptr;
        cudaMemsetAsync(p, 0, count * sizeof(T) + 256, st);
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
    double* cell(int planes) {
        double* p = dalloc<double>((size_t)L.PS * planes);
        return p ? p + L.H : nullptr;
    }
    ~caffe_diffusion() {
        if (st) cudaStreamSynchronize(st);
        for (void* p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

struct DView {
    Lat L;
    const double* vol;
    const double* cc;
    const double* S[3];
    const double* fc[3];
    const double* D[3];
    double* phi;
    double* face[3];
    double* patch[6];
    double* grad;
    int types[6];
};

DView view(caffe_diffusion* h) {
    DView v;
    v.L = h->L; v.vol = h->vol; v.cc = h->cc; v.phi = h->phi; v.grad = h->grad;
    for (int q = 0; q < 3; ++q) { v.S[q] = h->S[q]; v.fc[q] = h->fc[q]; v.D[q] = h->D[q]; v.face[q] = h->face[q]; }
    for (int f = 0; f < 6; ++f) { v.patch[f] = h->patch[f]; v.types[f] = h->types[f]; }
    return v;
}

// index of boundary element (i, j, k) in patch f: east / west k*nJ + j, north / south k*nI + i, top / bottom j*nI + i
__device__ __forceinline__ long long pidx(const Lat& L, int f, int i, int j, int k) {
    return f < 2 ? (long long)k * L.nJ + j : (f < 4 ? (long long)k * L.nI + i : (long long)j * L.nI + i);
}

// Diffusion.cpp:73-98 with setImplicit folding; coefficients of neighbours outside the block stored as zero
__global__ void diff_assemble_kernel(DView v, double* a0, double* a1, double* a2, double* a3, double* a4, double* a5, double* a6,
                                     double* b, double dt, int unsteady) {
    const Lat& L = v.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    double a[7];
    a[1] = v.D[0][L.fiI(i + 1, j, k)];
    a[2] = v.D[0][L.fiI(i, j, k)];
    a[3] = v.D[1][L.fiJ(i, j + 1, k)];
    a[4] = v.D[1][L.fiJ(i, j, k)];
    a[5] = v.D[2][L.fiK(i, j, k + 1)];
    a[6] = v.D[2][L.fiK(i, j, k)];
    const double a0P = unsteady ? v.vol[c] / dt : 0.;
    a[0] = -(a[1] + a[2] + a[3] + a[4] + a[5] + a[6]) + a0P;
    double bb = a0P * v.phi[c];
    const bool atB[6] = {i == L.nI - 1, i == 0, j == L.nJ - 1, j == 0, k == L.nK - 1, k == 0};
    for (int f = 0; f < 6; ++f) {
        if (!atB[f]) continue;
        if (v.types[f] == P_FIXED) bb -= a[f + 1] * v.patch[f][pidx(L, f, i, j, k)];
        else { a[0] += a[f + 1]; a[f + 1] = 0.; }
    }
    a0[c] = a[0];
    a1[c] = atB[0] ? 0. : a[1];
    a2[c] = atB[1] ? 0. : a[2];
    a3[c] = atB[2] ? 0. : a[3];
    a4[c] = atB[3] ? 0. : a[4];
    a5[c] = atB[4] ? 0. : a[5];
    a6[c] = atB[5] ? 0. : a[6];
    b[c] = bb;
}

// phi = x; zero-gradient / empty patches take the boundary cell's value and the boundary faces the
// patch's (PrimitiveBoundaryCondition::setBoundaries, Field.tpp:518-558)
__global__ void diff_cells_kernel(DView v, const double* x) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < v.L.N) v.phi[c] = x[c];
}
__global__ void diff_patches_kernel(DView v) {
    const Lat& L = v.L;
    const long long nIJ = (long long)L.nI * L.nJ, nJK = (long long)L.nJ * L.nK, nIK = (long long)L.nI * L.nK;
    long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long cnt[6] = {nJK, nJK, nIK, nIK, nIJ, nIJ};
    int f = 0;
    while (f < 6 && e >= cnt[f]) { e -= cnt[f]; ++f; }
    if (f >= 6 || v.types[f] == P_FIXED) return;
    int i, j, k;
    if (f < 2) { j = (int)(e % L.nJ); k = (int)(e / L.nJ); i = f == 0 ? L.nI - 1 : 0; }
    else if (f < 4) { i = (int)(e % L.nI); k = (int)(e / L.nI); j = f == 2 ? L.nJ - 1 : 0; }
    else { i = (int)(e % L.nI); j = (int)(e / L.nI); k = f == 4 ? L.nK - 1 : 0; }
    const double val = v.phi[L.cid(i, j, k)];
    v.patch[f][e] = val;
    if (f < 2) v.face[0][L.fiI(f == 0 ? L.nI : 0, j, k)] = val;
    else if (f < 4) v.face[1][L.fiJ(i, f == 2 ? L.nJ : 0, k)] = val;
    else v.face[2][L.fiK(i, j, f == 4 ? L.nK : 0)] = val;
}

// FvScheme::interpolateInteriorFaces, volume-weighted (FvScheme.tpp:12-40): each cell writes its
// east, north and top interior faces
__global__ void diff_interp_kernel(DView v) {
    const Lat& L = v.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    const double p = v.phi[c], V = v.vol[c];
    if (i < L.nI - 1) { double g = v.vol[c + 1] / (v.vol[c + 1] + V); v.face[0][L.fiI(i + 1, j, k)] = g * p + (1. - g) * v.phi[c + 1]; }
    if (j < L.nJ - 1) { double g = v.vol[c + L.nI] / (v.vol[c + L.nI] + V); v.face[1][L.fiJ(i, j + 1, k)] = g * p + (1. - g) * v.phi[c + L.nI]; }
    if (k < L.nK - 1) { double g = v.vol[c + L.nIJ] / (v.vol[c + L.nIJ] + V); v.face[2][L.fiK(i, j, k + 1)] = g * p + (1. - g) * v.phi[c + L.nIJ]; }
}

// divergence-theorem cell gradient (FvScalarScheme.cpp:48-66): sum_f phi_f S_f (outward), times 1/V
__global__ void diff_grad_kernel(DView v) {
    const Lat& L = v.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    const long long f[6] = {L.fiI(i + 1, j, k), L.fiI(i, j, k), L.fiJ(i, j + 1, k), L.fiJ(i, j, k), L.fiK(i, j, k + 1), L.fiK(i, j, k)};
    const long long nF[3] = {L.nFI, L.nFJ, L.nFK};
    double s[3] = {0., 0., 0.};
    for (int q = 0; q < 6; ++q) {
        const int dir = q >> 1;
        const double sg = (q & 1) ? -1. : 1.;
        const double val = v.face[dir][f[q]];
        const double* Sd = v.S[dir];
        double t0 = val * (sg * Sd[f[q]]), t1 = val * (sg * Sd[f[q] + nF[dir]]), t2 = val * (sg * Sd[f[q] + 2 * nF[dir]]);
        if (q == 0) { s[0] = t0; s[1] = t1; s[2] = t2; }
        else { s[0] = s[0] + t0; s[1] = s[1] + t1; s[2] = s[2] + t2; }
    }
    const double r = 1. / v.vol[c];
    v.grad[c] = s[0] * r;
    v.grad[c + L.PS] = s[1] * r;
    v.grad[c + 2 * L.PS] = s[2] * r;
}

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

// value of phi at a cell, or the patch beyond the block (Field::operator(), Field.tpp:89-128)
__device__ __forceinline__ double phi_at(const DView& v, int i, int j, int k) {
    const Lat& L = v.L;
    if (i >= L.nI) return v.patch[0][(long long)k * L.nJ + j];
    if (i < 0) return v.patch[1][(long long)k * L.nJ + j];
    if (j >= L.nJ) return v.patch[2][(long long)k * L.nI + i];
    if (j < 0) return v.patch[3][(long long)k * L.nI + i];
    if (k >= L.nK) return v.patch[4][(long long)j * L.nI + i];
    if (k < 0) return v.patch[5][(long long)j * L.nI + i];
    return v.phi[L.cid(i, j, k)];
}

// interior faces from both cells' gradients (cell-to-face vectors = face centroid - cell centroid),
// clamped to [min, max] of the lower cell and its six neighbours (FvScalarScheme.cpp:70-156)
__global__ void diff_extrap_kernel(DView v) {
    const Lat& L = v.L;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    const double p = v.phi[c];
    auto gdot = [&](long long cell, const double* fcd, long long nF, long long fi) {
        const double rx = fcd[fi] - v.cc[cell], ry = fcd[fi + nF] - v.cc[cell + L.PS], rz = fcd[fi + 2 * nF] - v.cc[cell + 2 * L.PS];
        return v.grad[cell] * rx + v.grad[cell + L.PS] * ry + v.grad[cell + 2 * L.PS] * rz;
    };
    double fE = 0., fN = 0., fT = 0.;
    const bool lE = i < L.nI - 1, lN = j < L.nJ - 1, lT = k < L.nK - 1;
    if (lE) { long long f = L.fiI(i + 1, j, k); fE = 0.5 * (p + gdot(c, v.fc[0], L.nFI, f) + v.phi[c + 1] + gdot(c + 1, v.fc[0], L.nFI, f)); }
    if (lN) { long long f = L.fiJ(i, j + 1, k); fN = 0.5 * (p + gdot(c, v.fc[1], L.nFJ, f) + v.phi[c + L.nI] + gdot(c + L.nI, v.fc[1], L.nFJ, f)); }
    if (lT) { long long f = L.fiK(i, j, k + 1); fT = 0.5 * (p + gdot(c, v.fc[2], L.nFK, f) + v.phi[c + L.nIJ] + gdot(c + L.nIJ, v.fc[2], L.nFK, f)); }
    double hi = p, lo = p;
    const double nb[6] = {phi_at(v, i + 1, j, k), phi_at(v, i - 1, j, k), phi_at(v, i, j + 1, k),
                          phi_at(v, i, j - 1, k), phi_at(v, i, j, k + 1), phi_at(v, i, j, k - 1)};
    for (int q = 0; q < 6; ++q) { hi = dmax(hi, nb[q]); lo = dmin(lo, nb[q]); }
    if (lE) v.face[0][L.fiI(i + 1, j, k)] = dmax(dmin(hi, fE), lo);
    if (lN) v.face[1][L.fiJ(i, j + 1, k)] = dmax(dmin(hi, fN), lo);
    if (lT) v.face[2][L.fiK(i, j, k + 1)] = dmax(dmin(hi, fT), lo);
}

// max_c |(A x - b)_c|: block maxima, then one atomicMax on the bits (non-negative doubles order as integers)
__global__ void __launch_bounds__(256) diff_residual_kernel(Lat L, const double* a0, const double* a1, const double* a2, const double* a3,
                                                            const double* a4, const double* a5, const double* a6, const double* x,
                                                            const double* b, unsigned long long* out) {
    __shared__ double sm[256];
    double m = 0.;
    for (long long c = blockIdx.x * 256ll + threadIdx.x; c < L.N; c += (long long)gridDim.x * 256) {
        double y = a0[c] * x[c] + a1[c] * x[c + 1] + a2[c] * x[c - 1] + a3[c] * x[c + L.nI] + a4[c] * x[c - L.nI] +
                   a5[c] * x[c + L.nIJ] + a6[c] * x[c - L.nIJ];
        double r = fabs(y - b[c]);
        m = m < r ? r : m;
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sm[threadIdx.x] = sm[threadIdx.x] < sm[threadIdx.x + w] ? sm[threadIdx.x + w] : sm[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(sm[0]));
}

int launch_assemble(caffe_diffusion* h, double dt) {
    diff_assemble_kernel<<<grid_for(h->L.N, 256), 256, 0, h->st>>>(view(h), h->a[0], h->a[1], h->a[2], h->a[3], h->a[4], h->a[5], h->a[6],
                                                                   h->b, dt, h->unsteady);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_solve(caffe_diffusion* h) {
    Op7 A;
    for (int q = 0; q < 7; ++q) A.a[q] = h->a[q];
    A.nI = h->L.nI; A.nIJ = h->L.nIJ;
    A.gh.n = 0; A.gh.cell = nullptr; A.gh.col = nullptr; A.gh.val = nullptr; A.gh.bits = nullptr;
    if (h->method == CAFFE_KSP_CG_JACOBI) return ksp_cg7(A, h->b, h->x, h->L, h->kw, h->rtol, h->maxit, h->st);
    return ksp_bicgstab(A, 1, h->b, h->x, h->L, h->kw, h->rtol, h->maxit, h->st);
}

int launch_post(caffe_diffusion* h) {
    const Lat& L = h->L;
    DView v = view(h);
    const long long nb = 2 * ((long long)L.nJ * L.nK + (long long)L.nI * L.nK + (long long)L.nI * L.nJ);
    diff_cells_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v, h->x);
    diff_patches_kernel<<<grid_for(nb, 256), 256, 0, h->st>>>(v);
    diff_interp_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v);
    diff_grad_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v);
    diff_extrap_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v);
    diff_grad_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v);
    CB_CUDA(cudaMemsetAsync(h->resMax, 0, sizeof(double), h->st));
    int blocks = (int)std::min<long long>(1024, (L.N + 255) / 256);
    diff_residual_kernel<<<blocks, 256, 0, h->st>>>(L, h->a[0], h->a[1], h->a[2], h->a[3], h->a[4], h->a[5], h->a[6], h->x, h->b,
                                                    reinterpret_cast<unsigned long long*>(h->resMax));
    CB_CHECK_LAUNCH();
    return 0;
}

int read_ksp(caffe_diffusion* h) {
    KspOut o;
    CB_CUDA(cudaMemcpyAsync(&o, h->kw.out, sizeof(KspOut), cudaMemcpyDeviceToHost, h->st));
    CB_CUDA(cudaStreamSynchronize(h->st));
    h->iters = o.iters[0];
    h->relres = o.relres[0];
    return 0;
}

}  // namespace

extern "C" {

int caffe_diffusion_create(const double* nodes, int nNI, int nNJ, int nNK, const int* bc_type, const double* ref_val, int time_accurate,
                           double phi0, int method, double rtol, int maxit, int device, caffe_diffusion** out) {
    clear_error();
    if (!out) { set_error("out is NULL"); return 1; }
    *out = nullptr;
    if (!nodes || !bc_type || !ref_val) { set_error("NULL argument"); return 1; }
    if (nNI < 2 || nNJ < 2 || nNK < 2) { set_error("a mesh needs at least 2 nodes per direction"); return 1; }
    for (int f = 0; f < 6; ++f)
        if (bc_type[f] < P_FIXED || bc_type[f] > P_EMPTY) { set_error("invalid boundary type on face " + std::to_string(f)); return 1; }
    if (method == CAFFE_KSP_BICGSTAB_SGS) {
        set_error("BiCGStab with symmetric Gauss-Seidel (the reference's PETSc PCSOR) is a sequential sweep and is not implemented "
                  "on the device: choose CAFFE_KSP_BICGSTAB_JACOBI or CAFFE_KSP_CG_JACOBI");
        return 1;
    }
    if (method != CAFFE_KSP_BICGSTAB_JACOBI && method != CAFFE_KSP_CG_JACOBI) { set_error("invalid Krylov method"); return 1; }
    if (maxit < 1 || !(rtol >= 0.)) { set_error("invalid solver tolerances"); return 1; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device available"); return 1; }
    if (device < 0 || device >= ndev) { set_error("device ordinal out of range"); return 1; }
    CB_CUDA(cudaSetDevice(device));
    caffe_diffusion* h = new caffe_diffusion();
    auto fail = [&]() { delete h; return 1; };
    h->device = device;
    h->L = make_lat(nNI - 1, nNJ - 1, nNK - 1);
    const Lat& L = h->L;
    for (int f = 0; f < 6; ++f) { h->types[f] = bc_type[f]; h->refs[f] = ref_val[f]; }
    h->unsteady = time_accurate ? 1 : 0; h->method = method; h->rtol = rtol; h->maxit = maxit;
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { set_error("stream creation failed"); return fail(); }
    const long long nf[3] = {L.nFI, L.nFJ, L.nFK};
    h->vol = h->cell(1); h->cc = h->cell(3);
    for (int q = 0; q < 3; ++q) { h->S[q] = h->dalloc<double>(3 * nf[q]); h->fc[q] = h->dalloc<double>(3 * nf[q]); h->D[q] = h->dalloc<double>(nf[q]);
                                  h->face[q] = h->dalloc<double>(nf[q]); }
    h->patchN[0] = h->patchN[1] = (long long)L.nJ * L.nK;
    h->patchN[2] = h->patchN[3] = (long long)L.nI * L.nK;
    h->patchN[4] = h->patchN[5] = (long long)L.nI * L.nJ;
    for (int f = 0; f < 6; ++f) h->patch[f] = h->dalloc<double>(h->patchN[f]);
    h->phi = h->cell(1); h->grad = h->cell(3);
    for (int q = 0; q < 7; ++q) h->a[q] = h->cell(1);
    h->b = h->cell(1); h->x = h->cell(1);
    h->resMax = h->dalloc<double>(1);
    std::memset(&h->kw, 0, sizeof(h->kw));
    h->kw.r = h->cell(2); h->kw.rp = h->cell(1);
    h->kw.p[0] = h->cell(1); h->kw.p[1] = h->cell(1); h->kw.v[0] = h->cell(1); h->kw.v[1] = h->cell(1);
    h->kw.t = h->cell(1); h->kw.invD = h->cell(1);
    h->kw.partials = h->dalloc<double>((size_t)2 * 8 * 8 * 1024);
    h->kw.out = h->dalloc<KspOut>(1);
    for (void* p : h->allocs)
        if (!p) { set_error("device allocation failed"); return fail(); }
    bool ok = h->vol && h->cc && h->phi && h->grad && h->b && h->x && h->resMax && h->kw.r && h->kw.rp && h->kw.p[0] && h->kw.p[1] &&
              h->kw.v[0] && h->kw.v[1] && h->kw.t && h->kw.invD && h->kw.partials && h->kw.out;
    for (int q = 0; q < 7; ++q) ok = ok && h->a[q];
    if (!ok) { set_error("device allocation failed"); return fail(); }
    // metrics from the nodes
    size_t nn = (size_t)nNI * nNJ * nNK * 3;
    double* dxyz = nullptr;
    if (cudaMalloc(&dxyz, nn * sizeof(double)) != cudaSuccess) { set_error("node upload allocation failed"); return fail(); }
    double* cvNone[3] = {nullptr, nullptr, nullptr};
    int rc = cudaMemcpyAsync(dxyz, nodes, nn * sizeof(double), cudaMemcpyHostToDevice, h->st) != cudaSuccess;
    if (!rc) rc = compute_metrics(L, dxyz, h->vol, h->cc, h->S, h->fc, h->D, cvNone, h->st);
    cudaStreamSynchronize(h->st);
    cudaFree(dxyz);
    if (rc) { set_error("metric computation failed"); return fail(); }
    // Diffusion::Diffusion: every patch and boundary face at its face's reference value
    // (PrimitiveBoundaryCondition(input, field) -> setFixedBoundaries), then phi = phi0
    for (int f = 0; f < 6; ++f) {
        std::vector<double> pv((size_t)h->patchN[f], ref_val[f]);
        if (cudaMemcpy(h->patch[f], pv.data(), pv.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("patch upload failed");
            return fail();
        }
    }
    std::vector<double> fI(L.nFI), fJ(L.nFJ), fK(L.nFK);
    for (int k = 0; k < L.nK; ++k)
        for (int j = 0; j < L.nJ; ++j) { fI[L.fiI(L.nI, j, k)] = ref_val[0]; fI[L.fiI(0, j, k)] = ref_val[1]; }
    for (int k = 0; k < L.nK; ++k)
        for (int i = 0; i < L.nI; ++i) { fJ[L.fiJ(i, L.nJ, k)] = ref_val[2]; fJ[L.fiJ(i, 0, k)] = ref_val[3]; }
    for (int j = 0; j < L.nJ; ++j)
        for (int i = 0; i < L.nI; ++i) { fK[L.fiK(i, j, L.nK)] = ref_val[4]; fK[L.fiK(i, j, 0)] = ref_val[5]; }
    std::vector<double> ph((size_t)L.N, phi0);
    if (cudaMemcpy(h->face[0], fI.data(), fI.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->face[1], fJ.data(), fJ.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->face[2], fK.data(), fK.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->phi, ph.data(), ph.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("initial upload failed");
        return fail();
    }
    *out = h;
    return 0;
}

int caffe_diffusion_destroy(caffe_diffusion* h) {
    if (!h) return 0;
    cudaSetDevice(h->device);
    delete h;
    return 0;
}

int caffe_diffusion_phase(caffe_diffusion* h, const char* name, double dt) {
    clear_error();
    if (!h || !name) { set_error("NULL argument"); return 1; }
    if (h->unsteady && !(dt > 0.)) { set_error("time step must be positive"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    std::string n(name);
    int rc;
    if (n == "assemble") rc = launch_assemble(h, dt);
    else if (n == "solve") rc = launch_solve(h) || read_ksp(h);
    else if (n == "post") rc = launch_post(h);
    else { set_error("unknown phase " + n); return 2; }
    if (rc) return rc;
    CB_CUDA(cudaStreamSynchronize(h->st));
    return 0;
}

int caffe_diffusion_solve(caffe_diffusion* h, double dt, double* residual_inf, int* iters, double* rel_res) {
    clear_error();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (h->unsteady && !(dt > 0.)) { set_error("time step must be positive"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (launch_assemble(h, dt) || launch_solve(h) || launch_post(h) || read_ksp(h)) return 1;
    double r = 0.;
    CB_CUDA(cudaMemcpy(&r, h->resMax, sizeof(double), cudaMemcpyDeviceToHost));
    if (residual_inf) *residual_inf = r;
    if (iters) *iters = h->iters;
    if (rel_res) *rel_res = h->relres;
    return 0;
}

long caffe_diffusion_array(caffe_diffusion* h, const char* name, double* host, long count, int dir) {
    clear_error();
    if (!h || !name) { set_error("NULL argument"); return -1; }
    const Lat& L = h->L;
    std::string n(name);
    double* base = nullptr;
    long long len = 0, stride = 0;
    int planes = 1;
    bool writable = false;
    if (n == "phi") { base = h->phi; len = L.N; writable = true; }
    else if (n == "x") { base = h->x; len = L.N; writable = true; }
    else if (n == "b") { base = h->b; len = L.N; }
    else if (n == "phiFaceI") { base = h->face[0]; len = L.nFI; }
    else if (n == "phiFaceJ") { base = h->face[1]; len = L.nFJ; }
    else if (n == "phiFaceK") { base = h->face[2]; len = L.nFK; }
    else if (n.size() == 9 && n.compare(0, 8, "phiPatch") == 0 && n[8] >= '0' && n[8] <= '5') { base = h->patch[n[8] - '0']; len = h->patchN[n[8] - '0']; }
    else if (n == "gradPhi") { base = h->grad; len = L.N; planes = 3; stride = L.PS; }
    else if (n == "cc") { base = h->cc; len = L.N; planes = 3; stride = L.PS; }
    else if (n == "A") { len = L.N; planes = 7; }
    else { set_error("unknown array " + n); return -1; }
    const long need = (long)(len * planes);
    if (!host) return need;
    if (count < need) { set_error("host buffer too small"); return -1; }
    if ((dir & 1) && !writable) { set_error("array is read-only: " + n); return -1; }
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->st) != cudaSuccess) { set_error("device error"); return -1; }
    if (planes == 1) {
        cudaError_t e = (dir & 1) ? cudaMemcpy(base, host, len * 8, cudaMemcpyHostToDevice) : cudaMemcpy(host, base, len * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { set_error("copy failed"); return -1; }
        return need;
    }
    // N x components, interleaved (the oracle's layout)
    std::vector<double> tmp((size_t)len);
    for (int q = 0; q < planes; ++q) {
        const double* src = n == "A" ? h->a[q] : base + q * stride;
        if (cudaMemcpy(tmp.data(), src, len * 8, cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
        for (long long c = 0; c < len; ++c) host[c * planes + q] = tmp[c];
    }
    return need;
}

}  // extern "C"
