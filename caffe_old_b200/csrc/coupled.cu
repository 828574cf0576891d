// Device path of the reference's Coupled solver (src/Solvers/Coupled.cpp:5-339): momentum and
// continuity assembled into one block system of 4 N unknowns (u_x, u_y, u_z, p, each numbered
// like the cells) and solved together.  One inner iteration is
//   assemble  momentum rows (upwind convection, diffusion, the pressure gradient through
//             volume-weighted face values: 14 entries) and continuity rows (the face velocities
//             and the Rhie-Chow pressure term: 28 entries), d = V / a_P (Coupled.cpp:54-245),
//             written straight into the values of a compressed-row matrix whose structure is
//             fixed by the mesh and built once;
//   solve     the block system on the persistent Jacobi-preconditioned Krylov kernels over the
//             compressed rows (Coupled.cpp:247-249);
//   post      u and p from the solution, the cell gradient of p, h = u + d grad p and the
//             Rhie-Chow face fluxes (Coupled.cpp:251-314).
// The reference's conventions stay as written: its face flux carries no density; p is never
// interpolated to interior faces before its divergence-theorem gradient, so those faces keep
// their initial zero; the boundary faces of grad p are never set and stay zero.  Boundary
// patches of fixed faces hold their reference values and the others their boundary cells'
// values, so every face value is formed on the fly from the cell arrays.  Built with --fmad=false
// and the operand order of the reference: everything outside the Krylov solve is bit for bit the
// CPU restatement's.
#include <climits>
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

struct caffe_coupled {
    int device = 0;
    cudaStream_t st = nullptr;
    Lat L;
    int utype[6] = {0, 0, 0, 0, 0, 0};   // PType of u and h per face
    int ptype[6] = {0, 0, 0, 0, 0, 0};   // PType of p per face
    double uref[6][3] = {};
    double pref[6] = {};
    double rho = 1., mu = 1., omega = 1., rtol = 1e-8, atol = 0.;
    int method = 1, maxit = 10000, unsteady = 0, nInner = 1;
    std::vector<void*> allocs;
    double* vol = nullptr;
    double* cc = nullptr;
    double* S[3] = {};
    double* fc[3] = {};
    double* D[3] = {};
    double* u = nullptr;    // 3 planes
    double* u0 = nullptr;   // 3 planes
    double* p = nullptr;
    double* d = nullptr;
    double* gp = nullptr;   // 3 planes
    double* h = nullptr;    // 3 planes
    double* mf[3] = {};
    int* ptr = nullptr;
    int* col = nullptr;
    int* diag = nullptr;
    double* val = nullptr;
    long long nnz = 0;
    double* b = nullptr;
    double* x = nullptr;
    double* contMax = nullptr;
    KspWork kw;
    int iters = 0, status = 0;
    double relres = 0.;

    template <class T>
    T* dalloc(size_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, count * sizeof(T) + 256) != cudaSuccess) return nullptr;
        cudaMemsetAsync(q, 0, count * sizeof(T) + 256, st);
        allocs.push_back(q);
        return static_cast<T*>(q);
    }
    double* cell(int planes) {
        double* q = dalloc<double>((size_t)L.PS * planes);
        return q ? q + L.H : nullptr;
    }
    ~caffe_coupled() {
        if (st) cudaStreamSynchronize(st);
        for (void* q : allocs) cudaFree(q);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

struct CView {
    Lat L;
    const double* vol;
    const double* S[3];
    const double* D[3];
    double* u;
    const double* u0;
    double* p;
    double* d;
    double* gp;
    double* h;
    double* mf[3];
    const int* ptr;
    double* val;
    double* b;
    int utype[6], ptype[6];
    double uref[6][3], pref[6];
    double rho, mu, omega;
};

CView view(caffe_coupled* h) {
    CView v;
    v.L = h->L; v.vol = h->vol; v.u = h->u; v.u0 = h->u0; v.p = h->p; v.d = h->d; v.gp = h->gp; v.h = h->h;
    for (int q = 0; q < 3; ++q) { v.S[q] = h->S[q]; v.D[q] = h->D[q]; v.mf[q] = h->mf[q]; }
    v.ptr = h->ptr; v.val = h->val; v.b = h->b;
    for (int f = 0; f < 6; ++f) {
        v.utype[f] = h->utype[f]; v.ptype[f] = h->ptype[f]; v.pref[f] = h->pref[f];
        for (int q = 0; q < 3; ++q) v.uref[f][q] = h->uref[f][q];
    }
    v.rho = h->rho; v.mu = h->mu; v.omega = h->omega;
    return v;
}

// std::max / std::min as the reference evaluates them (the first argument on a tie)
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

// The geometry one cell sees: for its faces E W N S T B whether a neighbour lies there, the
// offset to it, the face index in its direction's face array
struct CellFaces {
    int i, j, k;
    bool nb[6];
    long long off[6];
    long long fi[6];
};

__device__ __forceinline__ CellFaces cell_faces(const Lat& L, long long c) {
    CellFaces cf;
    L.ijk(c, cf.i, cf.j, cf.k);
    const int i = cf.i, j = cf.j, k = cf.k;
    cf.nb[0] = i < L.nI - 1; cf.nb[1] = i > 0; cf.nb[2] = j < L.nJ - 1; cf.nb[3] = j > 0; cf.nb[4] = k < L.nK - 1; cf.nb[5] = k > 0;
    cf.off[0] = 1; cf.off[1] = -1; cf.off[2] = L.nI; cf.off[3] = -L.nI; cf.off[4] = L.nIJ; cf.off[5] = -L.nIJ;
    cf.fi[0] = L.fiI(i + 1, j, k); cf.fi[1] = L.fiI(i, j, k); cf.fi[2] = L.fiJ(i, j + 1, k);
    cf.fi[3] = L.fiJ(i, j, k); cf.fi[4] = L.fiK(i, j, k + 1); cf.fi[5] = L.fiK(i, j, k);
    return cf;
}

__device__ __forceinline__ long long face_count(const Lat& L, int dir) { return dir == 0 ? L.nFI : (dir == 1 ? L.nFJ : L.nFK); }

// component q of the outward area vector of face f (HexaFvmMesh.h:79-84: S_W, S_S, S_B negated)
__device__ __forceinline__ double s_out(const CView& v, const CellFaces& cf, int f, int q) {
    const int dir = f >> 1;
    const double s = v.S[dir][cf.fi[f] + q * face_count(v.L, dir)];
    return (f & 1) ? -s : s;
}

// volume weight of face f for the cell (Mesh g: V_nb / (V_nb + V_P), 0 at the boundary)
__device__ __forceinline__ double g_of(const CView& v, const CellFaces& cf, long long c, int f) {
    if (!cf.nb[f]) return 0.;
    const double vn = v.vol[c + cf.off[f]];
    return vn / (vn + v.vol[c]);
}

// FvScheme::interpolateInteriorFaces (FvScheme.tpp:12-40): the face between lower cell lo and
// upper cell hi, written by the lower cell with its own east / north / top weight
__device__ __forceinline__ double interp(const double* fld, const double* vol, long long lo, long long hi) {
    const double g = vol[hi] / (vol[hi] + vol[lo]);
    return g * fld[lo] + (1. - g) * fld[hi];
}

// value of a cell field on face f of cell c: interior faces interpolated; boundary faces take
// `bnd` (the patch value)
__device__ __forceinline__ double face_val(const double* fld, const double* vol, const CellFaces& cf, long long c, int f, double bnd) {
    if (!cf.nb[f]) return bnd;
    const long long n = c + cf.off[f];
    return (f & 1) ? interp(fld, vol, n, c) : interp(fld, vol, c, n);
}

// Coupled.cpp:54-120: the three momentum rows of each cell and d = V / a_P
__global__ void __launch_bounds__(256) cp_momentum_kernel(CView v, double dt, int unsteady) {
    const Lat& L = v.L;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    const CellFaces cf = cell_faces(L, c);
    double Df[6], F[6];
    for (int f = 0; f < 6; ++f) {
        Df[f] = v.D[f >> 1][cf.fi[f]];
        F[f] = v.mf[f >> 1][cf.fi[f]];
    }
    const double a0P = unsteady ? v.rho * v.vol[c] / dt : 0.;
    const double mu = v.mu;
    double a[7];
    a[0] = (dmax(F[0], 0.) + mu * Df[0] - dmin(F[1], 0.) + mu * Df[1] + dmax(F[2], 0.) + mu * Df[2] - dmin(F[3], 0.) + mu * Df[3] +
            dmax(F[4], 0.) + mu * Df[4] - dmin(F[5], 0.) + mu * Df[5] + a0P) /
           v.omega;
    a[1] = dmin(F[0], 0.) - mu * Df[0];
    a[2] = -dmax(F[1], 0.) - mu * Df[1];
    a[3] = dmin(F[2], 0.) - mu * Df[2];
    a[4] = -dmax(F[3], 0.) - mu * Df[3];
    a[5] = dmin(F[4], 0.) - mu * Df[4];
    a[6] = -dmax(F[5], 0.) - mu * Df[5];
    double bu[3];
    const double sr = (1. - v.omega) * a[0];
    for (int q = 0; q < 3; ++q) {
        bu[q] = v.u0[c + q * L.PS] * a0P;
        bu[q] = bu[q] + v.u[c + q * L.PS] * sr;
    }
    // PrimitiveBoundaryCondition<Vector3D>::setImplicit (PrimitiveBoundaryCondition.tpp:145-255)
    for (int f = 0; f < 6; ++f) {
        if (cf.nb[f]) continue;
        if (v.utype[f] == P_FIXED) {
            for (int q = 0; q < 3; ++q) bu[q] = bu[q] - v.uref[f][q] * a[f + 1];
        } else {
            a[0] += a[f + 1];
            a[f + 1] = 0.;
        }
    }
    double g[6];
    for (int f = 0; f < 6; ++f) g[f] = g_of(v, cf, c, f);
    for (int q = 0; q < 3; ++q) {
        double s[6], ap[7];
        for (int f = 0; f < 6; ++f) s[f] = s_out(v, cf, f, q);
        ap[0] = g[0] * s[0] + g[1] * s[1] + g[2] * s[2] + g[3] * s[3] + g[4] * s[4] + g[5] * s[5];
        for (int f = 0; f < 6; ++f) ap[1 + f] = (1. - g[f]) * s[f];
        double bq = bu[q];
        for (int f = 0; f < 6; ++f) {
            if (cf.nb[f]) continue;
            if (v.ptype[f] == P_FIXED) bq = bq - ap[f + 1] * v.pref[f];
            else { ap[0] += ap[f + 1]; ap[f + 1] = 0.; }
        }
        const long long row = c + q * L.N;
        long long pos = v.ptr[row];
        v.val[pos++] = a[0];
        for (int f = 0; f < 6; ++f)
            if (cf.nb[f]) v.val[pos++] = a[f + 1];
        v.val[pos++] = ap[0];
        for (int f = 0; f < 6; ++f)
            if (cf.nb[f]) v.val[pos++] = ap[f + 1];
        v.b[row] = bq;
    }
    v.d[c] = v.vol[c] / a[0];
}

// Coupled.cpp:122-245: the continuity row of each cell (d on the faces: zero-gradient patches,
// interior faces volume-weighted)
__global__ void __launch_bounds__(256) cp_continuity_kernel(CView v) {
    const Lat& L = v.L;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    const CellFaces cf = cell_faces(L, c);
    const double rho = v.rho;
    double g[6];
    for (int f = 0; f < 6; ++f) g[f] = g_of(v, cf, c, f);
    long long pos = v.ptr[c + 3 * L.N];
    double bp = 0.;
    for (int q = 0; q < 3; ++q) {
        double s[6], a[7];
        for (int f = 0; f < 6; ++f) s[f] = s_out(v, cf, f, q);
        a[0] = rho * g[0] * s[0] + rho * g[1] * s[1] + rho * g[2] * s[2] + rho * g[3] * s[3] + rho * g[4] * s[4] + rho * g[5] * s[5];
        for (int f = 0; f < 6; ++f) a[1 + f] = rho * (1. - g[f]) * s[f];
        double t = 0.;
        for (int f = 0; f < 6; ++f) {
            if (cf.nb[f]) continue;
            if (v.utype[f] == P_FIXED) t = t - v.uref[f][q] * a[f + 1];
            else { a[0] += a[f + 1]; a[f + 1] = 0.; }
        }
        bp += t;
        v.val[pos++] = a[0];
        for (int f = 0; f < 6; ++f)
            if (cf.nb[f]) v.val[pos++] = a[f + 1];
    }
    // pressure part: the Rhie-Chow interpolation
    const double dc = v.d[c];
    double rd[6], tg[6];
    for (int f = 0; f < 6; ++f) {
        const double dF = face_val(v.d, v.vol, cf, c, f, dc);
        rd[f] = rho * dF * v.D[f >> 1][cf.fi[f]];
        double gf[3];
        for (int q = 0; q < 3; ++q) gf[q] = face_val(v.gp + q * L.PS, v.vol, cf, c, f, 0.);
        tg[f] = rho * dF * (gf[0] * s_out(v, cf, f, 0) + gf[1] * s_out(v, cf, f, 1) + gf[2] * s_out(v, cf, f, 2));
    }
    double a[7];
    a[0] = rd[0] + rd[1] + rd[2] + rd[3] + rd[4] + rd[5];
    for (int f = 0; f < 6; ++f) a[1 + f] = -rd[f];
    bp -= tg[0] + tg[1] + tg[2] + tg[3] + tg[4] + tg[5];
    for (int f = 0; f < 6; ++f) {
        if (cf.nb[f]) continue;
        if (v.ptype[f] == P_FIXED) bp = bp - a[f + 1] * v.pref[f];
        else { a[0] += a[f + 1]; a[f + 1] = 0.; }
    }
    v.val[pos++] = a[0];
    for (int f = 0; f < 6; ++f)
        if (cf.nb[f]) v.val[pos++] = a[f + 1];
    v.b[c + 3 * L.N] = bp;
}

// Coupled.cpp:251-262 per cell: u and p from the solution; grad p by the divergence theorem
// (FvScalarScheme.cpp:48-66) from p's faces, which are zero inside the block and the patch value
// on the boundary (the reference value of a fixed face, else the cell's own p); h = u + d grad p
__global__ void __launch_bounds__(256) cp_post_cells_kernel(CView v, const double* x) {
    const Lat& L = v.L;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    const CellFaces cf = cell_faces(L, c);
    double uc[3];
    for (int q = 0; q < 3; ++q) { uc[q] = x[c + q * L.N]; v.u[c + q * L.PS] = uc[q]; }
    const double pc = x[c + 3 * L.N];
    v.p[c] = pc;
    double s[3] = {0., 0., 0.};
    for (int f = 0; f < 6; ++f) {
        const double pf = cf.nb[f] ? 0. : (v.ptype[f] == P_FIXED ? v.pref[f] : pc);
        for (int q = 0; q < 3; ++q) {
            const double t = s_out(v, cf, f, q) * pf;
            s[q] = f == 0 ? t : s[q] + t;
        }
    }
    const double r = 1. / v.vol[c];
    const double dc = v.d[c];
    for (int q = 0; q < 3; ++q) {
        const double gq = s[q] * r;
        v.gp[c + q * L.PS] = gq;
        v.h[c + q * L.PS] = uc[q] + gq * dc;
    }
}

// Coupled::rhieChowInterpolateFaces (Coupled.cpp:282-314), one thread per face of direction DIR:
// F = S . h_f - d_f (p_upper - p_lower) D_f on interior and upper boundary faces,
// F = -(S_W . h_f) - d_f (p_patch - p_P) D_f on the lower boundary face (S_W = -S)
template <int DIR>
__global__ void __launch_bounds__(256) cp_flux_kernel(CView v) {
    const Lat& L = v.L;
    const long long nF = face_count(L, DIR);
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int fI = DIR == 0 ? L.nI + 1 : L.nI;
    const int fJ = DIR == 1 ? L.nJ + 1 : L.nJ;
    const int i = (int)(f % fI);
    const long long t = f / fI;
    const int j = (int)(t % fJ);
    const int k = (int)(t / fJ);
    const int idx = DIR == 0 ? i : (DIR == 1 ? j : k);
    const int n = DIR == 0 ? L.nI : (DIR == 1 ? L.nJ : L.nK);
    const long long step = DIR == 0 ? 1 : (DIR == 1 ? L.nI : L.nIJ);
    const double* Sd = v.S[DIR];
    const double S0 = Sd[f], S1 = Sd[f + nF], S2 = Sd[f + 2 * nF];
    const double Dd = v.D[DIR][f];
    double out;
    if (idx > 0 && idx < n) {
        const long long hi = L.cid(i, j, k), lo = hi - step;
        const double hf0 = interp(v.h, v.vol, lo, hi), hf1 = interp(v.h + L.PS, v.vol, lo, hi), hf2 = interp(v.h + 2 * L.PS, v.vol, lo, hi);
        const double df = interp(v.d, v.vol, lo, hi);
        out = hf0 * S0 + hf1 * S1 + hf2 * S2 - df * (v.p[hi] - v.p[lo]) * Dd;
    } else if (idx == n) {
        const int fb = 2 * DIR;   // east / north / top
        const long long lo = L.cid(i - (DIR == 0), j - (DIR == 1), k - (DIR == 2));
        const bool fx = v.utype[fb] == P_FIXED;
        const double hf0 = fx ? v.uref[fb][0] : v.h[lo], hf1 = fx ? v.uref[fb][1] : v.h[lo + L.PS], hf2 = fx ? v.uref[fb][2] : v.h[lo + 2 * L.PS];
        const double pn = v.ptype[fb] == P_FIXED ? v.pref[fb] : v.p[lo];
        out = hf0 * S0 + hf1 * S1 + hf2 * S2 - v.d[lo] * (pn - v.p[lo]) * Dd;
    } else {
        const int fb = 2 * DIR + 1;   // west / south / bottom
        const long long hi = L.cid(i, j, k);
        const bool fx = v.utype[fb] == P_FIXED;
        const double hf0 = fx ? v.uref[fb][0] : v.h[hi], hf1 = fx ? v.uref[fb][1] : v.h[hi + L.PS], hf2 = fx ? v.uref[fb][2] : v.h[hi + 2 * L.PS];
        const double pw = v.ptype[fb] == P_FIXED ? v.pref[fb] : v.p[hi];
        out = -(hf0 * -S0 + hf1 * -S1 + hf2 * -S2) - v.d[hi] * (pw - v.p[hi]) * Dd;
    }
    v.mf[DIR][f] = out;
}

// Coupled::computeContinuityError (Coupled.cpp:316-339): max_c |net face flux| / V_c, block
// maxima then one atomicMax on the bits (non-negative doubles order as integers)
__global__ void __launch_bounds__(256) cp_continuity_error_kernel(CView v, unsigned long long* out) {
    __shared__ double sm[256];
    const Lat& L = v.L;
    double m = 0.;
    for (long long c = blockIdx.x * 256ll + threadIdx.x; c < L.N; c += (long long)gridDim.x * 256) {
        const CellFaces cf = cell_faces(L, c);
        const double e = fabs(v.mf[0][cf.fi[0]] - v.mf[0][cf.fi[1]] + v.mf[1][cf.fi[2]] - v.mf[1][cf.fi[3]] + v.mf[2][cf.fi[4]] -
                              v.mf[2][cf.fi[5]]) /
                         v.vol[c];
        if (e > m) m = e;
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sm[threadIdx.x] = sm[threadIdx.x] < sm[threadIdx.x + w] ? sm[threadIdx.x + w] : sm[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(sm[0]));
}

// The fixed structure of the block system in the insertion order of the reference's rows
// (SparseMatrix::setRow with INSERT_VALUES, columns of neighbours outside the block skipped):
// momentum row of component q: u_q at P, E, W, N, S, T, B, then p at P, E, W, N, S, T, B;
// continuity row: u_x, u_y, u_z, p, each at P, E, W, N, S, T, B.
void build_structure(const Lat& L, std::vector<int>& ptr, std::vector<int>& col, std::vector<int>& diag) {
    const long long N = L.N;
    ptr.assign(4 * N + 1, 0);
    diag.assign(4 * N, -1);
    auto nbs = [&](long long c, long long* o) {
        int i, j, k, n = 0;
        L.ijk(c, i, j, k);
        if (i < L.nI - 1) o[n++] = 1;
        if (i > 0) o[n++] = -1;
        if (j < L.nJ - 1) o[n++] = L.nI;
        if (j > 0) o[n++] = -L.nI;
        if (k < L.nK - 1) o[n++] = L.nIJ;
        if (k > 0) o[n++] = -L.nIJ;
        return n;
    };
    long long total = 0;
    for (long long c = 0; c < N; ++c) {
        long long o[6];
        const int n = nbs(c, o);
        for (int q = 0; q < 3; ++q) ptr[c + q * N + 1] = 2 * (1 + n);
        ptr[c + 3 * N + 1] = 4 * (1 + n);
        total += 10 * (1 + n);
    }
    for (long long r = 0; r < 4 * N; ++r) ptr[r + 1] += ptr[r];
    col.assign(total, -1);
    for (long long c = 0; c < N; ++c) {
        long long o[6];
        const int n = nbs(c, o);
        for (int q = 0; q < 3; ++q) {
            const long long row = c + q * N;
            long long pos = ptr[row];
            diag[row] = (int)pos;
            for (int var : {q, 3}) {
                col[pos++] = (int)(c + var * N);
                for (int e = 0; e < n; ++e) col[pos++] = (int)(c + o[e] + var * N);
            }
        }
        const long long row = c + 3 * N;
        long long pos = ptr[row];
        for (int var = 0; var < 4; ++var) {
            if (var == 3) diag[row] = (int)pos;
            col[pos++] = (int)(c + var * N);
            for (int e = 0; e < n; ++e) col[pos++] = (int)(c + o[e] + var * N);
        }
    }
}

int launch_assemble(caffe_coupled* h, double dt, int part) {
    const CView v = view(h);
    const int blocks = grid_for(h->L.N, 256);
    if (part & 1) cp_momentum_kernel<<<blocks, 256, 0, h->st>>>(v, dt, h->unsteady);
    if (part & 2) cp_continuity_kernel<<<blocks, 256, 0, h->st>>>(v);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_solve(caffe_coupled* h) {
    OpCSR A;
    A.ptr = h->ptr; A.col = h->col; A.val = h->val; A.diag = h->diag;
    return ksp_csr(A, h->method, 4 * h->L.N, h->b, h->x, h->kw, h->rtol, h->maxit, h->st, h->atol);
}

int launch_post(caffe_coupled* h) {
    const Lat& L = h->L;
    const CView v = view(h);
    cp_post_cells_kernel<<<grid_for(L.N, 256), 256, 0, h->st>>>(v, h->x);
    cp_flux_kernel<0><<<grid_for(L.nFI, 256), 256, 0, h->st>>>(v);
    cp_flux_kernel<1><<<grid_for(L.nFJ, 256), 256, 0, h->st>>>(v);
    cp_flux_kernel<2><<<grid_for(L.nFK, 256), 256, 0, h->st>>>(v);
    CB_CHECK_LAUNCH();
    return 0;
}

int launch_continuity(caffe_coupled* h) {
    CB_CUDA(cudaMemsetAsync(h->contMax, 0, sizeof(double), h->st));
    const int blocks = (int)std::min<long long>(1024, (h->L.N + 255) / 256);
    cp_continuity_error_kernel<<<blocks, 256, 0, h->st>>>(view(h), reinterpret_cast<unsigned long long*>(h->contMax));
    CB_CHECK_LAUNCH();
    return 0;
}

int save_u0(caffe_coupled* h) {
    CB_CUDA(cudaMemcpyAsync(h->u0 - h->L.H, h->u - h->L.H, sizeof(double) * 3 * h->L.PS, cudaMemcpyDeviceToDevice, h->st));
    return 0;
}

int read_ksp(caffe_coupled* h) {
    KspOut o;
    CB_CUDA(cudaMemcpyAsync(&o, h->kw.out, sizeof(KspOut), cudaMemcpyDeviceToHost, h->st));
    CB_CUDA(cudaStreamSynchronize(h->st));
    h->iters = o.iters[0];
    h->relres = o.relres[0];
    h->status = o.status[0];
    return 0;
}

}  // namespace

extern "C" {

int caffe_coupled_create(const double* nodes, int nNI, int nNJ, int nNK, const caffe_case* cs, int device, caffe_coupled** out) {
    clear_error();
    if (!out) { set_error("out is NULL"); return 1; }
    *out = nullptr;
    if (!nodes || !cs) { set_error("NULL argument"); return 1; }
    if (nNI < 2 || nNJ < 2 || nNK < 2) { set_error("a mesh needs at least 2 nodes per direction"); return 1; }
    for (int f = 0; f < 6; ++f)
        if (cs->bc_type[f] < F_INLET || cs->bc_type[f] > F_ZERO_GRADIENT) { set_error("invalid boundary type on face " + std::to_string(f)); return 1; }
    if (cs->mom_method == CAFFE_KSP_BICGSTAB_SGS) {
        set_error("BiCGStab with symmetric Gauss-Seidel (the reference's PETSc PCSOR) is a sequential sweep and is not implemented "
                  "on the device: choose CAFFE_KSP_BICGSTAB_JACOBI or CAFFE_KSP_CG_JACOBI");
        return 1;
    }
    if (cs->mom_method != CAFFE_KSP_BICGSTAB_JACOBI && cs->mom_method != CAFFE_KSP_CG_JACOBI) { set_error("invalid Krylov method"); return 1; }
    if (cs->maxit < 1 || !(cs->mom_rtol >= 0.) || !(cs->mom_atol >= 0.)) { set_error("invalid solver tolerances"); return 1; }
    if (!(cs->omega_u > 0.) || !(cs->rho > 0.)) { set_error("omega_u and rho must be positive"); return 1; }
    if (cs->time_accurate && cs->n_inner < 1) { set_error("n_inner must be >= 1"); return 1; }
    const long long ncell = (long long)(nNI - 1) * (nNJ - 1) * (nNK - 1);
    if (70 * ncell >= INT_MAX) { set_error("mesh too large for 32-bit row pointers of the block system"); return 1; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { set_error("no CUDA device available"); return 1; }
    if (device < 0 || device >= ndev) { set_error("device ordinal out of range"); return 1; }
    CB_CUDA(cudaSetDevice(device));
    caffe_coupled* h = new caffe_coupled();
    auto fail = [&]() { delete h; return 1; };
    h->device = device;
    h->L = make_lat(nNI - 1, nNJ - 1, nNK - 1);
    const Lat& L = h->L;
    // Coupled::Coupled with FlowBoundaryConditions (FlowBoundaryConditions.cpp:3-73): u and h
    // fixed on inlets and walls, p fixed on outlets, empty faces empty, the rest zero-gradient
    for (int f = 0; f < 6; ++f) {
        const int t = cs->bc_type[f];
        h->utype[f] = (t == F_INLET || t == F_WALL) ? P_FIXED : (t == F_EMPTY ? P_EMPTY : P_ZERO_GRADIENT);
        h->ptype[f] = t == F_OUTLET ? P_FIXED : (t == F_EMPTY ? P_EMPTY : P_ZERO_GRADIENT);
        for (int q = 0; q < 3; ++q) h->uref[f][q] = cs->ref_vec[f][q];
        h->pref[f] = cs->ref_val[f];
    }
    h->rho = cs->rho; h->mu = cs->mu; h->omega = cs->omega_u;
    h->unsteady = cs->time_accurate ? 1 : 0;
    h->nInner = cs->time_accurate ? cs->n_inner : 1;
    h->method = cs->mom_method; h->rtol = cs->mom_rtol; h->atol = cs->mom_atol; h->maxit = cs->maxit;
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { set_error("stream creation failed"); return fail(); }
    std::vector<int> hptr, hcol, hdiag;
    build_structure(L, hptr, hcol, hdiag);
    h->nnz = (long long)hcol.size();
    const long long nf[3] = {L.nFI, L.nFJ, L.nFK};
    const long long n4 = 4 * L.N;
    h->vol = h->cell(1); h->cc = h->cell(3);
    for (int q = 0; q < 3; ++q) {
        h->S[q] = h->dalloc<double>(3 * nf[q]); h->fc[q] = h->dalloc<double>(3 * nf[q]); h->D[q] = h->dalloc<double>(nf[q]);
        h->mf[q] = h->dalloc<double>(nf[q]);
    }
    h->u = h->cell(3); h->u0 = h->cell(3); h->p = h->cell(1); h->d = h->cell(1); h->gp = h->cell(3); h->h = h->cell(3);
    h->ptr = h->dalloc<int>(n4 + 1); h->col = h->dalloc<int>(h->nnz); h->diag = h->dalloc<int>(n4); h->val = h->dalloc<double>(h->nnz);
    h->b = h->dalloc<double>(n4); h->x = h->dalloc<double>(n4);
    h->contMax = h->dalloc<double>(1);
    std::memset(&h->kw, 0, sizeof(h->kw));
    h->kw.r = h->dalloc<double>(2 * n4); h->kw.rp = h->dalloc<double>(n4);
    h->kw.p[0] = h->dalloc<double>(n4); h->kw.p[1] = h->dalloc<double>(n4);
    h->kw.v[0] = h->dalloc<double>(n4); h->kw.v[1] = h->dalloc<double>(n4);
    h->kw.t = h->dalloc<double>(n4); h->kw.invD = h->dalloc<double>(n4);
    h->kw.partials = h->dalloc<double>((size_t)2 * 8 * 8 * 1024);
    h->kw.out = h->dalloc<KspOut>(1);
    for (void* q : h->allocs)
        if (!q) { set_error("device allocation failed"); return fail(); }
    bool ok = h->vol && h->cc && h->u && h->u0 && h->p && h->d && h->gp && h->h && h->ptr && h->col && h->diag && h->val && h->b && h->x &&
              h->contMax && h->kw.r && h->kw.rp && h->kw.p[0] && h->kw.p[1] && h->kw.v[0] && h->kw.v[1] && h->kw.t && h->kw.invD &&
              h->kw.partials && h->kw.out;
    for (int q = 0; q < 3; ++q) ok = ok && h->S[q] && h->fc[q] && h->D[q] && h->mf[q];
    if (!ok) { set_error("device allocation failed"); return fail(); }
    if (cudaMemcpyAsync(h->ptr, hptr.data(), sizeof(int) * hptr.size(), cudaMemcpyHostToDevice, h->st) != cudaSuccess ||
        cudaMemcpyAsync(h->col, hcol.data(), sizeof(int) * hcol.size(), cudaMemcpyHostToDevice, h->st) != cudaSuccess ||
        cudaMemcpyAsync(h->diag, hdiag.data(), sizeof(int) * hdiag.size(), cudaMemcpyHostToDevice, h->st) != cudaSuccess) {
        set_error("structure upload failed");
        return fail();
    }
    const size_t nn = (size_t)nNI * nNJ * nNK * 3;
    double* dxyz = nullptr;
    if (cudaMalloc(&dxyz, nn * sizeof(double)) != cudaSuccess) { set_error("node upload allocation failed"); return fail(); }
    double* cvNone[3] = {nullptr, nullptr, nullptr};
    int rc = cudaMemcpyAsync(dxyz, nodes, nn * sizeof(double), cudaMemcpyHostToDevice, h->st) != cudaSuccess;
    if (!rc) rc = compute_metrics(L, dxyz, h->vol, h->cc, h->S, h->fc, h->D, cvNone, h->st);
    if (cudaStreamSynchronize(h->st) != cudaSuccess) rc = 1;
    cudaFree(dxyz);
    if (rc) { set_error("metric computation failed"); return fail(); }
    *out = h;
    return 0;
}

int caffe_coupled_destroy(caffe_coupled* h) {
    if (!h) return 0;
    cudaSetDevice(h->device);
    delete h;
    return 0;
}

int caffe_coupled_phase(caffe_coupled* h, const char* name, double dt) {
    clear_error();
    if (!h || !name) { set_error("NULL argument"); return 1; }
    if (h->unsteady && !(dt > 0.)) { set_error("time step must be positive"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    const std::string n(name);
    int rc;
    if (n == "save_u0") rc = save_u0(h);
    else if (n == "assemble") rc = launch_assemble(h, dt, 3);
    else if (n == "assemble_momentum") rc = launch_assemble(h, dt, 1);
    else if (n == "assemble_continuity") rc = launch_assemble(h, dt, 2);
    else if (n == "solve") rc = launch_solve(h) || read_ksp(h);
    else if (n == "post") rc = launch_post(h);
    else if (n == "continuity") rc = launch_continuity(h);
    else { set_error("unknown phase " + n); return 2; }
    if (rc) return rc;
    CB_CUDA(cudaStreamSynchronize(h->st));
    return 0;
}

int caffe_coupled_solve(caffe_coupled* h, double dt, double* continuity) {
    clear_error();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (h->unsteady && !(dt > 0.)) { set_error("time step must be positive"); return 1; }
    CB_CUDA(cudaSetDevice(h->device));
    if (save_u0(h)) return 1;
    for (int it = 0; it < h->nInner; ++it)
        if (launch_assemble(h, dt, 3) || launch_solve(h) || launch_post(h)) return 1;
    if (launch_continuity(h) || read_ksp(h)) return 1;
    double r = 0.;
    CB_CUDA(cudaMemcpy(&r, h->contMax, sizeof(double), cudaMemcpyDeviceToHost));
    if (continuity) *continuity = r;
    return 0;
}

int caffe_coupled_stats(caffe_coupled* h, int* iters, double* rel_res, int* status) {
    clear_error();
    if (!h) { set_error("handle is NULL"); return 1; }
    if (iters) *iters = h->iters;
    if (rel_res) *rel_res = h->relres;
    if (status) *status = h->status;
    return 0;
}

long long caffe_coupled_system(caffe_coupled* h, int* row_ptr, int* col, double* val) {
    clear_error();
    if (!h) { set_error("handle is NULL"); return -1; }
    if (!row_ptr && !col && !val) return h->nnz;
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->st) != cudaSuccess) { set_error("device error"); return -1; }
    const long long n4 = 4 * h->L.N;
    if ((row_ptr && cudaMemcpy(row_ptr, h->ptr, sizeof(int) * (n4 + 1), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (col && cudaMemcpy(col, h->col, sizeof(int) * h->nnz, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (val && cudaMemcpy(val, h->val, sizeof(double) * h->nnz, cudaMemcpyDeviceToHost) != cudaSuccess)) {
        set_error("copy failed");
        return -1;
    }
    return h->nnz;
}

long caffe_coupled_array(caffe_coupled* h, const char* name, double* host, long count, int dir) {
    clear_error();
    if (!h || !name) { set_error("NULL argument"); return -1; }
    const Lat& L = h->L;
    const std::string n(name);
    double* base = nullptr;
    long long len = 0;
    int planes = 1;
    bool writable = false;
    if (n == "u") { base = h->u; len = L.N; planes = 3; writable = true; }
    else if (n == "u0") { base = h->u0; len = L.N; planes = 3; writable = true; }
    else if (n == "p") { base = h->p; len = L.N; writable = true; }
    else if (n == "d") { base = h->d; len = L.N; }
    else if (n == "gradP") { base = h->gp; len = L.N; planes = 3; writable = true; }
    else if (n == "h") { base = h->h; len = L.N; planes = 3; }
    else if (n == "massFlowI") { base = h->mf[0]; len = L.nFI; writable = true; }
    else if (n == "massFlowJ") { base = h->mf[1]; len = L.nFJ; writable = true; }
    else if (n == "massFlowK") { base = h->mf[2]; len = L.nFK; writable = true; }
    else if (n == "b") { base = h->b; len = 4 * L.N; }
    else if (n == "x") { base = h->x; len = 4 * L.N; writable = true; }
    else { set_error("unknown array " + n); return -1; }
    const long need = (long)(len * planes);
    if (!host) return need;
    if (count < need) { set_error("host buffer too small"); return -1; }
    if ((dir & 1) && !writable) { set_error("array is read-only: " + n); return -1; }
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamSynchronize(h->st) != cudaSuccess) { set_error("device error"); return -1; }
    if (planes == 1) {
        const cudaError_t e = (dir & 1) ? cudaMemcpy(base, host, len * 8, cudaMemcpyHostToDevice) : cudaMemcpy(host, base, len * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { set_error("copy failed"); return -1; }
        return need;
    }
    // N x 3, interleaved (the oracle's layout)
    std::vector<double> tmp((size_t)len);
    for (int q = 0; q < planes; ++q) {
        double* plane = base + q * L.PS;
        if (dir & 1) {
            for (long long c = 0; c < len; ++c) tmp[c] = host[c * planes + q];
            if (cudaMemcpy(plane, tmp.data(), len * 8, cudaMemcpyHostToDevice) != cudaSuccess) { set_error("copy failed"); return -1; }
        } else {
            if (cudaMemcpy(tmp.data(), plane, len * 8, cudaMemcpyDeviceToHost) != cudaSuccess) { set_error("copy failed"); return -1; }
            for (long long c = 0; c < len; ++c) host[c * planes + q] = tmp[c];
        }
    }
    return need;
}

}  // extern "C"
