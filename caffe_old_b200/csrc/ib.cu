// Immersed-boundary ghost-cell method on the device (IbPiso.cpp:65-190).
//
// The reference classifies cells against the sphere, flags ghost cells and rebuilds the
// ghost rows (with an O(N) point location per ghost) at every time step and inner
// iteration.  Geometry is static, so those rows are identical every time: here they are
// built once, on the device, when the handle is created --
//   * one pass classifies cells (centroid inside the sphere -> solid/inactive),
//   * one pass flags ghosts (solid with a fluid 6-neighbour; outside the domain counts
//     as fluid, the default of IbPiso's AUXILLARY field patches),
//   * ghost cells are compacted in k-j-i order (per-1024-cell chunk counts, one scan),
//   * one thread per ghost finds the image point, locates its enclosing cell-centre
//     hexahedron in a window around the ghost (the reference scans the whole mesh; in a
//     valid mesh only cells next to the first hit can also contain the point, so the
//     first hit in k-j-i order is the same) and solves the 8x8 trilinear system,
// and per step only the solid-cell reset u = p = 0 is repeated.
// Compiled with --fmad=false: the stencil weights are bit-identical to the CPU oracle's.
#include <vector>
#include "ib.cuh"

namespace cb {

namespace {

struct v3 { double x, y, z; };
__device__ __forceinline__ v3 V(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 mul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 u, v3 v) { return V(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
__device__ __forceinline__ double mag(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ v3 unitv(v3 a) { double inv = 1. / mag(a); return V(inv * a.x, inv * a.y, inv * a.z); }

__device__ __forceinline__ v3 quadCentroid(v3 p0, v3 p1, v3 p2, v3 p3) {  // Geometry.cpp:14-20
    v3 d1 = add(p0, mul(sub(p2, p0), 0.5));
    v3 d2 = add(p1, mul(sub(p3, p1), 0.5));
    return add(d1, mul(sub(d2, d1), 0.5));
}
__device__ __forceinline__ v3 quadNormal(v3 p0, v3 p1, v3 p2) {  // Geometry.cpp:22-25 as written
    v3 a = cross(sub(p1, p0), sub(p2, p0));
    v3 b = cross(sub(p1, p0), sub(p2, p0));
    return mul(add(a, b), 0.5);
}
__device__ bool insideHex(v3 pt, const v3* p) {  // Geometry.cpp:178-256
    const int fv[6][4] = {{1, 2, 6, 5}, {0, 4, 7, 3}, {2, 3, 7, 6}, {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1}};
    for (int f = 0; f < 6; ++f) {
        v3 xc = quadCentroid(p[fv[f][0]], p[fv[f][1]], p[fv[f][2]], p[fv[f][3]]);
        v3 n = quadNormal(p[fv[f][0]], p[fv[f][1]], p[fv[f][2]]);
        if (dot(sub(xc, pt), n) < 0.) return false;
    }
    return true;
}

__device__ __forceinline__ v3 nodeAt(const double* xyz, const Lat& L, int i, int j, int k) {
    long long q = ((long long)k * (L.nJ + 1) + j) * (L.nI + 1) + i;
    return V(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]);
}
__device__ __forceinline__ v3 ccAt(const Geo& g, long long c) { return V(g.cc[c], g.cc[c + g.L.PS], g.cc[c + 2 * g.L.PS]); }

__device__ void nodeHex(const double* xyz, const Lat& L, int i, int j, int k, v3* p) {
    p[0] = nodeAt(xyz, L, i, j, k); p[1] = nodeAt(xyz, L, i + 1, j, k); p[2] = nodeAt(xyz, L, i + 1, j + 1, k);
    p[3] = nodeAt(xyz, L, i, j + 1, k); p[4] = nodeAt(xyz, L, i, j, k + 1); p[5] = nodeAt(xyz, L, i + 1, j, k + 1);
    p[6] = nodeAt(xyz, L, i + 1, j + 1, k + 1); p[7] = nodeAt(xyz, L, i, j + 1, k + 1);
}

// HexaFvmMesh::locateCell (HexaFvmMesh.cpp:345-376): first cell in k-j-i order containing pt.
__device__ bool locateCell(const double* xyz, const Lat& L, v3 pt, int hi, int hj, int hk, int& ri, int& rj, int& rk) {
    const int w = 5;
    int k0 = max(0, hk - w), k1 = min(L.nK - 1, hk + w);
    int j0 = max(0, hj - w), j1 = min(L.nJ - 1, hj + w);
    int i0 = max(0, hi - w), i1 = min(L.nI - 1, hi + w);
    v3 p[8];
    bool found = false;
    for (int k = k0; k <= k1 && !found; ++k)
        for (int j = j0; j <= j1 && !found; ++j)
            for (int i = i0; i <= i1 && !found; ++i) {
                nodeHex(xyz, L, i, j, k, p);
                if (insideHex(pt, p)) { ri = i; rj = j; rk = k; found = true; }
            }
    if (!found) return false;
    int bi = ri, bj = rj, bk = rk;
    for (int k = max(0, bk - 1); k <= min(L.nK - 1, bk + 1); ++k)
        for (int j = max(0, bj - 1); j <= min(L.nJ - 1, bj + 1); ++j)
            for (int i = max(0, bi - 1); i <= min(L.nI - 1, bi + 1); ++i) {
                if (L.cid(i, j, k) >= L.cid(ri, rj, rk)) continue;
                nodeHex(xyz, L, i, j, k, p);
                if (insideHex(pt, p)) { ri = i; rj = j; rk = k; }
            }
    return true;
}

// Interpolation::computeTrilinearCoeffs (Interpolation.cpp:135-180): solve M^T beta = m(x_IP)
// by Gaussian elimination with partial pivoting (the reference inverts M with LAPACK).
__device__ void trilinear(const v3* pts, v3 ip, double* beta) {
    double A[8][9];
    double mrow[8][8];
    for (int i = 0; i < 8; ++i) {
        double x = pts[i].x, y = pts[i].y, z = pts[i].z;
        mrow[i][0] = 1.; mrow[i][1] = x * y * z; mrow[i][2] = x * y; mrow[i][3] = y * z;
        mrow[i][4] = x * z; mrow[i][5] = x; mrow[i][6] = y; mrow[i][7] = z;
    }
    double x = ip.x, y = ip.y, z = ip.z;
    double rhs[8] = {1., x * y * z, x * y, y * z, x * z, x, y, z};
    for (int r = 0; r < 8; ++r) {
        for (int c = 0; c < 8; ++c) A[r][c] = mrow[c][r];
        A[r][8] = rhs[r];
    }
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        double best = fabs(A[c][c]);
        for (int r = c + 1; r < 8; ++r)
            if (fabs(A[r][c]) > best) { best = fabs(A[r][c]); piv = r; }
        if (piv != c)
            for (int q = 0; q < 9; ++q) { double t = A[c][q]; A[c][q] = A[piv][q]; A[piv][q] = t; }
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

__global__ void classify_kernel(Geo g, double cx, double cy, double cz, double R, uint8_t* fld) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= g.L.N) return;
    v3 x = ccAt(g, c);
    fld[c] = mag(sub(x, V(cx, cy, cz))) <= R ? 2 : 0;   // Sphere::isInside, Sphere.cpp:49-55
}

__global__ void ghost_flag_kernel(Lat L, const uint8_t* fld, uint8_t* status, int* chunkCount, int* nInactive) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int st = ST_ACTIVE;
    if (c < L.N && fld[c] == 2) {
        int i, j, k;
        L.ijk(c, i, j, k);
        auto fluid = [&](int a, int b, int d) {
            if (a < 0 || b < 0 || d < 0 || a >= L.nI || b >= L.nJ || d >= L.nK) return true;
            return fld[L.cid(a, b, d)] == 0;
        };
        bool g = fluid(i + 1, j, k) || fluid(i - 1, j, k) || fluid(i, j + 1, k) || fluid(i, j - 1, k) || fluid(i, j, k + 1) || fluid(i, j, k - 1);
        st = g ? ST_GHOST : ST_INACTIVE;
    }
    if (c < L.N) status[c] = (uint8_t)st;
    int isG = st == ST_GHOST, isI = st == ST_INACTIVE;
    int cnt = __syncthreads_count(isG);
    int ina = __syncthreads_count(isI);
    if (threadIdx.x == 0) {
        chunkCount[blockIdx.x] = cnt;
        if (ina) atomicAdd(nInactive, ina);
    }
}

__global__ void ghost_list_kernel(Lat L, const uint8_t* status, const int* chunkOffset, int* gCell, uint32_t* bits) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool isG = c < L.N && status[c] == ST_GHOST;
    unsigned m = __ballot_sync(0xffffffffu, isG);
    __shared__ int warpCount[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warpCount[w] = __popc(m);
    __syncthreads();
    int base = chunkOffset[blockIdx.x];
    for (int q = 0; q < w; ++q) base += warpCount[q];
    if (isG) {
        int idx = base + __popc(m & ((1u << lane) - 1u));
        gCell[idx] = (int)c;
        atomicOr(bits + (c >> 5), 1u << (c & 31));
    }
}

__global__ void ghost_rows_kernel(Geo g, const double* xyz, const uint8_t* status, int nGhost, const int* gCell, double cx, double cy,
                                  double cz, double R, int* gCol, double* vMom, double* vP, int* err) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nGhost) return;
    const Lat& L = g.L;
    long long c = gCell[q];
    int i, j, k;
    L.ijk(c, i, j, k);
    v3 ctr = V(cx, cy, cz);
    v3 xg = ccAt(g, c);
    v3 l = unitv(sub(xg, ctr));                 // Sphere::nearestIntersect, Sphere.cpp:23-30
    v3 bp = add(ctr, mul(l, R));
    v3 ip = sub(mul(bp, 2.), xg);               // IbPiso.cpp:137-138
    int i0, j0, k0;
    bool ok = locateCell(xyz, L, ip, i, j, k, i0, j0, k0);
    int ii[8], jj[8], kk[8];
    bool enc = false;
    if (ok) {
        // HexaFvmMesh::locateEnclosingCells (HexaFvmMesh.cpp:378-418)
        for (int kq = k0 - 1; kq <= k0 && !enc; ++kq)
            for (int jq = j0 - 1; jq <= j0 && !enc; ++jq)
                for (int iq = i0 - 1; iq <= i0 && !enc; ++iq) {
                    if (iq < 0 || jq < 0 || kq < 0 || iq + 1 >= L.nI || jq + 1 >= L.nJ || kq + 1 >= L.nK) { kq = k0 + 1; jq = j0 + 1; break; }
                    v3 p[8] = {ccAt(g, L.cid(iq, jq, kq)), ccAt(g, L.cid(iq + 1, jq, kq)), ccAt(g, L.cid(iq + 1, jq + 1, kq)),
                               ccAt(g, L.cid(iq, jq + 1, kq)), ccAt(g, L.cid(iq, jq, kq + 1)), ccAt(g, L.cid(iq + 1, jq, kq + 1)),
                               ccAt(g, L.cid(iq + 1, jq + 1, kq + 1)), ccAt(g, L.cid(iq, jq + 1, kq + 1))};
                    if (insideHex(ip, p)) {
                        const int di[8] = {0, 1, 1, 0, 0, 1, 1, 0}, dj[8] = {0, 0, 1, 1, 0, 0, 1, 1}, dk[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                        for (int m = 0; m < 8; ++m) { ii[m] = iq + di[m]; jj[m] = jq + dj[m]; kk[m] = kq + dk[m]; }
                        enc = true;
                    }
                }
    }
    int* col = gCol + 9 * q;
    double* vm = vMom + 9 * q;
    double* vp = vP + 9 * q;
    if (!enc) {
        atomicExch(err, 1);
        col[0] = (int)c; vm[0] = 1.; vp[0] = -1.;
        for (int m = 1; m < 9; ++m) { col[m] = -1; vm[m] = 0.; vp[m] = 0.; }
        return;
    }
    v3 pts[8];
    for (int m = 0; m < 8; ++m) pts[m] = ccAt(g, L.cid(ii[m], jj[m], kk[m]));
    double beta[8];
    trilinear(pts, ip, beta);
    // momentum row: u_G + sum beta u_m = 0, self-reference folded into the diagonal (IbPiso.cpp:148-165)
    double dm = 1., dp = -1.;
    col[0] = (int)c;
    for (int m = 0; m < 8; ++m) {
        bool self = ii[m] == i && jj[m] == j && kk[m] == k;
        long long cm = L.cid(ii[m], jj[m], kk[m]);
        if (self) {
            dm += beta[m];
            // the p' diagonal is reset to -1 on every pass (IbPiso.cpp:168-183): only a self
            // reference in the last stencil slot survives
            dp = -1.;
            dp += beta[m];
            col[m + 1] = -1; vm[m + 1] = 0.; vp[m + 1] = 0.;
        } else {
            dp = -1.;
            bool dropped = status[cm] == ST_INACTIVE;
            col[m + 1] = dropped ? -1 : (int)cm;
            vm[m + 1] = beta[m];
            vp[m + 1] = beta[m];
        }
    }
    vm[0] = dm;
    vp[0] = dp;
}

// every cell inside the sphere -- ghost cells included, which IbPiso::computeIbField marks
// SOLID before re-flagging them IB -- gets u = 0, p = 0 (IbPiso.cpp:74-80)
__global__ void solid_reset_kernel(Lat L, const uint8_t* status, double* u, double* p) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N || status[c] == ST_ACTIVE) return;
    u[c] = 0.; u[c + L.PS] = 0.; u[c + 2 * L.PS] = 0.;
    p[c] = 0.;
}

__global__ void ghost_diag_kernel(int nGhost, const int* gCell, const double* vMom, const double* vP, double* momDiag, double* pDiag) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nGhost) return;
    long long c = gCell[q];
    momDiag[c] = vMom[9 * q];
    pDiag[c] = vP[9 * q];
}

}  // namespace

int ib_create(IbState& s, const Lat& L, uint8_t*& status, const Alloc& alloc, cudaStream_t st) {
    (void)st;
    status = reinterpret_cast<uint8_t*>(alloc((size_t)L.N));
    s.nChunks = (L.N + 1023) / 1024;
    s.bits = reinterpret_cast<uint32_t*>(alloc(sizeof(uint32_t) * (size_t)(L.N / 32 + 2)));
    s.chunkCount = reinterpret_cast<int*>(alloc(sizeof(int) * (size_t)(s.nChunks + 1)));
    s.chunkOffset = reinterpret_cast<int*>(alloc(sizeof(int) * (size_t)(s.nChunks + 1)));
    s.err = reinterpret_cast<int*>(alloc(sizeof(int) * 4));
    if (!status || !s.bits || !s.chunkCount || !s.chunkOffset || !s.err) { set_error("IB allocation failed"); return 1; }
    return 0;
}

int ib_setup(IbState& s, const Geo& g, const caffe_case& cs, const double* d_xyz, uint8_t* status, const Alloc& alloc,
             cudaStream_t st) {
    const Lat& L = g.L;
    uint8_t* fld = reinterpret_cast<uint8_t*>(alloc((size_t)L.N));
    if (!fld) { set_error("IB allocation failed"); return 1; }
    int* nInactive = s.err + 1;
    CB_CUDA(cudaMemsetAsync(s.err, 0, sizeof(int) * 4, st));
    classify_kernel<<<grid_for(L.N, 256), 256, 0, st>>>(g, cs.ib_center[0], cs.ib_center[1], cs.ib_center[2], cs.ib_radius, fld);
    ghost_flag_kernel<<<(unsigned)s.nChunks, 1024, 0, st>>>(L, fld, status, s.chunkCount, nInactive);
    CB_CHECK_LAUNCH();
    std::vector<int> cnt((size_t)s.nChunks), off((size_t)s.nChunks + 1);
    int hostInactive = 0;
    CB_CUDA(cudaMemcpyAsync(cnt.data(), s.chunkCount, sizeof(int) * s.nChunks, cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaMemcpyAsync(&hostInactive, nInactive, sizeof(int), cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
    off[0] = 0;
    for (long long q = 0; q < s.nChunks; ++q) off[q + 1] = off[q] + cnt[q];
    s.nGhost = s.nGhostHost = off[s.nChunks];
    s.nInactiveHost = hostInactive;
    CB_CUDA(cudaMemcpyAsync(s.chunkOffset, off.data(), sizeof(int) * s.nChunks, cudaMemcpyHostToDevice, st));
    int cap = s.nGhost > 0 ? s.nGhost : 1;
    s.gCell = reinterpret_cast<int*>(alloc(sizeof(int) * cap));
    s.gCol = reinterpret_cast<int*>(alloc(sizeof(int) * 9 * (size_t)cap));
    s.gValMom = reinterpret_cast<double*>(alloc(sizeof(double) * 9 * (size_t)cap));
    s.gValP = reinterpret_cast<double*>(alloc(sizeof(double) * 9 * (size_t)cap));
    if (!s.gCell || !s.gCol || !s.gValMom || !s.gValP) { set_error("IB allocation failed"); return 1; }
    ghost_list_kernel<<<(unsigned)s.nChunks, 1024, 0, st>>>(L, status, s.chunkOffset, s.gCell, s.bits);
    CB_CHECK_LAUNCH();
    if (s.nGhost > 0) {
        ghost_rows_kernel<<<grid_for(s.nGhost, 64), 64, 0, st>>>(g, d_xyz, status, s.nGhost, s.gCell, cs.ib_center[0], cs.ib_center[1],
                                                              cs.ib_center[2], cs.ib_radius, s.gCol, s.gValMom, s.gValP, s.err);
        CB_CHECK_LAUNCH();
    }
    int herr = 0;
    CB_CUDA(cudaMemcpyAsync(&herr, s.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("IbPiso: an image point lies outside the cell-centre lattice (sphere too close to the boundary)"); return 1; }
    return 0;
}

int ib_compute_field(IbState& s, const Geo& g, const caffe_case& cs, double* u, double* p, const uint8_t* status, cudaStream_t st) {
    (void)s; (void)cs;
    solid_reset_kernel<<<grid_for(g.L.N, 256), 256, 0, st>>>(g.L, status, u, p);
    CB_CHECK_LAUNCH();
    return 0;
}

int ib_compute_coeffs(IbState& s, const Geo& g, const caffe_case& cs, const uint8_t* status, double* momDiag, double* pDiag,
                      cudaStream_t st) {
    (void)g; (void)cs; (void)status;
    if (s.nGhost == 0) return 0;
    ghost_diag_kernel<<<grid_for(s.nGhost, 256), 256, 0, st>>>(s.nGhost, s.gCell, s.gValMom, s.gValP, momDiag, pDiag);
    CB_CHECK_LAUNCH();
    return 0;
}

}  // namespace cb
