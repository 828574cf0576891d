// Mesh metrics on the device, computed once from the node array.
//
// Restates HexaFvmMesh::initializeCellsAndFaces (src/Domains/HexaFvmMesh/HexaFvmMesh.cpp:615-918)
// and the Geometry routines it uses (src/Math/Geometry.cpp:5-112, 258-277), keeping the
// reference's operand order.  This file is compiled with --fmad=false so that every
// product and sum is rounded separately, as in the reference's CPU build, which makes
// the metrics bit-identical to the CPU oracle's.
//
// Storage: one value per face instead of the reference's six per cell.  For an interior
// face between cells L and R, HexaFvmMesh stores dE(L) and dW(R); they are the same
// number (dW uses -S and -r, whose products equal those of S and r exactly), so the face
// keeps one D.  Likewise cW(R) == -cE(L) bit for bit, so one non-orthogonal vector per
// face is kept in the east-side orientation.  Volume weights g are recomputed from the
// two cell volumes when needed (three loads instead of six stored arrays).
#include "common.cuh"

namespace cb {

struct v3 { double x, y, z; };
__device__ __forceinline__ v3 V(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
__device__ __forceinline__ v3 mul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ v3 divr(v3 a, double s) { double r = 1. / s; return V(a.x * r, a.y * r, a.z * r); }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 u, v3 v) { return V(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
__device__ __forceinline__ double mag(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ v3 unitv(v3 a) { double inv = 1. / mag(a); return V(inv * a.x, inv * a.y, inv * a.z); }

__device__ __forceinline__ v3 node(const double* xyz, int nNI, int nNJ, int i, int j, int k) {
    long long q = ((long long)k * nNJ + j) * nNI + i;
    return V(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]);
}

__device__ double quadArea(const v3* p) {  // Geometry.cpp:5-12
    v3 r01 = sub(p[1], p[0]), r02 = sub(p[2], p[0]), r03 = sub(p[3], p[0]);
    return 0.5 * (mag(cross(r02, r01)) + mag(cross(r03, r02)));
}
__device__ v3 quadCentroid(const v3* p) {  // Geometry.cpp:14-20
    v3 d1 = add(p[0], mul(sub(p[2], p[0]), 0.5));
    v3 d2 = add(p[1], mul(sub(p[3], p[1]), 0.5));
    return add(d1, mul(sub(d2, d1), 0.5));
}
__device__ double hexVolume(const v3* p) {  // Geometry.cpp:40-59
    v3 s1265 = mul(cross(sub(p[6], p[1]), sub(p[5], p[2])), 0.5);
    v3 s5674 = mul(cross(sub(p[7], p[5]), sub(p[4], p[6])), 0.5);
    v3 s2376 = mul(cross(sub(p[7], p[2]), sub(p[6], p[3])), 0.5);
    return fabs(dot(add(add(s1265, s5674), s2376), sub(p[6], p[0])) / 3.);
}
__device__ v3 hexCentroid(const v3* p) {  // Geometry.cpp:61-109, 258-277
    const int tv[5][4] = {{4, 3, 6, 7}, {4, 1, 6, 5}, {4, 1, 6, 3}, {4, 0, 1, 3}, {3, 1, 2, 6}};
    v3 tc[5];
    double vol[5], sumV = 0.;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        v3 q0 = p[tv[t][0]], q1 = p[tv[t][1]], q2 = p[tv[t][2]], q3 = p[tv[t][3]];
        v3 s = V(0., 0., 0.);
        s = add(s, q0); s = add(s, q1); s = add(s, q2); s = add(s, q3);
        tc[t] = mul(s, 0.25);
        v3 a = sub(q1, q0), b = sub(q2, q0), c = sub(q3, q0);
        vol[t] = fabs(dot(a, cross(b, c))) / 6.;
        sumV += vol[t];
    }
    v3 c = V(0., 0., 0.);
#pragma unroll
    for (int t = 0; t < 5; ++t) c = add(c, mul(tc[t], vol[t]));
    return divr(c, sumV);
}

__global__ void cell_metrics_kernel(Lat L, const double* __restrict__ xyz, double* vol, double* cc) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= L.N) return;
    int i, j, k;
    L.ijk(c, i, j, k);
    int nNI = L.nI + 1, nNJ = L.nJ + 1;
    v3 p[8] = {node(xyz, nNI, nNJ, i, j, k), node(xyz, nNI, nNJ, i + 1, j, k), node(xyz, nNI, nNJ, i + 1, j + 1, k),
               node(xyz, nNI, nNJ, i, j + 1, k), node(xyz, nNI, nNJ, i, j, k + 1), node(xyz, nNI, nNJ, i + 1, j, k + 1),
               node(xyz, nNI, nNJ, i + 1, j + 1, k + 1), node(xyz, nNI, nNJ, i, j + 1, k + 1)};
    v3 ctr = hexCentroid(p);
    vol[c] = hexVolume(p);
    cc[c] = ctr.x; cc[c + L.PS] = ctr.y; cc[c + 2 * L.PS] = ctr.z;
}

// Face centroid and area-normal vector (HexaFvmMesh.cpp:699-789).
template <int DIR>
__global__ void face_metrics_kernel(Lat L, const double* __restrict__ xyz, double* S, double* fc) {
    long long nF = DIR == 0 ? L.nFI : (DIR == 1 ? L.nFJ : L.nFK);
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int fI = DIR == 0 ? L.nI + 1 : L.nI;
    int fJ = DIR == 1 ? L.nJ + 1 : L.nJ;
    int i = (int)(f % fI);
    long long t = f / fI;
    int j = (int)(t % fJ);
    int k = (int)(t / fJ);
    int nNI = L.nI + 1, nNJ = L.nJ + 1;
    v3 p[4];
    if (DIR == 0) {
        p[0] = node(xyz, nNI, nNJ, i, j, k); p[1] = node(xyz, nNI, nNJ, i, j + 1, k);
        p[2] = node(xyz, nNI, nNJ, i, j + 1, k + 1); p[3] = node(xyz, nNI, nNJ, i, j, k + 1);
    } else if (DIR == 1) {
        p[0] = node(xyz, nNI, nNJ, i, j, k); p[1] = node(xyz, nNI, nNJ, i, j, k + 1);
        p[2] = node(xyz, nNI, nNJ, i + 1, j, k + 1); p[3] = node(xyz, nNI, nNJ, i + 1, j, k);
    } else {
        p[0] = node(xyz, nNI, nNJ, i, j, k); p[1] = node(xyz, nNI, nNJ, i + 1, j, k);
        p[2] = node(xyz, nNI, nNJ, i + 1, j + 1, k); p[3] = node(xyz, nNI, nNJ, i, j + 1, k);
    }
    v3 tv = unitv(cross(sub(p[1], p[0]), sub(p[2], p[0])));
    double a = quadArea(p);
    v3 ctr = quadCentroid(p);
    v3 s = mul(tv, a);
    S[f] = s.x; S[f + nF] = s.y; S[f + 2 * nF] = s.z;
    fc[f] = ctr.x; fc[f + nF] = ctr.y; fc[f + 2 * nF] = ctr.z;
}

// d_f = |S|^2 / (S.r) and c_f = S - r |S|^2 / (S.r) (HexaFvmMesh.cpp:866-885), with r the
// cell-to-cell vector, or the cell-to-face vector at a boundary (HexaFvmMesh.cpp:218-294).
template <int DIR>
__global__ void face_D_kernel(Lat L, const double* __restrict__ S, const double* __restrict__ fc,
                              const double* __restrict__ cc, double* D, double* cv) {
    long long nF = DIR == 0 ? L.nFI : (DIR == 1 ? L.nFJ : L.nFK);
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int fI = DIR == 0 ? L.nI + 1 : L.nI;
    int fJ = DIR == 1 ? L.nJ + 1 : L.nJ;
    int i = (int)(f % fI);
    long long t = f / fI;
    int j = (int)(t % fJ);
    int k = (int)(t / fJ);
    int idx = DIR == 0 ? i : (DIR == 1 ? j : k);
    int n = DIR == 0 ? L.nI : (DIR == 1 ? L.nJ : L.nK);
    v3 s = V(S[f], S[f + nF], S[f + 2 * nF]);
    v3 face = V(fc[f], fc[f + nF], fc[f + 2 * nF]);
    // neighbouring cells: lower ("west") cell index idx-1, upper ("east") cell idx
    int li = i - (DIR == 0), lj = j - (DIR == 1), lk = k - (DIR == 2);
    bool west_boundary = idx == 0;
    v3 r;
    if (idx > 0 && idx < n) {
        long long cL = L.cid(li, lj, lk), cR = L.cid(i, j, k);
        r = sub(V(cc[cR], cc[cR + L.PS], cc[cR + 2 * L.PS]), V(cc[cL], cc[cL + L.PS], cc[cL + 2 * L.PS]));
    } else if (idx == n) {
        long long cL = L.cid(li, lj, lk);
        r = sub(face, V(cc[cL], cc[cL + L.PS], cc[cL + 2 * L.PS]));
    } else {
        long long cR = L.cid(i, j, k);
        r = sub(face, V(cc[cR], cc[cR + L.PS], cc[cR + 2 * L.PS]));
    }
    if (west_boundary) s = neg(s);   // the boundary face seen from its only cell: S_W = -S
    double dd = dot(s, s), dr = dot(s, r);
    D[f] = dd / dr;
    if (cv) {
        v3 c = sub(s, divr(mul(r, dd), dr));
        if (west_boundary) c = neg(c);   // store in the east-side orientation
        cv[f] = c.x; cv[f + nF] = c.y; cv[f + 2 * nF] = c.z;
    }
}

int compute_metrics(const Lat& L, const double* d_xyz, double* vol, double* cc, double* S[3], double* fc[3],
                    double* D[3], double* cv[3], cudaStream_t st) {
    const int B = 256;
    cell_metrics_kernel<<<grid_for(L.N, B), B, 0, st>>>(L, d_xyz, vol, cc);
    CB_CHECK_LAUNCH();
    face_metrics_kernel<0><<<grid_for(L.nFI, B), B, 0, st>>>(L, d_xyz, S[0], fc[0]);
    face_metrics_kernel<1><<<grid_for(L.nFJ, B), B, 0, st>>>(L, d_xyz, S[1], fc[1]);
    face_metrics_kernel<2><<<grid_for(L.nFK, B), B, 0, st>>>(L, d_xyz, S[2], fc[2]);
    CB_CHECK_LAUNCH();
    face_D_kernel<0><<<grid_for(L.nFI, B), B, 0, st>>>(L, S[0], fc[0], cc, D[0], cv[0]);
    face_D_kernel<1><<<grid_for(L.nFJ, B), B, 0, st>>>(L, S[1], fc[1], cc, D[1], cv[1]);
    face_D_kernel<2><<<grid_for(L.nFK, B), B, 0, st>>>(L, S[2], fc[2], cc, D[2], cv[2]);
    CB_CHECK_LAUNCH();
    return 0;
}

}  // namespace cb
