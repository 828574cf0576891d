// caffe_ksp7_solve_device_noalloc: the stand-alone 7-point Krylov solve for callers that
// must not allocate device memory.
//
// Who needs it: a host program that owns the GPU's memory itself -- for example one whose
// own allocator has reserved nearly all of HBM up front, or a time-stepping loop that cannot
// afford the device-wide synchronisation that cudaFree implies -- cannot let a library call
// cudaMalloc/cudaFree on every solve, as caffe_ksp7_solve_device does for its workspace.
// This variant keeps the whole workspace in one file-scope __device__ array that is part of
// the loaded library, so a call allocates nothing.  The caller still provides the
// coefficients, the right-hand side and the solution array in device memory.
//
// Limits and rules:
//   * the array is SCRATCH_BYTES = 16 MiB and is held on every GPU that loads the library
//     until the process exits;  a lattice fits when
//       ceil256(11 * (N + 2*ceil32(nI*nJ)) * 8) + 128 KiB + 256 bytes <= 16 MiB
//     (N = nI*nJ*nK; about 180 thousand cells for a cube); larger lattices are rejected
//     with an error before any work is queued;
//   * every call on a device uses the same array and leaves its contents behind; the used
//     part is cleared at the start of each call, and two calls whose work overlaps on the
//     GPU (different streams, or different host threads) race on it;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, under a lock); make that first call before any
//     stream capture.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "krylov.cuh"

namespace cb {
namespace {

constexpr size_t SCRATCH_BYTES = size_t(16) << 20;
// 2 buffers x 8 doubles x up to 1024 blocks of partials: the cooperative grid is capped at 4
// blocks per SM, so this covers GPUs of up to 256 SMs (B200: 148); checked per call
constexpr size_t PARTIAL_BYTES = size_t(128) << 10;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_ksp_scratch[SCRATCH_BYTES];

std::mutex g_lock;
void* g_addr[MAX_DEVICES] = {};

// Device address of g_ksp_scratch for the current device (looked up once per device).
int scratch_address(void** out) {
    int dev = 0;
    CB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) { set_error("device ordinal beyond the supported range"); return 1; }
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ksp_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cudaGetSymbolAddress of the solver scratch failed: ") + cudaGetErrorString(e));
            return 1;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return 0;
}

size_t round256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace
}  // namespace cb

using namespace cb;

extern "C" int caffe_ksp7_solve_device_noalloc(int nI, int nJ, int nK, const double* d_coef7, const double* d_b, double* d_x,
                                               int method, double rtol, int maxit, void* stream, int* iters, double* rel_res) {
    clear_error();
    if (nI < 1 || nJ < 1 || nK < 1 || !d_coef7 || !d_b || !d_x) { set_error("invalid arguments"); return 1; }
    if (maxit < 1) { set_error("maxit must be >= 1"); return 1; }
    if (method != CAFFE_KSP_BICGSTAB_JACOBI && method != CAFFE_KSP_CG_JACOBI) {
        set_error("caffe_ksp7_solve_device_noalloc: only CAFFE_KSP_BICGSTAB_JACOBI and CAFFE_KSP_CG_JACOBI run on the device");
        return 1;
    }
    Lat L = make_lat(nI, nJ, nK);
    // workspace: b and x copies, r (2 planes), rp, p[2], v[2], t, invD -- 11 halo-padded planes
    // planes are packed at exactly one plane stride (PS doubles): the CG's second r buffer is
    // addressed as r + PS
    const size_t plane = (size_t)L.PS * sizeof(double);
    const size_t vecBytes = round256(11 * plane);
    const size_t need = vecBytes + PARTIAL_BYTES + round256(sizeof(KspOut));
    if (need > SCRATCH_BYTES) {
        set_error("caffe_ksp7_solve_device_noalloc: a " + std::to_string(nI) + "x" + std::to_string(nJ) + "x" +
                  std::to_string(nK) + " lattice needs " + std::to_string(need) + " bytes of workspace, more than the " +
                  std::to_string(SCRATCH_BYTES) + " the no-allocation solver holds; use caffe_ksp7_solve_device");
        return 1;
    }
    // the block partials of the cooperative solve (2 buffers x grid x 8 doubles) must fit their
    // fixed slice: the grid is at most 4 blocks per SM
    const int grid = krylov_grid_size(method == CAFFE_KSP_CG_JACOBI ? 4 : 3);
    if ((size_t)2 * grid * 8 * sizeof(double) > PARTIAL_BYTES) {
        set_error("caffe_ksp7_solve_device_noalloc: the solver's grid of " + std::to_string(grid) +
                  " blocks needs more block-partial space than the no-allocation workspace holds");
        return 1;
    }
    void* base = nullptr;
    if (scratch_address(&base)) return 1;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char* s = static_cast<unsigned char*>(base);
    // the array keeps the previous call's data: clear the part this call uses (halos must be zero)
    CB_CUDA(cudaMemsetAsync(s, 0, need, st));
    auto vec = [&](int q) { return reinterpret_cast<double*>(s + (size_t)q * plane) + L.H; };
    double* b = vec(0);
    double* x = vec(1);
    KspWork w;
    std::memset(&w, 0, sizeof(w));
    w.r = vec(2);              // planes 2 and 3: the CG keeps its second r buffer one plane stride on
    w.rp = vec(4);
    w.p[0] = vec(5); w.p[1] = vec(6);
    w.v[0] = vec(7); w.v[1] = vec(8);
    w.t = vec(9);
    w.invD = vec(10);
    w.partials = reinterpret_cast<double*>(s + vecBytes);
    w.out = reinterpret_cast<KspOut*>(s + vecBytes + PARTIAL_BYTES);
    CB_CUDA(cudaMemcpyAsync(b, d_b, (size_t)L.N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    Op7 A;
    for (int q = 0; q < 7; ++q) A.a[q] = d_coef7 + (size_t)q * L.N;   // coefficients are read at their own row only
    A.nI = L.nI; A.nIJ = L.nIJ;
    A.gh.n = 0; A.gh.cell = nullptr; A.gh.col = nullptr; A.gh.val = nullptr; A.gh.bits = nullptr;
    int rc = method == CAFFE_KSP_CG_JACOBI ? ksp_cg7(A, b, x, L, w, rtol, maxit, st) : ksp_bicgstab(A, 1, b, x, L, w, rtol, maxit, st);
    if (rc) return rc;
    KspOut o;
    CB_CUDA(cudaMemcpyAsync(d_x, x, (size_t)L.N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CB_CUDA(cudaMemcpyAsync(&o, w.out, sizeof(KspOut), cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
    if (iters) *iters = o.iters[0];
    if (rel_res) *rel_res = o.relres[0];
    return o.status[0];
}
