// Learned preconditioner network kernels: 3x3x3 convolutions with 16 input and 16 output
// channels as implicit GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Data: activations are channel-last bf16, 16 channels (32 bytes) per cell, cell index
// (k*nJ + j)*nI + i; zero padding outside the lattice.
//
// One CTA owns an 8 (i) x 16 (j) tile of output cells and marches through KC consecutive
// k-planes.  Its warps specialise: one thread streams the input planes in by TMA up to three
// planes ahead through six staging slots, one thread issues the MMAs, and four warps drain the
// four TMEM accumulators (epilogue), each handing over to the next through mbarriers, so loads,
// MMAs and stores of different planes overlap.  For each output plane the tile is one UMMA problem
// M = 128 cells, N = 16 output channels, accumulated over the 27 taps with one
// tcgen05.mma.kind::f16 of K = 16 input channels per tap into a 128 x 16 FP32 accumulator
// in tensor memory.  The input planes arrive by TMA (cp.async.bulk.tensor, one thread issuing,
// completion on a per-slot mbarrier): a box of 8 (i) x 18 (j, one halo row each side) cells x 16
// channels lands as rows of 32 bytes (one cell's channels) with the 32-byte swizzle, which is the
// K-major SWIZZLE_32B operand layout of the MMA, so the A operand of tap (dk, dj, di) is input
// plane k+dk loaded at i offset di (three boxes per plane) and advanced by dj rows of 8 cells
// (256 bytes) in the descriptor; cells outside the lattice arrive as zeros.  B is the tap's
// 16 x 16 weight block (no-swizzle canonical layout).  Input planes rotate through the staging
// slots as the CTA moves along k, so each input plane is read from global memory once per tile.
// The tensor map covers this GPU's own activation buffer only (no cluster multicast).  The epilogue reads the accumulator with
// tcgen05.ld (one TMEM lane per thread = one cell), applies bias / ReLU, or the ReLU mask
// of the backward pass, and writes bf16 (or FP32 for the network output).
//
// Every mbarrier wait is bounded; a role whose wait runs out marks the CTA failed, the other roles
// stop at their next wait, the MMAs and TMA loads already issued are waited for (bounded), the
// CTA records an error and frees its tensor memory before leaving.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <array>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>
#include <cstring>
#include <string>

#include "common.cuh"
#include "cnn.cuh"

namespace cb {

namespace {

constexpr int TI = 8, TJ = 16;          // tile: 8 cells along i, 16 along j -> M = 128
constexpr int ROWS = TJ + 2;            // staged j-rows (one halo row each side)
constexpr int GROUP_BYTES = 256;        // one j-row of 8 cells x 16 channels, canonical layout
constexpr int BUF_BYTES = ROWS * GROUP_BYTES;          // 4608
constexpr int NPL = 6;                  // staged input-plane slots (each 3 i-shifted boxes)
constexpr int NACC = 4;                 // TMEM accumulators (16 columns each)
constexpr int W_BYTES = 27 * 512;       // 27 taps x 16 x 16 bf16
constexpr uint32_t TMEM_COLS = 16 * NACC;
constexpr int EPI_THREADS = 128;        // warps 0-3: epilogue
constexpr int PRODUCER_THREAD = 128;    // warp 4, lane 0: TMA loads
constexpr int MMA_THREAD = 160;         // warp 5, lane 0: MMA issue
constexpr int CONV_THREADS = 192;

// one lattice of a grouped convolution launch (kernel parameter space)
struct ConvJob {
    CUtensorMap map;                 // activations in (this GPU's own buffer)
    Lat L;
    __nv_bfloat16* out_bf;
    float* out_f;
    const __nv_bfloat16* mask;
    int KC, gx, gy;
};
struct ConvGroup {
    ConvJob job[CONV_MAX_JOBS];
    int ctaEnd[CONV_MAX_JOBS];       // inclusive prefix sums of the jobs' CTA counts
    int n;
};
constexpr long long WAIT_LIMIT = 1ll << 20;   // try_wait rounds (each may block briefly): about a second at most

// instruction descriptor: kind::f16, D = F32, A = B = BF16, both K-major, N = 16, M = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle (sm_100 version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

// the same test, letting the hardware suspend the thread for up to `ns` nanoseconds while the
// phase is incomplete (it resumes when the phase completes), so that waiting warps do not take
// issue slots from the producer and MMA threads
__device__ __forceinline__ bool mbar_try_sleep(uint32_t bar, uint32_t phase, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase), "r"(ns)
        : "memory");
    return ok != 0;
}
constexpr long long SLEEP_WAIT_LIMIT = 1ll << 19;   // rounds of at most SLEEP_NS each: about a second at most
constexpr uint32_t SLEEP_NS = 2000;

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase) {
    for (long long t = 0; t < WAIT_LIMIT; ++t)
        if (mbar_try(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// shared-memory matrix descriptor of a K-major SWIZZLE_32B operand: rows of 32 bytes (16 bf16 of
// K), 8-row groups SBO bytes apart; the start address must be 256-byte aligned (base offset 0)
__device__ __forceinline__ uint64_t sdesc_sw32(uint32_t saddr, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                                  // leading byte offset: 16 bytes (unused within the swizzle span)
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)6 << 61;                                  // layout type SWIZZLE_32B
    return d;
}

// TMA: one box of the activation tensor (channels, i, j, k) at coordinates (0, ci, cj, ck) into
// shared memory, completion counted on mbarrier `bar`
__device__ __forceinline__ void tma_load_box(uint32_t dst, const CUtensorMap* map, int ci, int cj, int ck, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        :
        : "r"(dst), "l"((uint64_t)map), "r"(0), "r"(ci), "r"(cj), "r"(ck), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

}  // namespace

// EPI: 0 bias + ReLU -> bf16; 1 bias -> FP32 channel 0 (network output); 2 backward data:
// multiply by (mask_act > 0) -> bf16.  Weights: packed canonical blocks, 27 x 512 bytes.
//
// Warp roles (192 threads): warps 0-3 run the epilogue (thread = TMEM lane = output cell), warp 4
// lane 0 issues the TMA loads, warp 5 lane 0 issues the MMAs.  They hand work over through
// mbarriers only:
//   full[s]   plane slot s has landed (TMA transaction count)
//   empty[s]  the last MMAs reading slot s have completed (tcgen05.commit after output plane o,
//             the last reader of input plane o)
//   accf[a]   accumulator a holds a finished output plane (tcgen05.commit)
//   acce[a]   the epilogue has read accumulator a (128 arrivals)
// Input plane q (= k0 - 1 + q) lives in slot q mod NPL; output plane o (= k0 + o) reads input
// planes o, o+1, o+2 and accumulates in TMEM columns 16 (o mod NACC).  The producer runs up to
// NPL - 3 planes ahead of the MMAs and the MMAs up to NACC - 1 planes ahead of the epilogue.
//
// One launch serves a group of up to CONV_MAX_JOBS lattices (the levels of a pyramid and both
// signs of the odd network form): the CTAs of job p are blocks ctaEnd[p-1] .. ctaEnd[p]-1, each
// job with its own tensor map, lattice, outputs and k-planes per CTA, and every job the same layer
// weights.
template <int EPI>
__global__ void __launch_bounds__(CONV_THREADS) conv3d_tc_kernel(const __grid_constant__ ConvGroup g,
                                                                 const __nv_bfloat16* __restrict__ wpack, const float* __restrict__ bias,
                                                                 int* err, const int* __restrict__ skip) {
    // a solve that has already converged turns its remaining launches into no-ops (uniform)
    if (skip && *skip) return;
    int job = 0;
    while (job + 1 < g.n && (int)blockIdx.x >= g.ctaEnd[job]) ++job;
    const ConvJob& J = g.job[job];
    const Lat L = J.L;
    const CUtensorMap* in_map = &J.map;
    __nv_bfloat16* out_bf = J.out_bf;
    float* out_f = J.out_f;
    const __nv_bfloat16* __restrict__ mask_act = J.mask;
    const int KC = J.KC;
    const int local = (int)blockIdx.x - (job > 0 ? g.ctaEnd[job - 1] : 0);
    const int bx = local % J.gx, by = (local / J.gx) % J.gy, bz = local / (J.gx * J.gy);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1 KiB-align the dynamic region
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* wsm = smem;                                // W_BYTES
    unsigned char* bufs = smem + W_BYTES;                     // NPL x 3 x BUF_BYTES
    __shared__ __align__(8) uint64_t full[NPL], empty[NPL], accf[NACC], acce[NACC];
    __shared__ uint32_t tmem_base_sh;
    __shared__ float bias_sh[16];
    __shared__ volatile int fail_sh;

    const int i0 = bx * TI, j0 = by * TJ;
    const int k0 = bz * KC;
    const int nO = min(k0 + KC, L.nK) - k0;   // output planes of this CTA
    const int nP = nO + 2;                    // input planes k0-1 .. k0+nO
    const int warp = threadIdx.x >> 5;

    // weights and bias to shared memory
    for (int u = threadIdx.x; u < W_BYTES / 16; u += blockDim.x)
        reinterpret_cast<uint4*>(wsm)[u] = reinterpret_cast<const uint4*>(wpack)[u];
    if (threadIdx.x < 16) bias_sh[threadIdx.x] = bias ? bias[threadIdx.x] : 0.f;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NPL; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[q])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[q])));
        }
        for (int q = 0; q < NACC; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf[q])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acce[q])), "r"(EPI_THREADS));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fail_sh = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_sh;

    // bounded wait that also gives up once another role has failed (checked every 16 rounds); the
    // epilogue warps suspend in hardware while they wait, the single producer and MMA threads poll
    // so that they resume at once
    auto wait = [&](uint64_t* b, uint32_t parity, bool sleep) -> bool {
        const uint32_t a = smem_u32(b);
        const long long limit = sleep ? SLEEP_WAIT_LIMIT : WAIT_LIMIT;
        for (long long t = 0; t < limit; ++t) {
            if (sleep ? mbar_try_sleep(a, parity, SLEEP_NS) : mbar_try(a, parity)) return true;
            if ((t & 15) == 15 && fail_sh) return false;
        }
        fail_sh = 1;
        return false;
    };

    if (threadIdx.x == PRODUCER_THREAD) {
        // TMA producer: plane q into slot q mod NPL once the MMAs have released the slot
        int issued[NPL] = {};
        for (int q = 0; q < nP; ++q) {
            const int sl = q % NPL;
            if (q >= NPL && !wait(&empty[sl], (uint32_t)((q / NPL - 1) & 1), false)) break;
            const uint32_t fb = smem_u32(&full[sl]);
            mbar_expect_tx(fb, 3 * BUF_BYTES);
            for (int sh = 0; sh < 3; ++sh)
                tma_load_box(smem_u32(bufs + (size_t)(sl * 3 + sh) * BUF_BYTES), in_map, i0 + sh - 1, j0 - 1, k0 - 1 + q, fb);
            ++issued[sl];
        }
        // every load in flight lands before the shared memory is released
        for (int sl = 0; sl < NPL; ++sl)
            if (issued[sl] > 0) mbar_wait_bounded(smem_u32(&full[sl]), (uint32_t)((issued[sl] - 1) & 1));
    } else if (threadIdx.x == MMA_THREAD) {
        // MMA issuer: the 27 taps of output plane o into accumulator o mod NACC
        const uint32_t wbase = smem_u32(wsm);
        const uint32_t bbase = smem_u32(bufs);
        int ready = 0;
        int committed[NACC] = {};
        for (int o = 0; o < nO; ++o) {
            const int a = o % NACC;
            bool ok = true;
            while (ok && ready < o + 3) {
                ok = wait(&full[ready % NPL], (uint32_t)((ready / NPL) & 1), false);
                ++ready;
            }
            if (ok && o >= NACC) ok = wait(&acce[a], (uint32_t)((o / NACC - 1) & 1), false);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            int t = 0;
#pragma unroll
            for (int dk = 0; dk < 3; ++dk) {
                const int sl = (o + dk) % NPL;
#pragma unroll
                for (int dj = 0; dj < 3; ++dj)
#pragma unroll
                    for (int di = 0; di < 3; ++di, ++t) {
                        const uint32_t a_addr = bbase + (uint32_t)((sl * 3 + di) * BUF_BYTES + dj * GROUP_BYTES);
                        mma_bf16(tmem + (uint32_t)(16 * a), sdesc_sw32(a_addr, 256), sdesc(wbase + (uint32_t)(t * 512), 128, 256),
                                 t > 0 ? 1u : 0u);
                    }
            }
            mma_commit(smem_u32(&accf[a]));
            mma_commit(smem_u32(&empty[o % NPL]));
            ++committed[a];
        }
        // every MMA issued completes before the tensor memory is released
        for (int a = 0; a < NACC; ++a)
            if (committed[a] > 0) mbar_wait_bounded(smem_u32(&accf[a]), (uint32_t)((committed[a] - 1) & 1));
    } else if (threadIdx.x < EPI_THREADS) {
        // epilogue: thread = TMEM lane = output cell (i0 + m mod 8, j0 + m / 8)
        const int m = threadIdx.x;
        const int i = i0 + (m & 7), j = j0 + (m >> 3);
        const bool inside = i < L.nI && j < L.nJ;
        for (int o = 0; o < nO; ++o) {
            const int a = o % NACC;
            // warp-uniform outcome: the tcgen05.ld below is a warp-wide instruction
            if (!__all_sync(0xffffffffu, wait(&accf[a], (uint32_t)((o / NACC) & 1), true) ? 1 : 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * a), v);
            asm volatile("tcgen05.fence::before_thread_sync;");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acce[a])) : "memory");
            if (inside) {
                const long long c = ((long long)(k0 + o) * L.nJ + j) * L.nI + i;
                if (EPI == 1) {
                    out_f[c] = v[0] + bias_sh[0];
                } else {
                    float r[16];
                    if (EPI == 0) {
#pragma unroll
                        for (int q = 0; q < 16; ++q) r[q] = fmaxf(v[q] + bias_sh[q], 0.f);
                    } else {
                        const uint4* mp = reinterpret_cast<const uint4*>(mask_act + c * 16);
                        const uint4 m0 = mp[0], m1 = mp[1];
                        const __nv_bfloat16* mk0 = reinterpret_cast<const __nv_bfloat16*>(&m0);
                        const __nv_bfloat16* mk1 = reinterpret_cast<const __nv_bfloat16*>(&m1);
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            r[q] = __bfloat162float(mk0[q]) > 0.f ? v[q] : 0.f;
                            r[8 + q] = __bfloat162float(mk1[q]) > 0.f ? v[8 + q] : 0.f;
                        }
                    }
                    __align__(16) __nv_bfloat16 ob[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) ob[q] = __float2bfloat16_rn(r[q]);
                    uint4* dst = reinterpret_cast<uint4*>(out_bf + c * 16);
                    dst[0] = reinterpret_cast<uint4*>(ob)[0];
                    dst[1] = reinterpret_cast<uint4*>(ob)[1];
                }
            }
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (threadIdx.x == 0 && fail_sh) atomicExch(err, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

size_t conv_smem_bytes() { return 1024 + W_BYTES + (size_t)NPL * 3 * BUF_BYTES; }

// ------------------------------------------------------------------ weight gradient
// dW[t][o][i] = sum_c x[c + off(t)][i] dz[c][o] (db[o] = sum_c dz[c][o]) as an implicit GEMM on the
// tensor cores: D[(t, i)][o] = sum_c A[(t, i)][c] B[o][c] with M = 128 rows = 8 taps x 16 input
// channels (four M tiles cover the 27 taps; rows of taps 27..31 are zero), N = 16 output channels
// and K = the cells, 16 per tcgen05.mma.  A CTA (128 threads) takes chunks of 16 consecutive cells
// along i, builds for each chunk the im2col tile A (taps x channels x cells) and the tile B
// (dz, channels x cells) in shared memory in the canonical no-swizzle K-major layout, and one
// thread issues the chunk's four MMAs into four 128 x 16 FP32 accumulators in tensor memory that
// stay there for all the CTA's chunks.  Two staging buffers alternate, so the next chunk is built
// while the MMAs of the previous one run.  At the end every thread reads its accumulator row
// (tcgen05.ld) and adds it to the FP32 gradient.
namespace {
constexpr int WG_CH = 16;                          // cells per chunk (the MMA's K)
constexpr int WG_TILE_BYTES = 16 * 256;            // 16 row groups of 8 rows x 2 K groups x 16 bytes
constexpr int WG_A_BYTES = 4 * WG_TILE_BYTES;      // four M tiles
constexpr int WG_B_BYTES = 512;                    // 16 x 16 bf16
constexpr int WG_STAGE_BYTES = WG_A_BYTES + WG_B_BYTES;
constexpr uint32_t WG_TMEM_COLS = 64;              // four 16-column accumulators

// byte offset of element (row m, K column k) in a canonical no-swizzle K-major tile
__device__ __forceinline__ int kmajor_off(int m, int k) { return (m >> 3) * 256 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2; }
}  // namespace

__global__ void __launch_bounds__(128) weight_grad_tc_kernel(Lat L, const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ dz,
                                                             float* dW, float* db, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base_sh;
    const int warp = threadIdx.x >> 5;
    const int chunksI = (L.nI + WG_CH - 1) / WG_CH;
    const long long nChunks = (long long)chunksI * L.nJ * L.nK;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(WG_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_sh;
    const uint32_t bar[2] = {smem_u32(&mbar[0]), smem_u32(&mbar[1])};
    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    bool failed = false;
    float dbs[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) dbs[o] = 0.f;
    int n = 0;
    for (long long u = blockIdx.x; u < nChunks; u += gridDim.x, ++n) {
        const int s = n & 1;
        // the MMAs that read this staging buffer two chunks ago must have finished
        if (pending[s]) {
            bool ok = mbar_wait_bounded(bar[s], phase[s]);
            // a wait that ran out keeps its phase and stays pending: the drain below waits for
            // those MMAs once more (bounded) before the tensor memory is freed
            if (ok) { phase[s] ^= 1u; pending[s] = false; }
            if (__syncthreads_or(ok ? 0 : 1)) { failed = true; break; }
        }
        unsigned char* A = smem + s * WG_STAGE_BYTES;
        unsigned char* B = A + WG_A_BYTES;
        const int ci = (int)(u % chunksI);
        const long long rest = u / chunksI;
        const int j = (int)(rest % L.nJ), k = (int)(rest / L.nJ);
        const int i0 = ci * WG_CH;
        // A: 32 taps x 16 cells, one (tap, cell) pair = 16 channels per step
        for (int p = threadIdx.x; p < 32 * WG_CH; p += blockDim.x) {
            const int cell = p & (WG_CH - 1), t = p / WG_CH;
            uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
            if (t < 27) {
                const int ii = i0 + cell + t % 3 - 1, jj = j + (t / 3) % 3 - 1, kk = k + t / 9 - 1;
                if (ii >= 0 && ii < L.nI && jj >= 0 && jj < L.nJ && kk >= 0 && kk < L.nK) {
                    const uint4* src = reinterpret_cast<const uint4*>(x + (((long long)kk * L.nJ + jj) * L.nI + ii) * 16);
                    lo = src[0];
                    hi = src[1];
                }
            }
            const __nv_bfloat16* vl = reinterpret_cast<const __nv_bfloat16*>(&lo);
            const __nv_bfloat16* vh = reinterpret_cast<const __nv_bfloat16*>(&hi);
            unsigned char* tile = A + (t >> 3) * WG_TILE_BYTES;
            const int m0 = (t & 7) * 16;
#pragma unroll
            for (int ch = 0; ch < 8; ++ch) {
                *reinterpret_cast<__nv_bfloat16*>(tile + kmajor_off(m0 + ch, cell)) = vl[ch];
                *reinterpret_cast<__nv_bfloat16*>(tile + kmajor_off(m0 + 8 + ch, cell)) = vh[ch];
            }
        }
        // B: dz of the chunk's cells (zero beyond the row), and the bias gradient
        if (threadIdx.x < WG_CH) {
            const int cell = threadIdx.x, ii = i0 + cell;
            uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
            if (ii < L.nI) {
                const uint4* src = reinterpret_cast<const uint4*>(dz + (((long long)k * L.nJ + j) * L.nI + ii) * 16);
                lo = src[0];
                hi = src[1];
            }
            const __nv_bfloat16* vl = reinterpret_cast<const __nv_bfloat16*>(&lo);
            const __nv_bfloat16* vh = reinterpret_cast<const __nv_bfloat16*>(&hi);
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                *reinterpret_cast<__nv_bfloat16*>(B + kmajor_off(o, cell)) = vl[o];
                *reinterpret_cast<__nv_bfloat16*>(B + kmajor_off(8 + o, cell)) = vh[o];
                dbs[o] += __bfloat162float(vl[o]);
                dbs[8 + o] += __bfloat162float(vh[o]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (threadIdx.x == 0) {
            const uint64_t bd = sdesc(smem_u32(B), 128, 256);
#pragma unroll 1
            for (int T = 0; T < 4; ++T) {
                const uint64_t ad = sdesc(smem_u32(A + T * WG_TILE_BYTES), 128, 256);
                mma_bf16(tmem + (uint32_t)(16 * T), ad, bd, n > 0 ? 1u : 0u);
            }
            mma_commit(bar[s]);
        }
        pending[s] = true;
    }
    // drain: every committed group completes before the accumulators are read or freed
    for (int q = 0; q < 2; ++q) {
        if (!pending[q]) continue;
        bool ok = mbar_wait_bounded(bar[q], phase[q]);
        phase[q] ^= 1u;
        if (!ok) failed = true;
    }
    const bool anyFail = __syncthreads_or(failed ? 1 : 0);
    if (anyFail) {
        if (threadIdx.x == 0) atomicExch(err, 1);
    } else if (n > 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // thread = accumulator row m = (tap, input channel) of each M tile
        const int m = threadIdx.x, tl = m >> 4, ch = m & 15;
#pragma unroll 1
        for (int T = 0; T < 4; ++T) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * T), v);
            const int t = 8 * T + tl;
            if (t < 27)
#pragma unroll
                for (int o = 0; o < 16; ++o) atomicAdd(dW + (t * 16 + o) * 16 + ch, v[o]);
        }
        if (threadIdx.x < WG_CH)
#pragma unroll
            for (int o = 0; o < 16; ++o) atomicAdd(db + o, dbs[o]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(WG_TMEM_COLS));
}

int launch_weight_grad(const Lat& L, const __nv_bfloat16* x, const __nv_bfloat16* dz, float* dW, float* db, int* err, cudaStream_t st) {
    const size_t smem = 1024 + 2 * (size_t)WG_STAGE_BYTES;
    static bool attr = false;
    if (!attr) {
        CB_CUDA(cudaFuncSetAttribute(weight_grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long nChunks = (long long)((L.nI + WG_CH - 1) / WG_CH) * L.nJ * L.nK;
    // a few CTAs per SM, each accumulating many chunks in tensor memory before its atomics
    const long long g = std::min<long long>(nChunks, 4LL * nsm);
    weight_grad_tc_kernel<<<(unsigned)(g > 0 ? g : 1), 128, smem, st>>>(L, x, dz, dW, db, err);
    CB_CHECK_LAUNCH();
    return 0;
}

namespace {
// cuTensorMapEncodeTiled from the driver, looked up once (no link-time dependency on libcuda)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
}  // namespace

// Tensor map of a channel-last bf16 activation buffer (16 channels per cell) of lattice L: dims
// (channel, i, j, k), box 16 x 8 x 18 x 1 (one staged plane of the convolution tile with its j
// halo), 32-byte swizzle, zero fill outside the lattice.
int make_act_tensor_map(CUtensorMap* map, const __nv_bfloat16* base, const Lat& L) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) { set_error("cuTensorMapEncodeTiled is not available from the driver"); return 1; }
    if (((uintptr_t)base & 15u) != 0) { set_error("activation buffer is not 16-byte aligned"); return 1; }
    cuuint64_t dims[4] = {16, (cuuint64_t)L.nI, (cuuint64_t)L.nJ, (cuuint64_t)L.nK};
    cuuint64_t strides[3] = {32, (cuuint64_t)32 * L.nI, (cuuint64_t)32 * L.nI * L.nJ};   // bytes, dims 1..3
    cuuint32_t box[4] = {16, (cuuint32_t)TI, (cuuint32_t)ROWS, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"); return 1; }
    return 0;
}

namespace {
// encoded maps are kept per (buffer, lattice): the solves reuse the same few activation buffers
const CUtensorMap* cached_map(const __nv_bfloat16* in, const Lat& L) {
    static std::vector<std::pair<std::array<long long, 4>, CUtensorMap>> cache;
    static std::mutex cacheLock;
    std::lock_guard<std::mutex> guard(cacheLock);
    const std::array<long long, 4> key = {(long long)(uintptr_t)in, L.nI, L.nJ, L.nK};
    for (auto& e : cache)
        if (e.first == key) return &e.second;
    CUtensorMap m;
    if (make_act_tensor_map(&m, in, L)) return nullptr;
    cache.emplace_back(key, m);
    return &cache.back().second;
}
}  // namespace

int launch_conv3d_group(int epi, const ConvSpec* specs, int n, const __nv_bfloat16* wpack, const float* bias, int* err, cudaStream_t st,
                        const int* skip) {
    const size_t smem = conv_smem_bytes();
    static bool attr = false;
    if (!attr) {
        CB_CUDA(cudaFuncSetAttribute(conv3d_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CB_CUDA(cudaFuncSetAttribute(conv3d_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CB_CUDA(cudaFuncSetAttribute(conv3d_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    for (int b = 0; b < n; b += CONV_MAX_JOBS) {
        ConvGroup g;
        std::memset(&g, 0, sizeof(g));
        g.n = std::min(CONV_MAX_JOBS, n - b);
        long long ctas = 0;
        for (int p = 0; p < g.n; ++p) {
            const ConvSpec& sp = specs[b + p];
            const Lat& L = sp.L;
            const CUtensorMap* mp = cached_map(sp.in, L);
            if (!mp) return 1;
            ConvJob& J = g.job[p];
            J.map = *mp;
            J.L = L;
            J.out_bf = sp.out_bf; J.out_f = sp.out_f; J.mask = sp.mask;
            J.gx = (L.nI + TI - 1) / TI;
            J.gy = (L.nJ + TJ - 1) / TJ;
            // k-planes per CTA: up to 16 (one staged plane serves three output planes), fewer on
            // small lattices so that the job alone would still cover the SMs twice
            const long long kc = (long long)J.gx * J.gy * L.nK / 296;
            J.KC = (int)(kc < 1 ? 1 : (kc > 16 ? 16 : kc));
            ctas += (long long)J.gx * J.gy * ((L.nK + J.KC - 1) / J.KC);
            if (ctas > (1ll << 30)) { set_error("convolution group too large"); return 1; }
            g.ctaEnd[p] = (int)ctas;
        }
        const unsigned grid = (unsigned)ctas;
        if (epi == 0) conv3d_tc_kernel<0><<<grid, CONV_THREADS, smem, st>>>(g, wpack, bias, err, skip);
        else if (epi == 1) conv3d_tc_kernel<1><<<grid, CONV_THREADS, smem, st>>>(g, wpack, bias, err, skip);
        else conv3d_tc_kernel<2><<<grid, CONV_THREADS, smem, st>>>(g, wpack, bias, err, skip);
        CB_CHECK_LAUNCH();
    }
    return 0;
}

int launch_conv3d(const Lat& L, int epi, const __nv_bfloat16* in, const __nv_bfloat16* wpack, const float* bias, __nv_bfloat16* out_bf,
                  float* out_f, const __nv_bfloat16* mask_act, int* err, cudaStream_t st, const int* skip) {
    ConvSpec sp;
    sp.L = L; sp.in = in; sp.out_bf = out_bf; sp.out_f = out_f; sp.mask = mask_act;
    return launch_conv3d_group(epi, &sp, 1, wpack, bias, err, st, skip);
}

}  // namespace cb
