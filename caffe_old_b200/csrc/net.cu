// Network plumbing around the tensor-core convolution: weight packing, input packing,
// forward and backward passes, weight gradients, and C entry points that run the network
// on host data (used to check the kernels against an FP64 CPU restatement).
#include <cuda_bf16.h>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/caffe_b200.h"
#include "common.cuh"
#include "cnn.cuh"

namespace cb {

namespace {

__device__ __forceinline__ int canon(int n, int k) {  // element offset of (row n, col k) in a 16x16 canonical K-major block
    return (n >> 3) * 128 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
}

// forward: block t of layer l holds W_l[t][out][in] as rows = out, K = in.
// backward data: block t' holds W_l[26 - t'][in][out]^T, i.e. rows = in, K = out.
__global__ void pack_weights_kernel(const float* __restrict__ params, __nv_bfloat16* wf, __nv_bfloat16* wb) {
    int l = blockIdx.y;
    int t = blockIdx.x;   // 27 blocks
    const float* W = params + (size_t)l * NET_LAYER_PARAMS;
    for (int e = threadIdx.x; e < 256; e += blockDim.x) {
        int o = e >> 4, i = e & 15;
        float v = W[(t * 16 + o) * 16 + i];
        wf[((size_t)l * 27 + t) * 256 + canon(o, i)] = __float2bfloat16_rn(v);
        // transposed + flipped: rows = in (i), K = out (o), tap 26 - t
        wb[((size_t)l * 27 + (26 - t)) * 256 + canon(i, o)] = __float2bfloat16_rn(v);
    }
}

__global__ void pack_input2_kernel(long long N, const float* __restrict__ x2, __nv_bfloat16* act0) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    __align__(16) __nv_bfloat16 v[16];
    v[0] = __float2bfloat16_rn(x2[2 * c]);
    v[1] = __float2bfloat16_rn(x2[2 * c + 1]);
    for (int q = 2; q < 16; ++q) v[q] = __float2bfloat16_rn(0.f);
    uint4* dst = reinterpret_cast<uint4*>(act0 + c * 16);
    dst[0] = reinterpret_cast<uint4*>(v)[0];
    dst[1] = reinterpret_cast<uint4*>(v)[1];
}

__global__ void pack_dy_kernel(long long N, const float* __restrict__ dy, __nv_bfloat16* gz) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    __align__(16) __nv_bfloat16 v[16];
    v[0] = __float2bfloat16_rn(dy[c]);
    for (int q = 1; q < 16; ++q) v[q] = __float2bfloat16_rn(0.f);
    uint4* dst = reinterpret_cast<uint4*>(gz + c * 16);
    dst[0] = reinterpret_cast<uint4*>(v)[0];
    dst[1] = reinterpret_cast<uint4*>(v)[1];
}

}  // namespace

int net_alloc(NetBuffers& nb, const Lat& L, void* (*alloc)(size_t, void*), void* ctx) {
    nb.L = L;
    size_t actBytes = (size_t)L.N * 16 * sizeof(__nv_bfloat16);
    for (int q = 0; q < 4; ++q) nb.act[q] = static_cast<__nv_bfloat16*>(alloc(actBytes, ctx));
    for (int q = 0; q < 2; ++q) nb.gz[q] = static_cast<__nv_bfloat16*>(alloc(actBytes, ctx));
    nb.wfwd = static_cast<__nv_bfloat16*>(alloc((size_t)NET_LAYERS * 27 * 512, ctx));
    nb.wbwd = static_cast<__nv_bfloat16*>(alloc((size_t)NET_LAYERS * 27 * 512, ctx));
    nb.params = static_cast<float*>(alloc(sizeof(float) * NET_PARAMS, ctx));
    nb.grad = static_cast<float*>(alloc(sizeof(float) * NET_PARAMS, ctx));
    nb.y = static_cast<float*>(alloc(sizeof(float) * (size_t)L.N, ctx));
    nb.err = static_cast<int*>(alloc(sizeof(int) * 4, ctx));
    bool ok = nb.wfwd && nb.wbwd && nb.params && nb.grad && nb.y && nb.err;
    for (int q = 0; q < 4; ++q) ok = ok && nb.act[q];
    for (int q = 0; q < 2; ++q) ok = ok && nb.gz[q];
    if (!ok) { set_error("network buffer allocation failed"); return 1; }
    return 0;
}

int net_alloc_shared(NetBuffers& nb, const Lat& L, const NetBuffers& owner, void* (*alloc)(size_t, void*), void* ctx) {
    nb.L = L;
    size_t actBytes = (size_t)L.N * 16 * sizeof(__nv_bfloat16);
    bool ok = true;
    for (int q = 0; q < 4; ++q) ok = ok && (nb.act[q] = static_cast<__nv_bfloat16*>(alloc(actBytes, ctx)));
    for (int q = 0; q < 2; ++q) ok = ok && (nb.gz[q] = static_cast<__nv_bfloat16*>(alloc(actBytes, ctx)));
    ok = ok && (nb.y = static_cast<float*>(alloc(sizeof(float) * (size_t)L.N, ctx)));
    if (!ok) { set_error("network buffer allocation failed"); return 1; }
    nb.wfwd = owner.wfwd; nb.wbwd = owner.wbwd; nb.params = owner.params; nb.grad = owner.grad; nb.err = owner.err;
    return 0;
}

int net_pack_weights(NetBuffers& nb, cudaStream_t st) {
    pack_weights_kernel<<<dim3(27, NET_LAYERS), 256, 0, st>>>(nb.params, nb.wfwd, nb.wbwd);
    CB_CHECK_LAUNCH();
    return 0;
}

int net_pack_input2(NetBuffers& nb, const float* x2, cudaStream_t st) {
    pack_input2_kernel<<<grid_for(nb.L.N, 256), 256, 0, st>>>(nb.L.N, x2, nb.act[0]);
    CB_CHECK_LAUNCH();
    return 0;
}

static const float* bias_of(const NetBuffers& nb, int l) { return nb.params + (size_t)l * NET_LAYER_PARAMS + 27 * 256; }
static const __nv_bfloat16* wf_of(const NetBuffers& nb, int l) { return nb.wfwd + (size_t)l * 27 * 256; }
static const __nv_bfloat16* wb_of(const NetBuffers& nb, int l) { return nb.wbwd + (size_t)l * 27 * 256; }

int net_forward_if(NetBuffers& nb, const int* skip, cudaStream_t st) {
    for (int l = 0; l < 3; ++l)
        if (launch_conv3d(nb.L, 0, nb.act[l], wf_of(nb, l), bias_of(nb, l), nb.act[l + 1], nullptr, nullptr, nb.err, st, skip)) return 1;
    return launch_conv3d(nb.L, 1, nb.act[3], wf_of(nb, 3), bias_of(nb, 3), nullptr, nb.y, nullptr, nb.err, st, skip);
}

int net_forward(NetBuffers& nb, cudaStream_t st) { return net_forward_if(nb, nullptr, st); }

int net_forward_group_if(NetBuffers* const* nets, int n, const int* skip, cudaStream_t st) {
    if (n < 1) return 0;
    std::vector<ConvSpec> sp((size_t)n);
    for (int l = 0; l < NET_LAYERS; ++l) {
        for (int q = 0; q < n; ++q) {
            NetBuffers& nb = *nets[q];
            if (nb.wfwd != nets[0]->wfwd) { set_error("grouped networks must share their weights"); return 1; }
            sp[q].L = nb.L;
            sp[q].in = nb.act[l];
            sp[q].out_bf = l < NET_LAYERS - 1 ? nb.act[l + 1] : nullptr;
            sp[q].out_f = l < NET_LAYERS - 1 ? nullptr : nb.y;
            sp[q].mask = nullptr;
        }
        if (launch_conv3d_group(l < NET_LAYERS - 1 ? 0 : 1, sp.data(), n, wf_of(*nets[0], l), bias_of(*nets[0], l), nets[0]->err, st, skip))
            return 1;
    }
    return 0;
}

static int weight_grad(NetBuffers& nb, int l, const __nv_bfloat16* x, const __nv_bfloat16* dz, cudaStream_t st) {
    float* g = nb.grad + (size_t)l * NET_LAYER_PARAMS;
    return launch_weight_grad(nb.L, x, dz, g, g + 27 * 256, nb.err, st);
}

int net_backward(NetBuffers& nb, const float* dy, cudaStream_t st) {
    const Lat& L = nb.L;
    pack_dy_kernel<<<grid_for(L.N, 256), 256, 0, st>>>(L.N, dy, nb.gz[0]);
    CB_CHECK_LAUNCH();
    int a = 0;
    for (int l = 3; l >= 0; --l) {
        if (weight_grad(nb, l, nb.act[l], nb.gz[a], st)) return 1;
        if (l == 0) break;
        // dL/dz of layer l-1 = (W_l^T applied to dz_l) where the layer's input was positive
        if (launch_conv3d(L, 2, nb.gz[a], wb_of(nb, l), nullptr, nb.gz[a ^ 1], nullptr, nb.act[l], nb.err, st)) return 1;
        a ^= 1;
    }
    return 0;
}

}  // namespace cb

using namespace cb;

namespace {

struct TmpAlloc {
    std::vector<void*> ptrs;
    static void* fn(size_t bytes, void* ctx) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes + 256) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, bytes + 256);
        static_cast<TmpAlloc*>(ctx)->ptrs.push_back(p);
        return p;
    }
    ~TmpAlloc() { for (void* p : ptrs) cudaFree(p); }
};

int run_host_net(int nI, int nJ, int nK, const float* params, const float* x2, const float* dy, float* y, float* dparams) {
    if (nI < 1 || nJ < 1 || nK < 1 || !params || !x2 || !y) { set_error("invalid arguments"); return 1; }
    Lat L = make_lat(nI, nJ, nK);
    TmpAlloc ta;
    NetBuffers nb;
    if (net_alloc(nb, L, &TmpAlloc::fn, &ta)) return 1;
    float* dx2 = static_cast<float*>(TmpAlloc::fn(sizeof(float) * 2 * L.N, &ta));
    float* ddy = dy ? static_cast<float*>(TmpAlloc::fn(sizeof(float) * L.N, &ta)) : nullptr;
    if (!dx2 || (dy && !ddy)) { set_error("allocation failed"); return 1; }
    CB_CUDA(cudaMemcpy(nb.params, params, sizeof(float) * NET_PARAMS, cudaMemcpyHostToDevice));
    CB_CUDA(cudaMemcpy(dx2, x2, sizeof(float) * 2 * L.N, cudaMemcpyHostToDevice));
    if (dy) CB_CUDA(cudaMemcpy(ddy, dy, sizeof(float) * L.N, cudaMemcpyHostToDevice));
    if (net_pack_weights(nb, 0) || net_pack_input2(nb, dx2, 0) || net_forward(nb, 0)) return 1;
    if (dy && net_backward(nb, ddy, 0)) return 1;
    CB_CUDA(cudaDeviceSynchronize());
    int herr = 0;
    CB_CUDA(cudaMemcpy(&herr, nb.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) { set_error("tensor-core convolution: an MMA completion wait timed out"); return 1; }
    CB_CUDA(cudaMemcpy(y, nb.y, sizeof(float) * L.N, cudaMemcpyDeviceToHost));
    if (dy && dparams) CB_CUDA(cudaMemcpy(dparams, nb.grad, sizeof(float) * NET_PARAMS, cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace

extern "C" {

int caffe_precond_param_count(void) { return NET_PARAMS; }

int caffe_precond_net_apply(int nI, int nJ, int nK, const float* params, const float* x2, float* y) {
    return run_host_net(nI, nJ, nK, params, x2, nullptr, y, nullptr);
}

int caffe_precond_net_grad(int nI, int nJ, int nK, const float* params, const float* x2, const float* dy, float* y, float* dparams) {
    if (!dy || !dparams) { set_error("invalid arguments"); return 1; }
    return run_host_net(nI, nJ, nK, params, x2, dy, y, dparams);
}

}  // extern "C"
