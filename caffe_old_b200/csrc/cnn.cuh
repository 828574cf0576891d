// Learned preconditioner network: a 4-layer 3-D convolutional network, 3x3x3 kernels,
// 16 channels, BF16 weights and activations with FP32 accumulation.
//   input  x0: 16 channels, channel 0 = Jacobi-scaled residual / its RMS, channel 1 = active-cell mask
//   layer 1..3: conv + bias + ReLU (16 -> 16 channels)
//   layer 4:    conv + bias, output channel 0 (y)
// Parameters (FP32 master copy): for each layer l = 0..3, W_l[27][16 out][16 in] then b_l[16];
// tap t = 9*(dk+1) + 3*(dj+1) + (di+1) for offsets dk, dj, di in {-1, 0, 1} along k, j, i.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace cb {

constexpr int NET_LAYERS = 4;
constexpr int NET_C = 16;
constexpr int NET_LAYER_PARAMS = 27 * 16 * 16 + 16;
constexpr int NET_PARAMS = NET_LAYERS * NET_LAYER_PARAMS;

size_t conv_smem_bytes();
// epi 0: bias + ReLU -> bf16;  1: bias -> FP32 channel 0;  2: times (mask_act > 0) -> bf16
// skip: optional device flag; while it holds non-zero the launch does nothing
int launch_conv3d(const Lat& L, int epi, const __nv_bfloat16* in, const __nv_bfloat16* wpack, const float* bias, __nv_bfloat16* out_bf,
                  float* out_f, const __nv_bfloat16* mask_act, int* err, cudaStream_t st, const int* skip = nullptr);

// One convolution layer over several lattices in one launch (the same weights and epilogue):
// input activations in, bf16 activations out (epi 0 / 2) or FP32 channel 0 out (epi 1), the
// ReLU mask of epi 2.
constexpr int CONV_MAX_JOBS = 16;
struct ConvSpec {
    Lat L;
    const __nv_bfloat16* in;
    __nv_bfloat16* out_bf;
    float* out_f;
    const __nv_bfloat16* mask;
};
int launch_conv3d_group(int epi, const ConvSpec* specs, int n, const __nv_bfloat16* wpack, const float* bias, int* err, cudaStream_t st,
                        const int* skip = nullptr);

// Weight gradient of one layer on the tensor cores: dW[t][o][i] += sum_c x[c + off(t)][i] dz[c][o],
// db[o] += sum_c dz[c][o] (FP32, accumulated into dW / db).
int launch_weight_grad(const Lat& L, const __nv_bfloat16* x, const __nv_bfloat16* dz, float* dW, float* db, int* err, cudaStream_t st);

// Device buffers of one network applied on one lattice.
struct NetBuffers {
    Lat L;
    __nv_bfloat16* act[4];      // x0 .. x3 (N x 16 each)
    __nv_bfloat16* gz[2];       // backward ping-pong (N x 16 each)
    __nv_bfloat16* wfwd;        // 4 x 27 x 512 bytes, forward packing
    __nv_bfloat16* wbwd;        // 4 x 27 x 512 bytes, transposed + flipped packing (backward data)
    float* params;              // NET_PARAMS (device master copy)
    float* grad;                // NET_PARAMS
    float* y;                   // N: network output
    int* err;
};

int net_alloc(NetBuffers& nb, const Lat& L, void* (*alloc)(size_t, void*), void* ctx);
// activations of another lattice that share the weights, gradient and error flag of `owner`
int net_alloc_shared(NetBuffers& nb, const Lat& L, const NetBuffers& owner, void* (*alloc)(size_t, void*), void* ctx);
int net_pack_weights(NetBuffers& nb, cudaStream_t st);
// forward from the packed 16-channel input already in act[0]; output in nb.y
int net_forward(NetBuffers& nb, cudaStream_t st);
// same, every launch a no-op while *skip is non-zero
int net_forward_if(NetBuffers& nb, const int* skip, cudaStream_t st);
// the forward passes of several networks that share one set of weights (nets[0]'s), one
// launch per layer for all of them
int net_forward_group_if(NetBuffers* const* nets, int n, const int* skip, cudaStream_t st);
// backward for dL/dy (FP32, N): accumulates dL/dparams into nb.grad
int net_backward(NetBuffers& nb, const float* dy, cudaStream_t st);
// act[0] from a 2-channel FP32 input laid out [N][2]
int net_pack_input2(NetBuffers& nb, const float* x2, cudaStream_t st);

}  // namespace cb
