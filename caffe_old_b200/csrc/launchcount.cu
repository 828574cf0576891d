// Launch counter: the library is linked with --wrap=cudaLaunchKernel and
// --wrap=cudaLaunchCooperativeKernel, so every kernel launch issued by this library (the
// <<<...>>> syntax compiles to cudaLaunchKernel) passes through these functions, which
// count it and forward to the CUDA runtime unchanged.
#include <atomic>
#include <cuda_runtime.h>

extern "C" {
cudaError_t __real_cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream);
cudaError_t __real_cudaLaunchCooperativeKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream);
}

namespace {
std::atomic<long long> g_launches{0};
}

extern "C" {
cudaError_t __wrap_cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return __real_cudaLaunchKernel(func, grid, block, args, smem, stream);
}
cudaError_t __wrap_cudaLaunchCooperativeKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return __real_cudaLaunchCooperativeKernel(func, grid, block, args, smem, stream);
}

long long caffe_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
}
