// Synthetic modal work of the spectral pipeline: complex values scaled by real
// weights (applySyntheticModalWorkInterleaved, model.cpp:269-274).  HBM-bound:
// one complex read, one real weight read and one complex write per element.

#include "pipeline.hpp"

#include "fft_device.cuh"

namespace skb {
namespace {

template <typename T>
__global__ void modal_work_kernel(const T* __restrict__ weights, const cx<T>* __restrict__ in, cx<T>* out,
                                  long long count) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
        const T w = __ldg(weights + i);
        const cx<T> v = in[i];
        out[i] = {w * v.x, w * v.y};
    }
}

}  // namespace

cudaError_t launch_modal_work(Precision p, const void* weights, const void* in, void* out, long long count,
                              cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int threads = 256;
    const long long blocks = std::min<long long>((count + threads - 1) / threads, 148LL * 16);
    if (p == Precision::f64)
        modal_work_kernel<double><<<unsigned(blocks), threads, 0, s>>>(
            static_cast<const double*>(weights), static_cast<const double2*>(in), static_cast<double2*>(out), count);
    else
        modal_work_kernel<float><<<unsigned(blocks), threads, 0, s>>>(
            static_cast<const float*>(weights), static_cast<const float2*>(in), static_cast<float2*>(out), count);
    return cudaGetLastError();
}

}  // namespace skb
