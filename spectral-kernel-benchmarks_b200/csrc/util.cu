#include "util.hpp"

#include "fft_device.cuh"

namespace skb {
namespace {

template <typename S, typename D>
__global__ void convert_kernel(const S* __restrict__ src, D* __restrict__ dst, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = D(src[i]);
}

template <typename T>
__global__ void split_kernel(const cx<T>* __restrict__ in, T* __restrict__ re, T* __restrict__ im, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const cx<T> v = in[i];
        re[i] = v.x;
        im[i] = v.y;
    }
}

template <typename T>
__global__ void interleave_kernel(const T* __restrict__ re, const T* __restrict__ im, cx<T>* __restrict__ out,
                                  long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = {re[i], im[i]};
}

unsigned blocks_for(long long n) {
    const long long b = (n + 255) / 256;
    return unsigned(b < 4096 ? (b < 1 ? 1 : b) : 4096);
}

}  // namespace

cudaError_t launch_convert_f64_to_f32(const double* src, float* dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    convert_kernel<double, float><<<blocks_for(n), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_convert_f32_to_f64(const float* src, double* dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    convert_kernel<float, double><<<blocks_for(n), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_split(bool f64, const void* interleaved, void* re, void* im, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (f64)
        split_kernel<double><<<blocks_for(n), 256, 0, s>>>(static_cast<const double2*>(interleaved),
                                                           static_cast<double*>(re), static_cast<double*>(im), n);
    else
        split_kernel<float><<<blocks_for(n), 256, 0, s>>>(static_cast<const float2*>(interleaved),
                                                          static_cast<float*>(re), static_cast<float*>(im), n);
    return cudaGetLastError();
}

cudaError_t launch_interleave(bool f64, const void* re, const void* im, void* interleaved, long long n,
                              cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (f64)
        interleave_kernel<double><<<blocks_for(n), 256, 0, s>>>(static_cast<const double*>(re),
                                                                static_cast<const double*>(im),
                                                                static_cast<double2*>(interleaved), n);
    else
        interleave_kernel<float><<<blocks_for(n), 256, 0, s>>>(static_cast<const float*>(re),
                                                               static_cast<const float*>(im),
                                                               static_cast<float2*>(interleaved), n);
    return cudaGetLastError();
}

}  // namespace skb
