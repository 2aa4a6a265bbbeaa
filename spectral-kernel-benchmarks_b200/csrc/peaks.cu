// SIMT FMA throughput of the current device (FP32 and FP64), measured.
//
// The FFT, pointwise and FP64-plain kernels of this library run on the SIMT
// pipes, whose peaks a measured copy bandwidth and a cuBLAS GEMM rate do not
// cover; their rooflines use these numbers instead of datasheet figures.

#include "peaks.hpp"

#include <cuda_runtime.h>

#include <algorithm>

namespace skb {
namespace {

constexpr int kChains = 8;  // independent FMA chains per thread

// Every thread runs kChains dependent chains a = fma(a, b, c) for `iters`
// rounds (2 flops per FMA).  With |b| < 1 the chains converge to
// c / (1 - b), so no value overflows or turns subnormal.
template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T* out, int iters, T b, T c) {
    T a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = T(threadIdx.x % 7 + i) * T(0.125);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], b, c);
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i];
    out[static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

template <typename T>
cudaError_t time_chains(int blocks, int iters, double* tflops) {
    T* out = nullptr;
    cudaError_t err = cudaMalloc(&out, sizeof(T) * static_cast<size_t>(blocks) * 256);
    if (err != cudaSuccess) return err;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {  // first run untimed
        cudaEventRecord(e0, s);
        fma_chain_kernel<T><<<blocks, 256, 0, s>>>(out, iters, T(0.999999), T(1e-6));
        cudaEventRecord(e1, s);
        err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess && rep > 0 && ms > 0.f) {
            const double flops = 2.0 * kChains * static_cast<double>(iters) * blocks * 256.0;
            best = std::max(best, flops / (ms * 1e-3) / 1e12);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(out);
    if (err == cudaSuccess) *tflops = best;
    return err;
}

}  // namespace

cudaError_t measure_simt_peaks(double* fp32Tflops, double* fp64Tflops) {
    int device = 0, sms = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess) return err;
    // Eight 256-thread blocks per SM (full occupancy at these few registers);
    // rounds sized for runs of roughly 10-20 ms on a B200.
    const int blocks = 8 * std::max(sms, 1);
    err = time_chains<float>(blocks, 1 << 16, fp32Tflops);
    if (err == cudaSuccess) err = time_chains<double>(blocks, 1 << 14, fp64Tflops);
    return err;
}

}  // namespace skb
