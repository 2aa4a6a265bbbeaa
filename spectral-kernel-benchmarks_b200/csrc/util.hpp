// Small element-wise device helpers used by the host adapters.
#pragma once

#include <cuda_runtime.h>

namespace skb {

// dst[i] = (float)src[i] or (double)src[i].
cudaError_t launch_convert_f64_to_f32(const double* src, float* dst, long long n, cudaStream_t s);
cudaError_t launch_convert_f32_to_f64(const float* src, double* dst, long long n, cudaStream_t s);
// Complex interleaved <-> split arrays; T is double when f64, float otherwise.
cudaError_t launch_split(bool f64, const void* interleaved, void* re, void* im, long long n, cudaStream_t s);
cudaError_t launch_interleave(bool f64, const void* re, const void* im, void* interleaved, long long n,
                              cudaStream_t s);

}  // namespace skb
