#pragma once

#include <cuda_runtime.h>

namespace skb {

// Best-of-three FP32 and FP64 FMA throughput (TFLOP/s, 2 flops per FMA) of the
// current device, from independent FMA chains at full occupancy.
cudaError_t measure_simt_peaks(double* fp32Tflops, double* fp64Tflops);

}  // namespace skb
