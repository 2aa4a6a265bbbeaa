#pragma once

#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

namespace skb {

// target = -scale*(u*qx + v*qy + w*qz) over `volume` points; shared = [u,v,w],
// derivative = [qx,qy,qz] volume-strided (pointwise_advection.cpp:143-147).
cudaError_t launch_pointwise(bool f64, long long volume, double scale, const void* shared, const void* derivative,
                             void* target, int smCount, cudaStream_t stream);

}  // namespace skb
