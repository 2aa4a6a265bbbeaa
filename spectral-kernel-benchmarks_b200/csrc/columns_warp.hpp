// Warp-per-plane FP32 column stages of the fused flux (embed + inverse c2c,
// forward c2c + retention).
#pragma once

#include <cuda_runtime.h>

#include "horizontal.hpp"

namespace skb {

// Power-of-two Ny in [32, 512].
bool columns_warp_supported(long long ny);
// Same contracts as launch_columns_embed / launch_columns_gather for FP32.
cudaError_t launch_columns_embed_warp(int ny, int nz, int columns, const ViewSet& views, const ModeTables& tables,
                                      DenseBins out, const void* tw, cudaStream_t s);
cudaError_t launch_columns_gather_warp(int ny, int nz, int columns, DenseBins in, const ViewSet& views,
                                       const ModeTables& tables, double scale, const void* tw, cudaStream_t s);

}  // namespace skb
