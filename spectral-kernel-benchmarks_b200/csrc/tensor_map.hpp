// TMA tensor maps (CUtensorMap) for this GPU's own device memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace skb {

// A 2-D tiled map over 8-byte elements (complex FP32): dim0 = `inner`
// contiguous elements, dim1 = `outer` rows `rowBytes` apart, boxes of
// boxInner x boxOuter elements, zero fill outside the tensor, swizzled so
// that a box row of 64 or 128 bytes (boxInner = 8 or 16) lands in the
// SWIZZLE_64B / SWIZZLE_128B shared-memory pattern.  Returns
// cudaErrorInvalidValue for shapes a tensor map cannot describe (base or
// row pitch not 16-byte aligned, box outside 1..256) and
// cudaErrorNotSupported when the driver does not export the encoder.
cudaError_t encode_complex_map_2d(CUtensorMap* map, const void* base, unsigned long long inner,
                                  unsigned long long outer, unsigned long long rowBytes, unsigned boxInner,
                                  unsigned boxOuter);

}  // namespace skb
