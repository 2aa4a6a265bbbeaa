// Allocation-free dense 2-D c2r inverse over a fixed static device array.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "model.hpp"
#include "runtime.hpp"

namespace skb {

// Size of the static scratch array every GPU that loads the library holds.
std::size_t static_inverse_scratch_limit();
// Scratch one call needs: three twiddle tables and the column spectrum.
std::size_t static_inverse_scratch_bytes(const Workload& w, Precision p);
// WVM spectrum [ky][kx][field][z] -> real [field][z][y][x], unnormalised,
// on stream s; throws Error(-1) when the workload needs more scratch than the
// array holds.  Calls whose GPU work overlaps race on the shared array.
void inverse_dense_static(const Workload& w, Precision p, const void* wvm, void* real, cudaStream_t s);

}  // namespace skb
