// Fused row stage of the split-precision flux (flux_rows.cu).
#pragma once

#include <cuda_runtime.h>

#include "horizontal.hpp"

namespace skb {

struct RowFluxArgs {
    int nx, ny, nz, keep;
    int zStride;          // bin planes per slot (>= nz; z-padding keeps each slot's planes 64-byte aligned)
    int members, fieldsIn, targets;
    float scale;          // 1/(Nx*Ny)^2 (benchmark.cpp:4040-4041)
    DenseBins binsIn;     // column-transformed input slots, plane (member*fieldsIn + slot)*zStride + z
    DenseBins binsOut;    // target bins, plane (member*targets + t)*zStride + z
    const void* twHalf;   // exp(-2 pi i k/(nx/2)), float2
    const void* twFull;   // exp(-2 pi i k/nx), float2
    int planes = 8;       // z-planes per CTA: 4, 8 or 16, and 24 for the two-planes-per-warp form (an autotuner choice)
    // Nx = 512 only: two planes per warp (16 lanes each, 16 x-pairs per lane)
    // with a radix-16 x radix-16 FFT; needs planes 8 or 16 (autotuner choice).
    // 2: the 8-plane form compiled for three resident CTAs per SM.
    int pairs = 0;
    // Two-planes-per-warp forms only: 1 fills each slot's stage with one TMA
    // tensor copy instead of per-thread cp.async, one slot ahead; 2 does so
    // two slots ahead through three stages (an autotuner choice; needs
    // `error`).
    int tma = 0;
    int* error = nullptr;  // device word set to 1 when a bounded wait expires
    // Test of the failure path (TMA forms): thread 0 of every CTA also waits,
    // briefly and bounded, on a barrier nothing signals, after slot 0's copy.
    int expireWaitForTest = 0;
};

bool rows_flux_supported(long long nx);
cudaError_t launch_rows_flux(const RowFluxArgs& a, cudaStream_t stream);

}  // namespace skb
