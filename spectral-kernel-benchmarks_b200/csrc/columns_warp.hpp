// Warp-per-plane FP32 column stages of the fused flux (embed + inverse c2c,
// forward c2c + retention).
#pragma once

#include <cuda_runtime.h>

#include "horizontal.hpp"

namespace skb {

// Power-of-two Ny in [32, 512].
bool columns_warp_supported(long long ny);
// Same contracts as launch_columns_embed / launch_columns_gather for FP32,
// except that view f's planes start at bin plane f * zStride (zStride >= nz;
// padding planes are neither read nor written).
cudaError_t launch_columns_embed_warp(int ny, int nz, int zStride, int columns, const ViewSet& views, const ModeTables& tables,
                                      DenseBins out, const void* tw, cudaStream_t s);
cudaError_t launch_columns_gather_warp(int ny, int nz, int zStride, int columns, DenseBins in, const ViewSet& views,
                                       const ModeTables& tables, double scale, const void* tw, cudaStream_t s);

// Band forms, in place on dense bins [ky][kx < columns][plane] (plane of slot
// f: f * zStride + z): band[kx] bounds the retained cells of column kx
// (min(ky, Ny - ky) <= band[kx]).  Inverse: band cells in, whole column out.
// Forward: whole column in, band cells (times scale) out.
// Band kernel forms: kBandDefault is the direct three-pass kernel at Ny = 512
// and the warp-per-plane kernel below; kBandWarp selects the warp-per-plane
// kernel at every size; kBandPersist the persistent direct kernel (Ny = 512
// only), which loads the next tile during the current one's passes;
// kBandDirect4 the direct kernel compiled for four resident CTAs per SM
// instead of three (at most 64 registers a thread), for more loads in flight.
// The forms at 512 are autotuner candidates.
constexpr int kBandDefault = 0;
constexpr int kBandWarp = 1;
constexpr int kBandPersist = 2;
constexpr int kBandDirect4 = 3;
// kBand16: the direct kernel with 16 planes per CTA over the flat plane index
// (128-byte global accesses per ky row; Ny = 512).
constexpr int kBand16 = 4;
// kBand32: the same with 32 planes per CTA (256-byte accesses, one CTA per SM).
constexpr int kBand32 = 5;
// kBand16Pipe16/32/64: the 16-plane form with one CTA per SM walking 16, 32
// or 64 kx columns, the next column's loads in flight during the current
// one's passes.
constexpr int kBand16Pipe16 = 6;
constexpr int kBand16Pipe32 = 7;
constexpr int kBand16Pipe64 = 8;
constexpr int band_pipe_columns(int form) {
    return form == kBand16Pipe16 ? 16 : form == kBand16Pipe32 ? 32 : form == kBand16Pipe64 ? 64 : 0;
}
cudaError_t launch_columns_inverse_band(int ny, int nz, int zStride, int slots, int columns, DenseBins bins,
                                        const int* band, const void* tw, int form, cudaStream_t s);
cudaError_t launch_columns_forward_band(int ny, int nz, int zStride, int slots, int columns, DenseBins bins,
                                        const int* band, double scale, const void* tw, int form, cudaStream_t s);

}  // namespace skb
