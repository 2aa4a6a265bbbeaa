// K^2-grouped vertical modal GEMM (vertical_gemm.cpp:534-596 of the reference).
//
// For every K^2 group g with complex columns c in [c0_g, c0_g + n_g) (column
// = field + fields*mode, so a group's columns are contiguous):
//     out[c][r] = sum_s A_g[r][s] * in[c][s]
// with A_g real, R x S, row-major.  Forward: A = F_g (Nj x Nz), in = physical
// retained spectra [mode][field][z], out = modal [mode][field][j].  Inverse:
// A = I_g (Nz x Nj) and the roles swap.  Real and imaginary parts share the
// matrix (the reference's split form: two real GEMMs per group).

#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace skb {

enum class GemmPrecision { f64 = 0, f32 = 1, tf32x3 = 2, bf16x3 = 3 };

// SIMT tiles, in one of two numberings.
// Member tiles (virtual == false): a tile is up to the tile width of one
// member's columns of one group; tileColumn is its first global complex
// column (member * memberColumns + column within the member).
// Virtual tiles (virtual == true): runs of the (member, column) list of one
// group, numbered like the tensor-core work units below: virtual column v of
// group g is member v / groupColumns[g], complex column
// groupFirst[g] + v % groupColumns[g] of that member.  Concatenating the
// members keeps a group's tiles full when it has few columns per member (a
// field subset, small groups); each tile carries its group's groupColumns /
// groupFirst so that a CTA's first loads do not wait on a dependent read.
struct GroupTiles {
    const int* tileGroup;     // K^2 group of each CTA tile
    const int* tileColumn;    // first global (member tiles) or virtual column of each tile
    const int* tileCount;     // columns in each tile (<= tile width)
    const int* tilePer;       // virtual tiles: groupColumns of the tile's group
    const int* tileFirst;     // virtual tiles: groupFirst of the tile's group
    int tiles;
    long long memberColumns;  // complex columns per member
    long long matrixStride;   // elements between group matrices (0: one matrix for all groups)
    bool virtualColumns;      // the numbering of tileColumn
};

// Operand element: complex interleaved (im == nullptr) or split re/im arrays.
struct ComplexOperand {
    void* re;
    void* im;
};

// Column tile width (complex columns per CTA) used to build GroupTiles.
int gemm_tile_columns(GemmPrecision p);

// Tensor-core split-TF32x3 form (tc_gemm.cu).  Work units are runs of the
// (member, column) list of one group: virtual column v of group g is member
// v / groupColumns[g], column groupFirst[g] + v % groupColumns[g] of that
// member, i.e. global complex column member*memberColumns + ...
// Optional cell-addressed operand instead of the compact [column][len] array
// (the fused flux's dense bin arrays, full WVM-order spectra, or a field
// subset of a compact array).  Plan column (member, mode, f) lives at element
//   cell[mode] + member * memberStride + field * zStride + i   (i along the column)
// with field = fieldMap[f] (f itself without a map) and memberStride =
// fields * zStride when left 0.  conj[mode] != 0 where the cell holds the
// conjugate of the value; partner[mode] >= 0 (output side) is a second cell,
// the kx = 0 Hermitian partner, that receives the conjugate of the value.
struct BinBoundary {
    const long long* cell = nullptr;  // nullptr: compact operand
    const long long* partner = nullptr;
    const unsigned char* conj = nullptr;
    int fields = 1;              // plan fields per mode
    int zStride = 0;             // elements between consecutive stored fields
    long long memberStride = 0;  // elements between members (0: fields * zStride)
    const int* fieldMap = nullptr;  // plan field -> stored field (nullptr: identity)
    long long memberColumns = 0;    // plan columns per member (the SIMT form sets it)
};

struct TcGemmArgs {
    // Group operand images (tc_gemm_build_images), one every imageStride
    // bytes; imageStride 0: one image shared by all groups.
    const unsigned char* B;
    long long imageStride;
    int R, S, NP, KCH;
    const int* unitGroup;
    const int* unitColumn;  // first virtual column of the unit
    const int* unitCount;   // virtual columns in the unit
    int units;
    // Per-CTA unit ranges: CTA c walks units ctaFirst[c] .. ctaFirst[c+1]-1 (a
    // group's units sit in one range, so its operand image is loaded once per
    // CTA); the launch has `ctas` CTAs.  ctaFirst null: CTA c walks units c,
    // c + gridDim.x, ... of one grid of min(units, SMs) CTAs.
    const int* ctaFirst;
    int ctas;
    const int* groupColumns;  // complex columns per member in each group
    const int* groupFirst;    // first complex column of each group within a member
    long long memberColumns;
    const float2* in;  // [column][S] complex FP32 (or the bin array, see inBins)
    float2* out;       // [column][R] complex FP32 (or the bin array, see outBins)
    int* error;        // set to nonzero if a bounded wait expired
    BinBoundary inBins, outBins;
    // Test of the expired-wait path: the MMA lane of every CTA first waits on
    // a barrier that nothing arrives on, so that bounded wait runs out.
    int expireWaitForTest;
    // Operand form: 0 split TF32x3 (kind::tf32), 1 split BF16x3 (kind::f16).
    int kind;
};
bool tc_gemm_supported(int R, int S);
size_t tc_gemm_smem_bytes(int R, int S);
// Bytes of one group's operand image: the group matrix split into TF32 hi/lo
// parts, zero-padded to a multiple of 16 rows and of 32 k, in the swizzled
// shared-memory layout the kernel's MMAs read.
size_t tc_gemm_image_bytes(int R, int S);
// natural [groups][R][S] FP32 (device) -> images[groups] (device), split
// into TF32 hi / lo (kind 0) or BF16 h / m / l (kind 1); same size either way.
cudaError_t tc_gemm_build_images(const float* natural, int groups, int R, int S, int kind, void* images,
                                 cudaStream_t stream);
int tc_gemm_unit_tiles();
cudaError_t launch_tc_gemm(const TcGemmArgs& args, cudaStream_t stream);

// inBins / outBins (optional): cell-addressed operands (BinBoundary) instead of
// the compact [column][len] arrays.
cudaError_t launch_grouped_gemm(GemmPrecision p, int R, int S, const void* matrices, const GroupTiles& tiles,
                                ComplexOperand in, ComplexOperand out, cudaStream_t stream,
                                const BinBoundary* inBins = nullptr, const BinBoundary* outBins = nullptr);

}  // namespace skb
