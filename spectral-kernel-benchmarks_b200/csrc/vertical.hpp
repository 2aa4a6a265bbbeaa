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

#include <cuda_runtime.h>

namespace skb {

enum class GemmPrecision { f64 = 0, f32 = 1, tf32x3 = 2, bf16x3 = 3 };

struct GroupTiles {
    const int* tileGroup;   // matrix (K^2 group) of each CTA tile
    const int* tileColumn;  // first complex column of each tile
    const int* tileCount;   // complex columns in each tile (<= tile width)
    int tiles;
};

// Operand element: complex interleaved (im == nullptr) or split re/im arrays.
struct ComplexOperand {
    void* re;
    void* im;
};

// Column tile width (complex columns per CTA) used to build GroupTiles.
int gemm_tile_columns(GemmPrecision p);

cudaError_t launch_grouped_gemm(GemmPrecision p, int R, int S, const void* matrices, const GroupTiles& tiles,
                                ComplexOperand in, ComplexOperand out, cudaStream_t stream);

}  // namespace skb
