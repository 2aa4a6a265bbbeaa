// Launch interface of the horizontal (x/y) transform kernels.
//
// Two kernels make every horizontal operator:
//   row kernels     length-Nx r2c / c2r along x for B planes at one y,
//                   reading/writing real planes [plane][y][x] and a dense bin
//                   array [y][kx][plane] that keeps kx < K.
//   column kernels  length-Ny c2c along y for B planes of one kx column,
//                   reading either a dense bin array or retained modes
//                   (zero-fill + kx = 0 Hermitian repair), and writing either a
//                   dense bin array or retained modes (conjugation + scale).
// With K = Nx/2+1 and the dense array laid out as the WVM spectrum this is the
// full 2-D r2c/c2r (fftw_provider.cpp:537-610); with K = the active kx band and
// retained-mode I/O it is the pruned transform (pruned_fftw_provider.cpp:315-517).

#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace skb {

constexpr int kMaxViews = 128;

// One field of retained (compact) coefficients: element (mode, z) lives at
// z + modeStride*mode.  Interleaved complex when imag == nullptr (re points at
// the complex array), split real/imaginary arrays otherwise.
struct FieldView {
    void* re;
    void* im;
    long long modeStride;
};

struct ViewSet {
    FieldView v[kMaxViews];
    int count;
};

struct ModeTables {
    // cell map for embedding: map[kx*Ny + ky] = (mode << 1 | conj), or -1.
    const int* cellMap;
    // per-kx gather lists: entries colStart[kx] .. colStart[kx+1]-1 of
    // colKy[] and colMode[] (mode << 1 | conj).
    const int* colStart;
    const int* colKy;
    const int* colMode;
    // gather map: map[kx*Ny + ky] = (mode << 1 | conj) for stored cells only, or -1.
    const int* gatherMap;
};

enum class Precision { f64 = 0, f32 = 1 };

struct DenseBins {
    void* data;          // complex T
    long long planes;    // stride between consecutive kx (total planes)
    long long kxStride;  // number of kx entries per ky row
};

// x-direction transforms.  Planes [0, planes) of real volumes laid out
// [plane][y][x]; bins kept for kx < keep.
cudaError_t launch_rows_forward(Precision p, int nx, int ny, long long planes, int keep, const void* real,
                                DenseBins bins, const void* twHalf, const void* twFull, cudaStream_t stream);
cudaError_t launch_rows_inverse(Precision p, int nx, int ny, long long planes, int keep, DenseBins bins, void* real,
                                const void* twHalf, const void* twFull, cudaStream_t stream);

// y-direction transforms over kx in [0, columns).
// sign = -1 forward, +1 inverse.
cudaError_t launch_columns_dense(Precision p, int sign, int ny, int columns, long long planes, DenseBins in,
                                 DenseBins out, const void* tw, cudaStream_t stream);
// Inverse: retained views -> dense bins (zero fill + Hermitian repair).
cudaError_t launch_columns_embed(Precision p, int ny, int nz, int columns, const ViewSet& views,
                                 const ModeTables& tables, DenseBins out, const void* tw, cudaStream_t stream);
// Forward: dense bins -> retained views (conjugation, scale).
cudaError_t launch_columns_gather(Precision p, int ny, int nz, int columns, DenseBins in, const ViewSet& views,
                                  const ModeTables& tables, double scale, const void* tw, cudaStream_t stream);

// Retention / embedding directly on a dense WVM spectrum (no transform).
cudaError_t launch_gather_dense(Precision p, int ny, int nz, long long modes, const int* modeKx, const int* modeKy,
                                const unsigned char* modeConj, DenseBins in, const ViewSet& views, double scale,
                                cudaStream_t stream);
cudaError_t launch_embed_dense(Precision p, int ny, int nz, int columns, const ViewSet& views,
                               const ModeTables& tables, DenseBins out, cudaStream_t stream);

// Largest supported power-of-two transform length along x (Nx) and y (Ny).
constexpr int kMaxLength = 2048;
bool supported_length(long long n);

}  // namespace skb
