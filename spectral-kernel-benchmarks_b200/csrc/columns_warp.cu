// Warp-per-plane column transforms with fused retention, FP32, for the fused
// flux's two column stages.
//
// A CTA handles one kx column of B consecutive z-planes of one field view.
// Global traffic is CTA-wide and coalesced over the planes (B consecutive z of
// one mode, or of one (ky, kx) bin, are contiguous in HBM); each warp then
// transforms one plane's Ny-point column in its own padded shared region with
// warp_fft, so the only CTA-wide barriers are the one after the loads and the
// one before the stores.  The embed form scatters the retained modes of the
// column (with the kx = 0 Hermitian partner) and zero-fills the rest; the
// gather form keeps only the retained ky of the column and writes them, scaled
// and conjugated where the mode stores its partner, into the view.

#include "columns_warp.hpp"

#include <algorithm>
#include "async_copy.cuh"
#include "fft_device.cuh"

namespace skb {
namespace {

// Per-plane region: pad16 of the largest index plus slack, rounded so that
// region % 16 == 2 — the B planes of one ky then land in distinct banks when
// consecutive threads fill or drain consecutive planes.
template <int N>
constexpr int plane_region() {
    constexpr int base = N + N / 16 + 1;
    return base + ((2 - base % 16) + 16) % 16;
}

template <int N, int B>
__global__ void __launch_bounds__(32 * B, 4) columns_embed_warp_kernel(int nz, int zStride, ViewSet views, ModeTables tables,
                                                                    DenseBins out, const float2* __restrict__ tw) {
    constexpr int NT = 32 * B;
    constexpr int XP = plane_region<N>();
    constexpr int ITER = N * B / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const FieldView view = views.v[f];
    const int* map = tables.cellMap + static_cast<long long>(kx) * N;
    const int b = tid % B;  // NT is a multiple of B: every iteration has the same plane
    const int z = z0 + b;
    // Retained cells are copied asynchronously straight into the plane
    // regions (no register staging, so many copies are in flight per SM);
    // other cells are zero-filled by the same instruction.
    int e[ITER];
#pragma unroll
    for (int it = 0; it < ITER; ++it) e[it] = __ldg(map + (tid + it * NT) / B);
    const bool inRange = z < nz;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        float2* dst = xs + b * XP + pad16((tid + it * NT) / B);
        const bool have = inRange && e[it] >= 0;
        const long long i = have ? z + view.modeStride * (e[it] >> 1) : 0;
        if (view.im == nullptr) {
            cp_async8(dst, reinterpret_cast<const float2*>(view.re) + i, have ? 8 : 0);
        } else {
            cp_async4(&dst->x, reinterpret_cast<const float*>(view.re) + i, have ? 4 : 0);
            cp_async4(&dst->y, reinterpret_cast<const float*>(view.im) + i, have ? 4 : 0);
        }
    }
    cp_async_commit();
    cp_async_wait_all();
    // Cells that store the conjugate partner: negate in place (each thread
    // fixes the cells it copied).
#pragma unroll
    for (int it = 0; it < ITER; ++it)
        if (inRange && e[it] >= 0 && (e[it] & 1)) {
            float2* dst = xs + b * XP + pad16((tid + it * NT) / B);
            dst->y = -dst->y;
        }
    __syncthreads();
    if (z0 + warp < nz) warp_fft<float, N, +1>(xs + warp * XP, tw, lane);
    __syncthreads();
    if (z < nz) {
        float2* dst = static_cast<float2*>(out.data) + static_cast<long long>(f) * zStride + z + out.planes * kx;
        const long long rowStride = out.planes * out.kxStride;
#pragma unroll
        for (int it = 0; it < ITER; ++it) {
            const int ky = (tid + it * NT) / B;
            dst[rowStride * ky] = xs[b * XP + pad16(ky)];
        }
    }
}

template <int N, int B>
__global__ void __launch_bounds__(32 * B, 4) columns_gather_warp_kernel(int nz, int zStride, DenseBins in, ViewSet views,
                                                                     ModeTables tables, float scale,
                                                                     const float2* __restrict__ tw) {
    constexpr int NT = 32 * B;
    constexpr int XP = plane_region<N>();
    constexpr int ITER = N * B / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid % B;
    const int z = z0 + b;
    {
        const float2* src =
            static_cast<const float2*>(in.data) + static_cast<long long>(f) * zStride + z + in.planes * kx;
        const long long rowStride = in.planes * in.kxStride;
#pragma unroll
        for (int it = 0; it < ITER; ++it) {
            const int ky = (tid + it * NT) / B;
            cp_async8(xs + b * XP + pad16(ky), z < nz ? src + rowStride * ky : src, z < nz ? 8 : 0);
        }
        cp_async_commit();
        cp_async_wait_all();
    }
    __syncthreads();
    if (z0 + warp < nz) warp_fft<float, N, -1>(xs + warp * XP, tw, lane);
    __syncthreads();
    if (z >= nz) return;
    const FieldView view = views.v[f];
    const int begin = __ldg(tables.colStart + kx);
    const int end = __ldg(tables.colStart + kx + 1);
    for (int e = begin + tid / B; e < end; e += NT / B) {
        const int ky = __ldg(tables.colKy + e);
        const int mc = __ldg(tables.colMode + e);
        float2 v = xs[b * XP + pad16(ky)];
        v.x *= scale;
        v.y *= (mc & 1) ? -scale : scale;
        const long long i = z + view.modeStride * (mc >> 1);
        if (view.im == nullptr) {
            reinterpret_cast<float2*>(view.re)[i] = v;
        } else {
            reinterpret_cast<float*>(view.re)[i] = v.x;
            reinterpret_cast<float*>(view.im)[i] = v.y;
        }
    }
}

// ---------------------------------------------------------------------------
// 512-point columns with the first and last FFT passes at the HBM boundary.
// Three radix-8 Stockham passes (Ns = 1, 8, 64).  Pass 1 is done by thread
// (plane b = t % 8, butterflies j) straight from global memory: its eight
// inputs are ky = j + 64r of plane b, and consecutive threads take
// consecutive planes, so every load instruction reads 64 contiguous bytes per
// ky.  Pass 2 is warp-per-plane in shared memory.  Pass 3 is again thread
// (b, j): its outputs are ky = j + 64r of plane b, stored straight to global
// memory with the same coalescing.  Each element touches shared memory four
// times instead of eight.
// Two layouts share a plane's region: pass 1 writes element e at pad16(e),
// pass 2 reads that and writes element e at e + 8(e/64), which pass 3 reads.
// With a plane region of 2 mod 16 elements every access is free of bank
// conflicts: in a half-warp the two butterflies of pass 1 differ by 2 and
// those of pass 3 by 1 (planes b = 0..7 then fill the other residues), and
// the pass-2 stores of butterflies j and j + 8 land 72 = 8 (mod 16) apart.
// Twiddles of passes 2 and 3 come from the lane-ordered table of
// rr_fill_table, copied into shared memory once per CTA.
constexpr int kDirectN = 512;
constexpr int kDirectRegion = 578;  // > 511 + 8 * 7, and 578 % 16 == 2
static_assert(kDirectRegion % 16 == 2 && kDirectRegion > 567, "direct plane region");
constexpr int kDirectTable = rr_table_size<kDirectN>();

// The CTA's twiddle table, after the eight plane regions; filled by all 256
// threads, read after the CTA's next barrier.
__device__ __forceinline__ const float2* direct_table(float2* xs, const float2* __restrict__ tw, int tid) {
    float2* tt = xs + 8 * kDirectRegion;
    rr_fill_table<float, kDirectN>(tt, tw, tid, 256);
    return tt;
}

// Pass-3 inputs of butterfly j (< 64) of plane b: elements j + 64r in the
// pass-2 layout, times their twiddles.
template <int SIGN>
__device__ __forceinline__ void direct_last_inputs(const float2* xs, const float2* tt, int b, int j, float2 (&v)[8]) {
    const float2* in = xs + b * kDirectRegion + j;
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = in[72 * r];
#pragma unroll
    for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], twiddle_plain<SIGN>(tt + 56 + j, 64 * (r - 1)));
}

__device__ __forceinline__ int pass1_butterfly(int t, int q) {
    const int h = t >> 4;
    return 4 * (h >> 1) + (h & 1) + 2 * ((t >> 3) & 1) + 32 * q;
}

// Addresses of the passes as per-lane bases plus compile-time offsets
// (j < 64): pass-1 stores pad16(8j + r) = 8j + j/2 + r, pass-2 loads
// pad16(j + 64r) = j + j/16 + 68r, pass-2 stores of element 64(j/8) + j%8 + 8r
// at 72(j/8) + j%8 + 8r, pass-3 loads of element j + 64r at j + 72r.
template <int SIGN>
__device__ __forceinline__ void direct_middle_pass(float2* xs, const float2* tt, int warp, int lane) {
    float2* x = xs + warp * kDirectRegion;
    float2 v[2][8];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        const float2* in = x + j + (j >> 4);
#pragma unroll
        for (int r = 0; r < 8; ++r) v[q][r] = in[68 * r];
        const float2* t2 = tt + (j % 8);
#pragma unroll
        for (int r = 1; r < 8; ++r) v[q][r] = cmul(v[q][r], twiddle_plain<SIGN>(t2, 8 * (r - 1)));
        dft8<SIGN>(v[q]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        float2* o = x + 72 * (j / 8) + (j % 8);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[8 * r] = v[q][r];
    }
}

__global__ void __launch_bounds__(256, 3) columns_embed_direct_kernel(int nz, int zStride, ViewSet views, ModeTables tables,
                                                                      DenseBins out, const float2* __restrict__ tw) {
    constexpr int B = 8, N = kDirectN, XP = kDirectRegion;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float2* tt = direct_table(xs, tw, tid);
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid & 7;
    const int z = z0 + b;
    const bool inRange = z < nz;
    const int* map = tables.cellMap + static_cast<long long>(kx) * N;
    {
        const FieldView view = views.v[f];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = pass1_butterfly(tid, q);
            int e[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) e[r] = __ldg(map + j + 64 * r);
            float2 v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                v[r] = make_float2(0.f, 0.f);
                if (inRange && e[r] >= 0) {
                    const long long i = z + view.modeStride * (e[r] >> 1);
                    if (view.im == nullptr) {
                        v[r] = __ldg(reinterpret_cast<const float2*>(view.re) + i);
                    } else {
                        v[r] = make_float2(__ldg(reinterpret_cast<const float*>(view.re) + i),
                                           __ldg(reinterpret_cast<const float*>(view.im) + i));
                    }
                    if (e[r] & 1) v[r].y = -v[r].y;
                }
            }
            dft8<+1>(v);
            float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
            for (int r = 0; r < 8; ++r) o[r] = v[r];
        }
    }
    __syncthreads();
    if (z0 + warp < nz) direct_middle_pass<+1>(xs, tt, warp, lane);  // planes beyond Nz stay idle
    __syncthreads();
    if (!inRange) return;
    float2* dst = static_cast<float2*>(out.data) + static_cast<long long>(f) * zStride + z + out.planes * kx;
    const long long rowStride = out.planes * out.kxStride;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = (tid >> 3) + 32 * q;
        float2 v[8];
        direct_last_inputs<+1>(xs, tt, b, j, v);
        dft8<+1>(v);
#pragma unroll
        for (int r = 0; r < 8; ++r) dst[rowStride * (j + 64 * r)] = v[r];
    }
}

__global__ void __launch_bounds__(256, 3) columns_gather_direct_kernel(int nz, int zStride, DenseBins in, ViewSet views,
                                                                       ModeTables tables, float scale,
                                                                       const float2* __restrict__ tw) {
    constexpr int B = 8, N = kDirectN, XP = kDirectRegion;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float2* tt = direct_table(xs, tw, tid);
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid & 7;
    const int z = z0 + b;
    const bool inRange = z < nz;
    {
        const float2* src = static_cast<const float2*>(in.data) + static_cast<long long>(f) * zStride + z + in.planes * kx;
        const long long rowStride = in.planes * in.kxStride;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = pass1_butterfly(tid, q);
            float2 v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = inRange ? __ldg(src + rowStride * (j + 64 * r)) : make_float2(0.f, 0.f);
            dft8<-1>(v);
            float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
            for (int r = 0; r < 8; ++r) o[r] = v[r];
        }
    }
    __syncthreads();
    if (z0 + warp < nz) direct_middle_pass<-1>(xs, tt, warp, lane);
    __syncthreads();
    if (!inRange) return;
    const FieldView view = views.v[f];
    const int* map = tables.gatherMap + static_cast<long long>(kx) * N;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = (tid >> 3) + 32 * q;
        int e[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) e[r] = __ldg(map + j + 64 * r);
        float2 v[8];
        direct_last_inputs<-1>(xs, tt, b, j, v);
        dft8<-1>(v);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            if (e[r] < 0) continue;
            float2 o = v[r];
            o.x *= scale;
            o.y *= (e[r] & 1) ? -scale : scale;
            const long long i = z + view.modeStride * (e[r] >> 1);
            if (view.im == nullptr) {
                reinterpret_cast<float2*>(view.re)[i] = o;
            } else {
                reinterpret_cast<float*>(view.re)[i] = o.x;
                reinterpret_cast<float*>(view.im)[i] = o.y;
            }
        }
    }
}

constexpr size_t kDirectSmem = sizeof(float2) * (8 * kDirectRegion + kDirectTable);

constexpr int kPlanes = 8;

template <int N>
size_t smem_bytes() {
    return sizeof(float2) * size_t(kPlanes) * plane_region<N>();
}

template <typename K>
cudaError_t prepare(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

template <int N>
cudaError_t embed_n(int nz, int zStride, int columns, const ViewSet& views, const ModeTables& tables, DenseBins out,
                    const void* tw, cudaStream_t s) {
    auto kernel = columns_embed_warp_kernel<N, kPlanes>;
    const size_t bytes = smem_bytes<N>();
    cudaError_t err = prepare(kernel, bytes);
    if (err != cudaSuccess) return err;
    const int zChunks = (nz + kPlanes - 1) / kPlanes;
    kernel<<<dim3(unsigned(zChunks * views.count), unsigned(columns)), 32 * kPlanes, bytes, s>>>(
        nz, zStride, views, tables, out, static_cast<const float2*>(tw));
    return cudaGetLastError();
}

template <int N>
cudaError_t gather_n(int nz, int zStride, int columns, DenseBins in, const ViewSet& views, const ModeTables& tables, double scale,
                     const void* tw, cudaStream_t s) {
    auto kernel = columns_gather_warp_kernel<N, kPlanes>;
    const size_t bytes = smem_bytes<N>();
    cudaError_t err = prepare(kernel, bytes);
    if (err != cudaSuccess) return err;
    const int zChunks = (nz + kPlanes - 1) / kPlanes;
    kernel<<<dim3(unsigned(zChunks * views.count), unsigned(columns)), 32 * kPlanes, bytes, s>>>(
        nz, zStride, in, views, tables, float(scale), static_cast<const float2*>(tw));
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Band forms for the fused flux, in place on the dense bin array.  The
// retained cells of column kx (with their kx = 0 Hermitian partners) are
// exactly the band min(ky, Ny - ky) <= band[kx] (checked on the host), and the
// vertical GEMM reads and writes the retained values at their cells directly,
// so these kernels need no mode map: the inverse reads the band cells (the
// rest of the column is zero) and writes the whole column; the forward reads
// the whole column and writes back only the band cells.  Slot f's planes start
// at plane f * zStride.
__device__ __forceinline__ bool in_band(int ky, int n, int band) { return min(ky, n - ky) <= band; }

// MINB: CTAs per SM the register allocation must allow (3, or 4 for the
// kBandDirect4 form, which trades registers for loads in flight).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) columns_inverse_band_kernel(int nz, int zStride, DenseBins bins,
                                                                      const int* __restrict__ bandOf,
                                                                      const float2* __restrict__ tw) {
    constexpr int B = 8, N = kDirectN, XP = kDirectRegion;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float2* tt = direct_table(xs, tw, tid);
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid & 7;
    const int z = z0 + b;
    const bool inRange = z < nz;
    const int band = __ldg(bandOf + kx);
    float2* col = static_cast<float2*>(bins.data) + static_cast<long long>(f) * zStride + z + bins.planes * kx;
    const long long rowStride = bins.planes * bins.kxStride;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = pass1_butterfly(tid, q);
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int ky = j + 64 * r;
            v[r] = (inRange && in_band(ky, N, band)) ? col[rowStride * ky] : make_float2(0.f, 0.f);
        }
        dft8<+1>(v);
        float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[r] = v[r];
    }
    __syncthreads();
    if (z0 + warp < nz) direct_middle_pass<+1>(xs, tt, warp, lane);  // planes beyond Nz stay idle
    __syncthreads();
    if (!inRange) return;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = (tid >> 3) + 32 * q;
        float2 v[8];
        direct_last_inputs<+1>(xs, tt, b, j, v);
        dft8<+1>(v);
#pragma unroll
        for (int r = 0; r < 8; ++r) col[rowStride * (j + 64 * r)] = v[r];
    }
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) columns_forward_band_kernel(int nz, int zStride, DenseBins bins,
                                                                      const int* __restrict__ bandOf, float scale,
                                                                      const float2* __restrict__ tw) {
    constexpr int B = 8, N = kDirectN, XP = kDirectRegion;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float2* tt = direct_table(xs, tw, tid);
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid & 7;
    const int z = z0 + b;
    const bool inRange = z < nz;
    float2* col = static_cast<float2*>(bins.data) + static_cast<long long>(f) * zStride + z + bins.planes * kx;
    const long long rowStride = bins.planes * bins.kxStride;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = pass1_butterfly(tid, q);
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = inRange ? col[rowStride * (j + 64 * r)] : make_float2(0.f, 0.f);
        dft8<-1>(v);
        float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[r] = v[r];
    }
    __syncthreads();
    if (z0 + warp < nz) direct_middle_pass<-1>(xs, tt, warp, lane);
    __syncthreads();
    if (!inRange) return;
    const int band = __ldg(bandOf + kx);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = (tid >> 3) + 32 * q;
        float2 v[8];
        direct_last_inputs<-1>(xs, tt, b, j, v);
        dft8<-1>(v);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int ky = j + 64 * r;
            if (in_band(ky, N, band)) col[rowStride * ky] = make_float2(scale * v[r].x, scale * v[r].y);
        }
    }
}

// Persistent forms of the two direct band kernels: two CTAs per SM walk the
// (kx, slot, z-chunk) tiles in the launch order of the kernels above, and each
// thread issues the next tile's sixteen loads before running the current
// tile's three passes, so the next tile's HBM reads overlap this tile's
// shared-memory passes and stores.  Tile t is (kx, slot, z-chunk) =
// (t / (zChunks * slots), (t % (zChunks * slots)) / zChunks, t % zChunks).
template <int SIGN>
__global__ void __launch_bounds__(256, 2) columns_band_persist_kernel(int nz, int zStride, int slots, int columns,
                                                                       DenseBins bins, const int* __restrict__ bandOf,
                                                                       float scale, const float2* __restrict__ tw) {
    // SIGN = +1: inverse (read the band, write every row);
    // SIGN = -1: forward (read every row, write the band, times scale).
    constexpr int B = 8, N = kDirectN, XP = kDirectRegion;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float2* tt = direct_table(xs, tw, tid);
    const int b = tid & 7;
    const int zChunks = (nz + B - 1) / B;
    const long long perColumn = static_cast<long long>(zChunks) * slots;
    const long long tiles = perColumn * columns;
    const long long rowStride = bins.planes * bins.kxStride;
    struct Tile {
        int kx, z0, band;
        float2* col;
    };
    auto tile_at = [&](long long t) {
        Tile T;
        T.kx = static_cast<int>(t / perColumn);
        const int x = static_cast<int>(t - T.kx * perColumn);
        const int f = x / zChunks;
        T.z0 = (x - f * zChunks) * B;
        T.band = __ldg(bandOf + T.kx);
        T.col = static_cast<float2*>(bins.data) + static_cast<long long>(f) * zStride + T.z0 + b + bins.planes * T.kx;
        return T;
    };
    auto load = [&](const Tile& T, float2 (&v)[2][8]) {
        const bool inRange = T.z0 + b < nz;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = pass1_butterfly(tid, q);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int ky = j + 64 * r;
                const bool have = inRange && (SIGN < 0 || in_band(ky, N, T.band));
                v[q][r] = have ? T.col[rowStride * ky] : make_float2(0.f, 0.f);
            }
        }
    };
    long long t = blockIdx.x;
    if (t >= tiles) return;  // whole CTA; no barrier has been reached
    Tile cur = tile_at(t);
    float2 v[2][8];
    load(cur, v);
    for (; t < tiles; t += gridDim.x) {
        // Pass 1 of this tile from registers.
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = pass1_butterfly(tid, q);
            dft8<SIGN>(v[q]);
            float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
            for (int r = 0; r < 8; ++r) o[r] = v[q][r];
        }
        // The next tile's loads, in flight during passes 2 and 3.
        const long long tn = t + gridDim.x;
        Tile next = cur;
        if (tn < tiles) {
            next = tile_at(tn);
            load(next, v);
        }
        __syncthreads();
        if (cur.z0 + warp < nz) direct_middle_pass<SIGN>(xs, tt, warp, lane);  // planes beyond Nz stay idle
        __syncthreads();
        if (cur.z0 + b < nz) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int j = (tid >> 3) + 32 * q;
                float2 w[8];
                direct_last_inputs<SIGN>(xs, tt, b, j, w);
                dft8<SIGN>(w);
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int ky = j + 64 * r;
                    if (SIGN > 0)
                        cur.col[rowStride * ky] = w[r];
                    else if (in_band(ky, N, cur.band))
                        cur.col[rowStride * ky] = make_float2(scale * w[r].x, scale * w[r].y);
                }
            }
        }
        __syncthreads();  // this tile's reads of xs precede the next tile's pass 1
        cur = next;
    }
}

// Generic-N band forms (warp per plane, cp.async staging).
template <int N, int B>
__global__ void __launch_bounds__(32 * B, 4) columns_inverse_band_warp_kernel(int nz, int zStride, DenseBins bins,
                                                                              const int* __restrict__ bandOf,
                                                                              const float2* __restrict__ tw) {
    constexpr int NT = 32 * B;
    constexpr int XP = plane_region<N>();
    constexpr int ITER = N * B / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid % B;
    const int z = z0 + b;
    const bool inRange = z < nz;
    const int band = __ldg(bandOf + kx);
    float2* col = static_cast<float2*>(bins.data) + static_cast<long long>(f) * zStride + z + bins.planes * kx;
    const long long rowStride = bins.planes * bins.kxStride;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int ky = (tid + it * NT) / B;
        const bool have = inRange && in_band(ky, N, band);
        cp_async8(xs + b * XP + pad16(ky), have ? col + rowStride * ky : col, have ? 8 : 0);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (z0 + warp < nz) warp_fft<float, N, +1>(xs + warp * XP, tw, lane);
    __syncthreads();
    if (!inRange) return;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int ky = (tid + it * NT) / B;
        col[rowStride * ky] = xs[b * XP + pad16(ky)];
    }
}

template <int N, int B>
__global__ void __launch_bounds__(32 * B, 4) columns_forward_band_warp_kernel(int nz, int zStride, DenseBins bins,
                                                                              const int* __restrict__ bandOf,
                                                                              float scale,
                                                                              const float2* __restrict__ tw) {
    constexpr int NT = 32 * B;
    constexpr int XP = plane_region<N>();
    constexpr int ITER = N * B / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const int b = tid % B;
    const int z = z0 + b;
    const bool inRange = z < nz;
    float2* col = static_cast<float2*>(bins.data) + static_cast<long long>(f) * zStride + z + bins.planes * kx;
    const long long rowStride = bins.planes * bins.kxStride;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int ky = (tid + it * NT) / B;
        cp_async8(xs + b * XP + pad16(ky), inRange ? col + rowStride * ky : col, inRange ? 8 : 0);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (z0 + warp < nz) warp_fft<float, N, -1>(xs + warp * XP, tw, lane);
    __syncthreads();
    if (!inRange) return;
    const int band = __ldg(bandOf + kx);
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int ky = (tid + it * NT) / B;
        if (in_band(ky, N, band)) {
            const float2 v = xs[b * XP + pad16(ky)];
            col[rowStride * ky] = make_float2(scale * v.x, scale * v.y);
        }
    }
}

// 16- and 32-plane forms of the two direct band kernels (kBand16, kBand32).
// A CTA of 32 B threads owns B consecutive planes of the flat plane index
// (slot * zStride + z) and one kx column, so each pass-1 load and pass-3 store
// instruction moves 8 B contiguous bytes of one ky row (the 8-plane forms move
// 64, which held the stage near 45 % of HBM: a copy with the same addressing
// and no FFT ran at the same speed, and at 16 planes about 1.6x faster).
// Chunks over the flat index keep every chunk full of real planes except where
// it crosses a slot's z padding (planes with z >= Nz are skipped).
// Pass-1 thread (plane b = t % B, butterflies j).  B = 16: the two butterflies
// of a warp are j and j + 2, and with the 2-mod-16 plane region the pass-1
// stores and pass-3 loads of a warp fill every bank pair exactly twice.
// B = 32: a warp is 32 planes of one butterfly, and a plane region of 1 mod 16
// does the same.
// SIGN = +1: inverse (read the band, write every row); SIGN = -1: forward
// (read every row, write the band times scale).
template <int B>
__device__ __forceinline__ int band_wide_butterfly(int t, int q) {
    if constexpr (B == 16) {
        const int a = (t >> 5) & 15, c = (t >> 4) & 1;
        return 4 * (a >> 1) + (a & 1) + 2 * c + 32 * q;
    } else {
        return (t >> 5) + 32 * q;
    }
}
template <int B>
constexpr int band_wide_region() {
    return B == 16 ? kDirectRegion : 577;  // 577 % 16 == 1, > 511 + 8 * 7
}
template <int B>
constexpr size_t band_wide_smem() {
    return sizeof(float2) * (size_t(B) * band_wide_region<B>() + kDirectTable);
}

// The direct kernels' middle pass with an explicit plane region.
template <int SIGN, int XP>
__device__ __forceinline__ void wide_middle_pass(float2* xs, const float2* tt, int warp, int lane) {
    float2* x = xs + warp * XP;
    float2 v[2][8];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        const float2* in = x + j + (j >> 4);
#pragma unroll
        for (int r = 0; r < 8; ++r) v[q][r] = in[68 * r];
        const float2* t2 = tt + (j % 8);
#pragma unroll
        for (int r = 1; r < 8; ++r) v[q][r] = cmul(v[q][r], twiddle_plain<SIGN>(t2, 8 * (r - 1)));
        dft8<SIGN>(v[q]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        float2* o = x + 72 * (j / 8) + (j % 8);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[8 * r] = v[q][r];
    }
}

template <int B, int SIGN>
__global__ void __launch_bounds__(32 * B, 32 / B) columns_band_wide_kernel(int nz, int zStride, long long flatPlanes,
                                                                          DenseBins bins,
                                                                          const int* __restrict__ bandOf, float scale,
                                                                          const float2* __restrict__ tw) {
    constexpr int N = kDirectN, XP = band_wide_region<B>();
    constexpr int NT = 32 * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xs = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float2* tt = xs + B * XP;
    rr_fill_table<float, N>(tt, tw, tid, NT);
    const long long p0 = static_cast<long long>(blockIdx.x) * B;
    const int kx = blockIdx.y;
    const int b = tid % B;
    const long long p = p0 + b;
    const bool inRange = p < flatPlanes && static_cast<int>(p % zStride) < nz;
    const int band = __ldg(bandOf + kx);
    float2* col = static_cast<float2*>(bins.data) + p + bins.planes * kx;
    const long long rowStride = bins.planes * bins.kxStride;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = band_wide_butterfly<B>(tid, q);
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int ky = j + 64 * r;
            const bool load = inRange && (SIGN < 0 || in_band(ky, N, band));
            v[r] = load ? col[rowStride * ky] : make_float2(0.f, 0.f);
        }
        dft8<SIGN>(v);
        float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[r] = v[r];
    }
    __syncthreads();
    {
        const long long pw = p0 + warp;  // planes beyond Nz (or the array) stay idle
        if (pw < flatPlanes && static_cast<int>(pw % zStride) < nz) wide_middle_pass<SIGN, XP>(xs, tt, warp, lane);
    }
    __syncthreads();
    if (!inRange) return;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = (tid / B) + 32 * q;
        const float2* in = xs + b * XP + j;  // pass-3 inputs: elements j + 64 r at j + 72 r
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = in[72 * r];
#pragma unroll
        for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], twiddle_plain<SIGN>(tt + 56 + j, 64 * (r - 1)));
        dft8<SIGN>(v);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int ky = j + 64 * r;
            if (SIGN > 0)
                col[rowStride * ky] = v[r];
            else if (in_band(ky, N, band))
                col[rowStride * ky] = make_float2(scale * v[r].x, scale * v[r].y);
        }
    }
}

// Pipelined 16-plane forms (kBand16Pipe*): one CTA per SM walks `perCta` kx
// columns of its 16 planes (every gridDim.y-th column), with the pass-1 loads
// of the next column issued into registers right after the current column's
// pass 1, so they are in flight during its middle pass and pass 3.  Two
// shared-memory regions alternate between columns; the passes are those of
// columns_band_wide_kernel.
constexpr size_t band_pipe_smem() {
    return sizeof(float2) * (2 * size_t(16) * band_wide_region<16>() + kDirectTable);
}
template <int SIGN>
__global__ void __launch_bounds__(512, 1) columns_band_pipe_kernel(int nz, int zStride, long long flatPlanes,
                                                                   int columns, DenseBins bins,
                                                                   const int* __restrict__ bandOf, float scale,
                                                                   const float2* __restrict__ tw) {
    constexpr int B = 16;
    constexpr int N = kDirectN, XP = band_wide_region<B>();
    constexpr int NT = 32 * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* xsAll = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float2* tt = xsAll + 2 * B * XP;
    rr_fill_table<float, N>(tt, tw, tid, NT);
    const long long p0 = static_cast<long long>(blockIdx.x) * B;
    const int b = tid % B;
    const long long p = p0 + b;
    const bool inRange = p < flatPlanes && static_cast<int>(p % zStride) < nz;
    const long long pw = p0 + warp;
    const bool warpActive = pw < flatPlanes && static_cast<int>(pw % zStride) < nz;
    const long long rowStride = bins.planes * bins.kxStride;
    float2* base = static_cast<float2*>(bins.data) + p;
    // Pass-1 inputs of column kx into v (the loads are only issued here).
    auto load = [&](int kx, float2 (&v)[2][8]) {
        const int band = __ldg(bandOf + kx);
        const float2* col = base + bins.planes * kx;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = band_wide_butterfly<B>(tid, q);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int ky = j + 64 * r;
                const bool ld = inRange && (SIGN < 0 || in_band(ky, N, band));
                v[q][r] = ld ? col[rowStride * ky] : make_float2(0.f, 0.f);
            }
        }
    };
    float2 v[2][8];
    int kx = blockIdx.y;
    if (kx < columns) load(kx, v);
    for (int i = 0; kx < columns; ++i, kx += gridDim.y) {
        float2* xs = xsAll + (i & 1) * B * XP;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = band_wide_butterfly<B>(tid, q);
            dft8<SIGN>(v[q]);
            float2* o = xs + b * XP + 8 * j + (j >> 1);
#pragma unroll
            for (int r = 0; r < 8; ++r) o[r] = v[q][r];
        }
        const int next = kx + static_cast<int>(gridDim.y);
        if (next < columns) load(next, v);
        __syncthreads();
        if (warpActive) wide_middle_pass<SIGN, XP>(xs, tt, warp, lane);
        __syncthreads();
        if (inRange) {
            const int band = __ldg(bandOf + kx);
            float2* col = base + bins.planes * kx;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int j = (tid / B) + 32 * q;
                const float2* in = xs + b * XP + j;
                float2 w[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) w[r] = in[72 * r];
#pragma unroll
                for (int r = 1; r < 8; ++r) w[r] = cmul(w[r], twiddle_plain<SIGN>(tt + 56 + j, 64 * (r - 1)));
                dft8<SIGN>(w);
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int ky = j + 64 * r;
                    if (SIGN > 0)
                        col[rowStride * ky] = w[r];
                    else if (in_band(ky, N, band))
                        col[rowStride * ky] = make_float2(scale * w[r].x, scale * w[r].y);
                }
            }
        }
    }
}

template <int SIGN>
cudaError_t launch_band_pipe(int nz, int zStride, int slots, int columns, DenseBins bins, const int* band,
                             float scale, const void* tw, int perCta, cudaStream_t s) {
    auto kernel = columns_band_pipe_kernel<SIGN>;
    cudaError_t err = prepare(kernel, band_pipe_smem());
    if (err != cudaSuccess) return err;
    const long long flat = static_cast<long long>(slots) * zStride;
    const dim3 grid(unsigned((flat + 15) / 16), unsigned((columns + perCta - 1) / perCta));
    kernel<<<grid, 512, band_pipe_smem(), s>>>(nz, zStride, flat, columns, bins, band, scale,
                                               static_cast<const float2*>(tw));
    return cudaGetLastError();
}

template <int B, int SIGN>
cudaError_t launch_band_wide(int nz, int zStride, int slots, int columns, DenseBins bins, const int* band, float scale,
                             const void* tw, cudaStream_t s) {
    auto kernel = columns_band_wide_kernel<B, SIGN>;
    cudaError_t err = prepare(kernel, band_wide_smem<B>());
    if (err != cudaSuccess) return err;
    const long long flat = static_cast<long long>(slots) * zStride;
    const dim3 grid(unsigned((flat + B - 1) / B), unsigned(columns));
    kernel<<<grid, 32 * B, band_wide_smem<B>(), s>>>(nz, zStride, flat, bins, band, scale,
                                                     static_cast<const float2*>(tw));
    return cudaGetLastError();
}

template <int SIGN>
cudaError_t launch_band_persist(int nz, int zStride, int slots, int columns, DenseBins bins, const int* band,
                                float scale, const void* tw, cudaStream_t s) {
    auto kernel = columns_band_persist_kernel<SIGN>;
    cudaError_t err = prepare(kernel, kDirectSmem);
    if (err != cudaSuccess) return err;
    static int cachedDevice = -1, cachedBlocks = 0;
    int device = 0;
    err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    if (device != cachedDevice) {
        int perSm = 0, sms = 0;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, 256, kDirectSmem);
        if (err != cudaSuccess) return err;
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (err != cudaSuccess) return err;
        cachedBlocks = std::max(1, perSm) * std::max(1, sms);
        cachedDevice = device;
    }
    const long long tiles = static_cast<long long>((nz + 7) / 8) * slots * columns;
    const int blocks = static_cast<int>(std::min<long long>(tiles, cachedBlocks));
    kernel<<<blocks, 256, kDirectSmem, s>>>(nz, zStride, slots, columns, bins, band, scale,
                                            static_cast<const float2*>(tw));
    return cudaGetLastError();
}

template <int N>
cudaError_t inverse_band_n(int nz, int zStride, int slots, int columns, DenseBins bins, const int* band, const void* tw,
                           int form, cudaStream_t s) {
    constexpr int B = 8;
    const int zChunks = (nz + B - 1) / B;
    const dim3 grid(unsigned(zChunks * slots), unsigned(columns));
    if (N == kDirectN && form == kBandPersist)
        return launch_band_persist<+1>(nz, zStride, slots, columns, bins, band, 1.0f, tw, s);
    if (N == kDirectN && form == kBand16)
        return launch_band_wide<16, +1>(nz, zStride, slots, columns, bins, band, 1.0f, tw, s);
    if (N == kDirectN && form == kBand32)
        return launch_band_wide<32, +1>(nz, zStride, slots, columns, bins, band, 1.0f, tw, s);
    if (N == kDirectN && band_pipe_columns(form) > 0)
        return launch_band_pipe<+1>(nz, zStride, slots, columns, bins, band, 1.0f, tw, band_pipe_columns(form), s);
    if (N == kDirectN && form != kBandWarp) {
        auto kernel = form == kBandDirect4 ? columns_inverse_band_kernel<4> : columns_inverse_band_kernel<3>;
        cudaError_t err = prepare(kernel, kDirectSmem);
        if (err != cudaSuccess) return err;
        kernel<<<grid, 256, kDirectSmem, s>>>(nz, zStride, bins, band, static_cast<const float2*>(tw));
    } else {
        auto kernel = columns_inverse_band_warp_kernel<N, B>;
        const size_t bytes = sizeof(float2) * size_t(B) * plane_region<N>();
        cudaError_t err = prepare(kernel, bytes);
        if (err != cudaSuccess) return err;
        kernel<<<grid, 32 * B, bytes, s>>>(nz, zStride, bins, band, static_cast<const float2*>(tw));
    }
    return cudaGetLastError();
}

template <int N>
cudaError_t forward_band_n(int nz, int zStride, int slots, int columns, DenseBins bins, const int* band, double scale,
                           const void* tw, int form, cudaStream_t s) {
    constexpr int B = 8;
    const int zChunks = (nz + B - 1) / B;
    const dim3 grid(unsigned(zChunks * slots), unsigned(columns));
    if (N == kDirectN && form == kBandPersist)
        return launch_band_persist<-1>(nz, zStride, slots, columns, bins, band, float(scale), tw, s);
    if (N == kDirectN && form == kBand16)
        return launch_band_wide<16, -1>(nz, zStride, slots, columns, bins, band, float(scale), tw, s);
    if (N == kDirectN && form == kBand32)
        return launch_band_wide<32, -1>(nz, zStride, slots, columns, bins, band, float(scale), tw, s);
    if (N == kDirectN && band_pipe_columns(form) > 0)
        return launch_band_pipe<-1>(nz, zStride, slots, columns, bins, band, float(scale), tw, band_pipe_columns(form), s);
    if (N == kDirectN && form != kBandWarp) {
        auto kernel = form == kBandDirect4 ? columns_forward_band_kernel<4> : columns_forward_band_kernel<3>;
        cudaError_t err = prepare(kernel, kDirectSmem);
        if (err != cudaSuccess) return err;
        kernel<<<grid, 256, kDirectSmem, s>>>(nz, zStride, bins, band, float(scale), static_cast<const float2*>(tw));
    } else {
        auto kernel = columns_forward_band_warp_kernel<N, B>;
        const size_t bytes = sizeof(float2) * size_t(B) * plane_region<N>();
        cudaError_t err = prepare(kernel, bytes);
        if (err != cudaSuccess) return err;
        kernel<<<grid, 32 * B, bytes, s>>>(nz, zStride, bins, band, float(scale), static_cast<const float2*>(tw));
    }
    return cudaGetLastError();
}

}  // namespace

bool columns_warp_supported(long long ny) { return ny >= 32 && ny <= 512 && (ny & (ny - 1)) == 0; }

cudaError_t launch_columns_embed_warp(int ny, int nz, int zStride, int columns, const ViewSet& views, const ModeTables& tables,
                                      DenseBins out, const void* tw, cudaStream_t s) {
    if (views.count <= 0 || columns <= 0) return cudaSuccess;
    switch (ny) {
        case 32: return embed_n<32>(nz, zStride, columns, views, tables, out, tw, s);
        case 64: return embed_n<64>(nz, zStride, columns, views, tables, out, tw, s);
        case 128: return embed_n<128>(nz, zStride, columns, views, tables, out, tw, s);
        case 256: return embed_n<256>(nz, zStride, columns, views, tables, out, tw, s);
        case 512: {
            cudaError_t err = prepare(columns_embed_direct_kernel, kDirectSmem);
            if (err != cudaSuccess) return err;
            const int zChunks = (nz + 7) / 8;
            columns_embed_direct_kernel<<<dim3(unsigned(zChunks * views.count), unsigned(columns)), 256, kDirectSmem,
                                          s>>>(nz, zStride, views, tables, out, static_cast<const float2*>(tw));
            return cudaGetLastError();
        }
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_columns_gather_warp(int ny, int nz, int zStride, int columns, DenseBins in, const ViewSet& views,
                                       const ModeTables& tables, double scale, const void* tw, cudaStream_t s) {
    if (views.count <= 0 || columns <= 0) return cudaSuccess;
    switch (ny) {
        case 32: return gather_n<32>(nz, zStride, columns, in, views, tables, scale, tw, s);
        case 64: return gather_n<64>(nz, zStride, columns, in, views, tables, scale, tw, s);
        case 128: return gather_n<128>(nz, zStride, columns, in, views, tables, scale, tw, s);
        case 256: return gather_n<256>(nz, zStride, columns, in, views, tables, scale, tw, s);
        case 512: {
            cudaError_t err = prepare(columns_gather_direct_kernel, kDirectSmem);
            if (err != cudaSuccess) return err;
            const int zChunks = (nz + 7) / 8;
            columns_gather_direct_kernel<<<dim3(unsigned(zChunks * views.count), unsigned(columns)), 256, kDirectSmem,
                                           s>>>(nz, zStride, in, views, tables, float(scale), static_cast<const float2*>(tw));
            return cudaGetLastError();
        }
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace skb

namespace skb {

cudaError_t launch_columns_inverse_band(int ny, int nz, int zStride, int slots, int columns, DenseBins bins,
                                        const int* band, const void* tw, int form, cudaStream_t s) {
    if (slots <= 0 || columns <= 0) return cudaSuccess;
    switch (ny) {
        case 32: return inverse_band_n<32>(nz, zStride, slots, columns, bins, band, tw, form, s);
        case 64: return inverse_band_n<64>(nz, zStride, slots, columns, bins, band, tw, form, s);
        case 128: return inverse_band_n<128>(nz, zStride, slots, columns, bins, band, tw, form, s);
        case 256: return inverse_band_n<256>(nz, zStride, slots, columns, bins, band, tw, form, s);
        case 512: return inverse_band_n<512>(nz, zStride, slots, columns, bins, band, tw, form, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_columns_forward_band(int ny, int nz, int zStride, int slots, int columns, DenseBins bins,
                                        const int* band, double scale, const void* tw, int form, cudaStream_t s) {
    if (slots <= 0 || columns <= 0) return cudaSuccess;
    switch (ny) {
        case 32: return forward_band_n<32>(nz, zStride, slots, columns, bins, band, scale, tw, form, s);
        case 64: return forward_band_n<64>(nz, zStride, slots, columns, bins, band, scale, tw, form, s);
        case 128: return forward_band_n<128>(nz, zStride, slots, columns, bins, band, scale, tw, form, s);
        case 256: return forward_band_n<256>(nz, zStride, slots, columns, bins, band, scale, tw, form, s);
        case 512: return forward_band_n<512>(nz, zStride, slots, columns, bins, band, scale, tw, form, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace skb
