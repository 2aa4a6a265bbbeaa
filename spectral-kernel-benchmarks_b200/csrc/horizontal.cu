// Horizontal transform kernels (row r2c/c2r along x, column c2c along y with
// fused retention/embedding).  See horizontal.hpp for the decomposition and
// fft_device.cuh for the shared-memory FFT.

#include "horizontal.hpp"

#include "fft_device.cuh"

namespace skb {
namespace {

// Batch width: 128-byte rows of complex values, capped so one CTA has at most
// 1024 threads (fft_threads(N) * B <= 1024).
template <typename T, int N>
constexpr int batch_width() {
    constexpr int natural = 128 / int(sizeof(cx<T>));
    constexpr int cap = N >= 8 ? 8192 / N : 1024;
    return natural < cap ? natural : cap;
}

template <typename T, int N>
constexpr int cta_threads() {
    return fft_threads(N) * batch_width<T, N>();
}

// ---------------------------------------------------------------------------
// Row forward: real rows of length NX = 2M -> bins kx in [0, keep).
// Grid (plane chunks, ny).  The real row is read as M complex pairs
// z[m] = x[2m] + i x[2m+1], transformed, then split into the real spectrum:
//   X[k] = (Z[k] + conj Z[M-k])/2 - i/2 * W^k (Z[k] - conj Z[M-k]),  W = e^{-2 pi i/NX}.
template <typename T, int M>
__global__ void __launch_bounds__(cta_threads<T, M>()) rows_forward_kernel(
    int ny, long long planes, int keep, const T* __restrict__ real, DenseBins bins, const cx<T>* __restrict__ twHalf,
    const cx<T>* __restrict__ twFull) {
    using V = cx<T>;
    constexpr int B = batch_width<T, M>();
    constexpr int NT = cta_threads<T, M>();
    extern __shared__ unsigned char smem_raw[];
    V* data = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;
    const long long p0 = (long long)blockIdx.x * B;
    const int y = blockIdx.y;
    constexpr int NX = 2 * M;
    constexpr int LD = B + 1;  // padded so the walk along x below is conflict-free
    // Consecutive threads take consecutive x-pairs of one row: full-line loads,
    // all of a thread's loads issued before the first shared store.
    static_assert((M * B) % NT == 0, "whole load rounds");
#pragma unroll
    for (int it = 0; it < (M * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int m = idx % M;
        const int b = idx / M;
        const long long p = p0 + b;
        V v = {T(0), T(0)};
        if (p < planes) v = *reinterpret_cast<const V*>(real + (p * ny + y) * NX + 2 * m);
        data[m * LD + b] = v;
    }
    __syncthreads();
    fft_smem<T, M, B, -1, LD>(data, twHalf, tid, true);
    V* out = reinterpret_cast<V*>(bins.data);
    for (int idx = tid; idx < keep * B; idx += NT) {
        const int b = idx % B;
        const int k = idx / B;
        const long long p = p0 + b;
        if (p >= planes) continue;
        V X;
        const V z0 = data[b];
        if (k == 0) {
            X = {z0.x + z0.y, T(0)};
        } else if (k == M) {
            X = {z0.x - z0.y, T(0)};
        } else {
            const V zk = data[k * LD + b];
            const V zm = cconj(data[(M - k) * LD + b]);
            const V e = cscale(cadd(zk, zm), T(0.5));
            const V d = csub(zk, zm);
            // o = -i/2 * d
            const V o = {T(0.5) * d.y, T(-0.5) * d.x};
            X = cadd(e, cmul(__ldg(twFull + k), o));
        }
        out[p + bins.planes * ((long long)k + bins.kxStride * y)] = X;
    }
}

// Row inverse: bins kx in [0, keep) (zero above) -> real rows, unnormalised,
// with FFTW's c2r semantics (imaginary parts of the kx = 0 and kx = NX/2 bins
// are ignored).  Pre-process Z[k] = (X[k] + conj X[M-k]) + i e^{+2 pi i k/NX}
// (X[k] - conj X[M-k]), then an inverse length-M FFT gives x[2m] + i x[2m+1].
template <typename T, int M>
__global__ void __launch_bounds__(cta_threads<T, M>()) rows_inverse_kernel(
    int ny, long long planes, int keep, DenseBins bins, T* __restrict__ real, const cx<T>* __restrict__ twHalf,
    const cx<T>* __restrict__ twFull) {
    using V = cx<T>;
    constexpr int B = batch_width<T, M>();
    constexpr int NT = cta_threads<T, M>();
    extern __shared__ unsigned char smem_raw[];
    V* data = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;
    const long long p0 = (long long)blockIdx.x * B;
    const int y = blockIdx.y;
    constexpr int NX = 2 * M;
    constexpr int LD = B + 1;
    const V* in = reinterpret_cast<const V*>(bins.data);
    auto load = [&](int k, int b) -> V {
        const long long p = p0 + b;
        if (k >= keep || p >= planes) return V{T(0), T(0)};
        V v = in[p + bins.planes * ((long long)k + bins.kxStride * y)];
        if (k == 0 || k == M) v.y = T(0);
        return v;
    };
    // Pairs (k, M-k) for k in [0, M/2]; k = 0 pairs with the Nyquist bin M.
    constexpr int pairs = M / 2 + 1;
    // FP64 issues all of a thread's loads first; FP32 measured faster rolled.
    constexpr int kUnroll = sizeof(T) == 8 ? (pairs * B + NT - 1) / NT : 1;
#pragma unroll kUnroll
    for (int it = 0; it < (pairs * B + NT - 1) / NT; ++it) {
        const int idx = tid + it * NT;
        if (idx >= pairs * B) break;
        const int b = idx % B;
        const int k = idx / B;
        if (k == 0) {
            const V x0 = load(0, b);
            const V xm = load(M, b);
            data[b] = {x0.x + xm.x, x0.x - xm.x};
            continue;
        }
        const int kk = M - k;
        const V xk = load(k, b);
        const V xm = load(kk, b);
        {
            const V s = cadd(xk, cconj(xm));
            const V d = csub(xk, cconj(xm));
            const V t = cmulc(d, __ldg(twFull + k));  // d * e^{+2 pi i k/NX}
            data[k * LD + b] = {s.x - t.y, s.y + t.x};   // s + i t
        }
        if (kk != k) {
            const V s = cadd(xm, cconj(xk));
            const V d = csub(xm, cconj(xk));
            const V t = cmulc(d, __ldg(twFull + kk));
            data[kk * LD + b] = {s.x - t.y, s.y + t.x};
        }
    }
    __syncthreads();
    fft_smem<T, M, B, +1, LD>(data, twHalf, tid, true);
    // Consecutive threads write consecutive x-pairs of one row.
#pragma unroll
    for (int it = 0; it < (M * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int m = idx % M;
        const int b = idx / M;
        const long long p = p0 + b;
        if (p < planes) *reinterpret_cast<V*>(real + (p * ny + y) * NX + 2 * m) = data[m * LD + b];
    }
}

// Length-1 rows (Nx = 2): X[0] = x0 + x1, X[1] = x0 - x1.
template <typename T>
__global__ void rows_pair_kernel(int dir, int ny, long long planes, int keep, const T* __restrict__ realIn,
                                 T* __restrict__ realOut, DenseBins bins) {
    using V = cx<T>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= planes * ny) return;
    const long long p = i % planes;
    const long long y = i / planes;
    V* b = reinterpret_cast<V*>(bins.data);
    if (dir < 0) {
        const T x0 = realIn[(p * ny + y) * 2], x1 = realIn[(p * ny + y) * 2 + 1];
        b[p + bins.planes * (0 + bins.kxStride * y)] = {x0 + x1, T(0)};
        if (keep > 1) b[p + bins.planes * (1 + bins.kxStride * y)] = {x0 - x1, T(0)};
    } else {
        const T a = b[p + bins.planes * (0 + bins.kxStride * y)].x;
        const T c = keep > 1 ? b[p + bins.planes * (1 + bins.kxStride * y)].x : T(0);
        realOut[(p * ny + y) * 2] = a + c;
        realOut[(p * ny + y) * 2 + 1] = a - c;
    }
}

// ---------------------------------------------------------------------------
// Column transforms.  Grid (plane chunks, columns).

template <typename T>
__device__ __forceinline__ cx<T> view_load(const FieldView& v, long long mode, int z) {
    const long long i = z + v.modeStride * mode;
    if (v.im == nullptr) return reinterpret_cast<const cx<T>*>(v.re)[i];
    return {reinterpret_cast<const T*>(v.re)[i], reinterpret_cast<const T*>(v.im)[i]};
}

template <typename T>
__device__ __forceinline__ void view_store(const FieldView& v, long long mode, int z, cx<T> x) {
    const long long i = z + v.modeStride * mode;
    if (v.im == nullptr) {
        reinterpret_cast<cx<T>*>(v.re)[i] = x;
    } else {
        reinterpret_cast<T*>(v.re)[i] = x.x;
        reinterpret_cast<T*>(v.im)[i] = x.y;
    }
}

template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(cta_threads<T, N>()) columns_dense_kernel(long long planes, DenseBins in,
                                                                            DenseBins out,
                                                                            const cx<T>* __restrict__ tw) {
    using V = cx<T>;
    constexpr int B = batch_width<T, N>();
    constexpr int NT = cta_threads<T, N>();
    extern __shared__ unsigned char smem_raw[];
    V* data = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;
    const long long p0 = (long long)blockIdx.x * B;
    const long long kx = blockIdx.y;
    const V* src = reinterpret_cast<const V*>(in.data);
    static_assert((N * B) % NT == 0, "whole load rounds");
#pragma unroll
    for (int it = 0; it < (N * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int b = idx % B;
        const int ky = idx / B;
        const long long p = p0 + b;
        V v = {T(0), T(0)};
        if (p < planes) v = src[p + in.planes * (kx + in.kxStride * ky)];
        data[ky * B + b] = v;
    }
    __syncthreads();
    fft_smem<T, N, B, SIGN>(data, tw, tid, true);
    V* dst = reinterpret_cast<V*>(out.data);
#pragma unroll
    for (int it = 0; it < (N * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int b = idx % B;
        const int ky = idx / B;
        const long long p = p0 + b;
        if (p < planes) dst[p + out.planes * (kx + out.kxStride * ky)] = data[ky * B + b];
    }
}

// Inverse column with retained-mode input: chunk c covers view f = c / zChunks,
// z in [z0, z0+B).  Dense output plane index = f*nz + z.
template <typename T, int N>
__global__ void __launch_bounds__(cta_threads<T, N>()) columns_embed_kernel(int nz, ViewSet views, ModeTables tables,
                                                                            DenseBins out,
                                                                            const cx<T>* __restrict__ tw) {
    using V = cx<T>;
    constexpr int B = batch_width<T, N>();
    constexpr int NT = cta_threads<T, N>();
    extern __shared__ unsigned char smem_raw[];
    V* data = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const FieldView view = views.v[f];
    const int* map = tables.cellMap + (long long)kx * N;
    static_assert((N * B) % NT == 0, "whole load rounds");
    // FP64 issues all of a thread's loads first; FP32 measured faster rolled.
    constexpr int kUnroll = sizeof(T) == 8 ? (N * B) / NT : 1;
#pragma unroll kUnroll
    for (int it = 0; it < (N * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int b = idx % B;
        const int ky = idx / B;
        const int z = z0 + b;
        V v = {T(0), T(0)};
        const int e = __ldg(map + ky);
        if (e >= 0 && z < nz) {
            v = view_load<T>(view, e >> 1, z);
            if (e & 1) v = cconj(v);
        }
        data[ky * B + b] = v;
    }
    __syncthreads();
    fft_smem<T, N, B, +1>(data, tw, tid, true);
    V* dst = reinterpret_cast<V*>(out.data);
    const long long pBase = (long long)f * nz;
#pragma unroll
    for (int it = 0; it < (N * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int b = idx % B;
        const int ky = idx / B;
        const int z = z0 + b;
        if (z < nz) dst[pBase + z + out.planes * (kx + out.kxStride * ky)] = data[ky * B + b];
    }
}

// Forward column with retained-mode output.
template <typename T, int N>
__global__ void __launch_bounds__(cta_threads<T, N>()) columns_gather_kernel(int nz, DenseBins in, ViewSet views,
                                                                             ModeTables tables, T scale,
                                                                             const cx<T>* __restrict__ tw) {
    using V = cx<T>;
    constexpr int B = batch_width<T, N>();
    constexpr int NT = cta_threads<T, N>();
    extern __shared__ unsigned char smem_raw[];
    V* data = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;
    const int zChunks = (nz + B - 1) / B;
    const int f = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int kx = blockIdx.y;
    const V* src = reinterpret_cast<const V*>(in.data);
    const long long pBase = (long long)f * nz;
    static_assert((N * B) % NT == 0, "whole load rounds");
#pragma unroll
    for (int it = 0; it < (N * B) / NT; ++it) {
        const int idx = tid + it * NT;
        const int b = idx % B;
        const int ky = idx / B;
        const int z = z0 + b;
        V v = {T(0), T(0)};
        if (z < nz) v = src[pBase + z + in.planes * ((long long)kx + in.kxStride * ky)];
        data[ky * B + b] = v;
    }
    __syncthreads();
    fft_smem<T, N, B, -1>(data, tw, tid, true);
    const FieldView view = views.v[f];
    const int begin = __ldg(tables.colStart + kx);
    const int end = __ldg(tables.colStart + kx + 1);
    for (int idx = tid; idx < (end - begin) * B; idx += NT) {
        const int b = idx % B;
        const int e = begin + idx / B;
        const int z = z0 + b;
        if (z >= nz) continue;
        const int ky = __ldg(tables.colKy + e);
        const int mc = __ldg(tables.colMode + e);
        V v = cscale(data[ky * B + b], scale);
        if (mc & 1) v = cconj(v);
        view_store<T>(view, mc >> 1, z, v);
    }
}

// Plain retention from a dense spectrum: one thread per (mode, z) of a view.
template <typename T>
__global__ void gather_dense_kernel(int nz, long long modes, const int* __restrict__ modeKx,
                                    const int* __restrict__ modeKy, const unsigned char* __restrict__ modeConj,
                                    DenseBins in, ViewSet views, T scale) {
    using V = cx<T>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= modes * nz) return;
    const int z = int(i % nz);
    const long long m = i / nz;
    const V* src = reinterpret_cast<const V*>(in.data);
    V v = src[(long long)f * nz + z + in.planes * ((long long)__ldg(modeKx + m) + in.kxStride * __ldg(modeKy + m))];
    v = cscale(v, scale);
    if (__ldg(modeConj + m)) v = cconj(v);
    view_store<T>(views.v[f], m, z, v);
}

// Plain embedding into a dense spectrum: every cell of the column band is
// written (zero where no mode lands), so no separate clear is needed.
template <typename T>
__global__ void embed_dense_kernel(int ny, int nz, ViewSet views, ModeTables tables, DenseBins out) {
    using V = cx<T>;
    const int f = blockIdx.z;
    const int kx = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)ny * nz) return;
    const int z = int(i % nz);
    const int ky = int(i / nz);
    const int e = __ldg(tables.cellMap + (long long)kx * ny + ky);
    V v = {T(0), T(0)};
    if (e >= 0) {
        v = view_load<T>(views.v[f], e >> 1, z);
        if (e & 1) v = cconj(v);
    }
    reinterpret_cast<V*>(out.data)[(long long)f * nz + z + out.planes * ((long long)kx + out.kxStride * ky)] = v;
}

// ---------------------------------------------------------------------------
// Dispatch helpers.

template <typename T, int N>
size_t smem_bytes() {
    return size_t(N) * batch_width<T, N>() * sizeof(cx<T>);
}

// Row kernels pad each shared row by one element (stride B + 1).
template <typename T, int N>
size_t row_smem_bytes() {
    return size_t(N) * (batch_width<T, N>() + 1) * sizeof(cx<T>);
}

template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

#define SKB_LENGTH_SWITCH(n, ...)       \
    switch (n) {                        \
        case 2: { constexpr int L = 2; __VA_ARGS__; } break;       \
        case 4: { constexpr int L = 4; __VA_ARGS__; } break;       \
        case 8: { constexpr int L = 8; __VA_ARGS__; } break;       \
        case 16: { constexpr int L = 16; __VA_ARGS__; } break;     \
        case 32: { constexpr int L = 32; __VA_ARGS__; } break;     \
        case 64: { constexpr int L = 64; __VA_ARGS__; } break;     \
        case 128: { constexpr int L = 128; __VA_ARGS__; } break;   \
        case 256: { constexpr int L = 256; __VA_ARGS__; } break;   \
        case 512: { constexpr int L = 512; __VA_ARGS__; } break;   \
        case 1024: { constexpr int L = 1024; __VA_ARGS__; } break; \
        default: return cudaErrorInvalidValue;              \
    }

template <typename T>
cudaError_t rows_forward_t(int nx, int ny, long long planes, int keep, const void* real, DenseBins bins,
                           const void* twHalf, const void* twFull, cudaStream_t stream) {
    const int M = nx / 2;
    if (M == 1) {
        const long long n = planes * ny;
        rows_pair_kernel<T><<<unsigned((n + 255) / 256), 256, 0, stream>>>(-1, ny, planes, keep,
                                                                            static_cast<const T*>(real), nullptr, bins);
        return cudaGetLastError();
    }
    SKB_LENGTH_SWITCH(M, {
        constexpr int B = batch_width<T, L>();
        auto kernel = rows_forward_kernel<T, L>;
        const size_t bytes = row_smem_bytes<T, L>();
        cudaError_t err = allow_smem(kernel, bytes);
        if (err != cudaSuccess) return err;
        dim3 grid(unsigned((planes + B - 1) / B), unsigned(ny));
        kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(ny, planes, keep, static_cast<const T*>(real), bins,
                                                             static_cast<const cx<T>*>(twHalf),
                                                             static_cast<const cx<T>*>(twFull));
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t rows_inverse_t(int nx, int ny, long long planes, int keep, DenseBins bins, void* real,
                           const void* twHalf, const void* twFull, cudaStream_t stream) {
    const int M = nx / 2;
    if (M == 1) {
        const long long n = planes * ny;
        rows_pair_kernel<T><<<unsigned((n + 255) / 256), 256, 0, stream>>>(+1, ny, planes, keep, nullptr,
                                                                            static_cast<T*>(real), bins);
        return cudaGetLastError();
    }
    SKB_LENGTH_SWITCH(M, {
        constexpr int B = batch_width<T, L>();
        auto kernel = rows_inverse_kernel<T, L>;
        const size_t bytes = row_smem_bytes<T, L>();
        cudaError_t err = allow_smem(kernel, bytes);
        if (err != cudaSuccess) return err;
        dim3 grid(unsigned((planes + B - 1) / B), unsigned(ny));
        kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(ny, planes, keep, bins, static_cast<T*>(real),
                                                             static_cast<const cx<T>*>(twHalf),
                                                             static_cast<const cx<T>*>(twFull));
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t columns_dense_t(int sign, int ny, int columns, long long planes, DenseBins in, DenseBins out,
                            const void* tw, cudaStream_t stream) {
    SKB_LENGTH_SWITCH(ny, {
        constexpr int B = batch_width<T, L>();
        const size_t bytes = smem_bytes<T, L>();
        dim3 grid(unsigned((planes + B - 1) / B), unsigned(columns));
        if (sign < 0) {
            auto kernel = columns_dense_kernel<T, L, -1>;
            cudaError_t err = allow_smem(kernel, bytes);
            if (err != cudaSuccess) return err;
            kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(planes, in, out, static_cast<const cx<T>*>(tw));
        } else {
            auto kernel = columns_dense_kernel<T, L, +1>;
            cudaError_t err = allow_smem(kernel, bytes);
            if (err != cudaSuccess) return err;
            kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(planes, in, out, static_cast<const cx<T>*>(tw));
        }
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t columns_embed_t(int ny, int nz, int columns, const ViewSet& views, const ModeTables& tables,
                            DenseBins out, const void* tw, cudaStream_t stream) {
    SKB_LENGTH_SWITCH(ny, {
        constexpr int B = batch_width<T, L>();
        const size_t bytes = smem_bytes<T, L>();
        auto kernel = columns_embed_kernel<T, L>;
        cudaError_t err = allow_smem(kernel, bytes);
        if (err != cudaSuccess) return err;
        const int zChunks = (nz + B - 1) / B;
        dim3 grid(unsigned(zChunks * views.count), unsigned(columns));
        kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(nz, views, tables, out, static_cast<const cx<T>*>(tw));
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t columns_gather_t(int ny, int nz, int columns, DenseBins in, const ViewSet& views,
                             const ModeTables& tables, double scale, const void* tw, cudaStream_t stream) {
    SKB_LENGTH_SWITCH(ny, {
        constexpr int B = batch_width<T, L>();
        const size_t bytes = smem_bytes<T, L>();
        auto kernel = columns_gather_kernel<T, L>;
        cudaError_t err = allow_smem(kernel, bytes);
        if (err != cudaSuccess) return err;
        const int zChunks = (nz + B - 1) / B;
        dim3 grid(unsigned(zChunks * views.count), unsigned(columns));
        kernel<<<grid, cta_threads<T, L>(), bytes, stream>>>(nz, in, views, tables, T(scale),
                                                             static_cast<const cx<T>*>(tw));
    });
    return cudaGetLastError();
}

}  // namespace

bool supported_length(long long n) { return n >= 2 && n <= 1024 && (n & (n - 1)) == 0; }

cudaError_t launch_rows_forward(Precision p, int nx, int ny, long long planes, int keep, const void* real,
                                DenseBins bins, const void* twHalf, const void* twFull, cudaStream_t stream) {
    if (planes <= 0) return cudaSuccess;
    return p == Precision::f64 ? rows_forward_t<double>(nx, ny, planes, keep, real, bins, twHalf, twFull, stream)
                               : rows_forward_t<float>(nx, ny, planes, keep, real, bins, twHalf, twFull, stream);
}

cudaError_t launch_rows_inverse(Precision p, int nx, int ny, long long planes, int keep, DenseBins bins, void* real,
                                const void* twHalf, const void* twFull, cudaStream_t stream) {
    if (planes <= 0) return cudaSuccess;
    return p == Precision::f64 ? rows_inverse_t<double>(nx, ny, planes, keep, bins, real, twHalf, twFull, stream)
                               : rows_inverse_t<float>(nx, ny, planes, keep, bins, real, twHalf, twFull, stream);
}

cudaError_t launch_columns_dense(Precision p, int sign, int ny, int columns, long long planes, DenseBins in,
                                 DenseBins out, const void* tw, cudaStream_t stream) {
    if (planes <= 0 || columns <= 0) return cudaSuccess;
    return p == Precision::f64 ? columns_dense_t<double>(sign, ny, columns, planes, in, out, tw, stream)
                               : columns_dense_t<float>(sign, ny, columns, planes, in, out, tw, stream);
}

cudaError_t launch_columns_embed(Precision p, int ny, int nz, int columns, const ViewSet& views,
                                 const ModeTables& tables, DenseBins out, const void* tw, cudaStream_t stream) {
    if (views.count <= 0 || columns <= 0) return cudaSuccess;
    return p == Precision::f64 ? columns_embed_t<double>(ny, nz, columns, views, tables, out, tw, stream)
                               : columns_embed_t<float>(ny, nz, columns, views, tables, out, tw, stream);
}

cudaError_t launch_columns_gather(Precision p, int ny, int nz, int columns, DenseBins in, const ViewSet& views,
                                  const ModeTables& tables, double scale, const void* tw, cudaStream_t stream) {
    if (views.count <= 0 || columns <= 0) return cudaSuccess;
    return p == Precision::f64 ? columns_gather_t<double>(ny, nz, columns, in, views, tables, scale, tw, stream)
                               : columns_gather_t<float>(ny, nz, columns, in, views, tables, scale, tw, stream);
}

cudaError_t launch_gather_dense(Precision p, int ny, int nz, long long modes, const int* modeKx, const int* modeKy,
                                const unsigned char* modeConj, DenseBins in, const ViewSet& views, double scale,
                                cudaStream_t stream) {
    (void)ny;
    if (modes <= 0 || views.count <= 0) return cudaSuccess;
    const long long n = modes * nz;
    dim3 grid(unsigned((n + 255) / 256), unsigned(views.count));
    if (p == Precision::f64)
        gather_dense_kernel<double><<<grid, 256, 0, stream>>>(nz, modes, modeKx, modeKy, modeConj, in, views, scale);
    else
        gather_dense_kernel<float><<<grid, 256, 0, stream>>>(nz, modes, modeKx, modeKy, modeConj, in, views,
                                                             float(scale));
    return cudaGetLastError();
}

cudaError_t launch_embed_dense(Precision p, int ny, int nz, int columns, const ViewSet& views,
                               const ModeTables& tables, DenseBins out, cudaStream_t stream) {
    if (views.count <= 0 || columns <= 0) return cudaSuccess;
    const long long n = (long long)ny * nz;
    dim3 grid(unsigned((n + 255) / 256), unsigned(columns), unsigned(views.count));
    if (p == Precision::f64)
        embed_dense_kernel<double><<<grid, 256, 0, stream>>>(ny, nz, views, tables, out);
    else
        embed_dense_kernel<float><<<grid, 256, 0, stream>>>(ny, nz, views, tables, out);
    return cudaGetLastError();
}

}  // namespace skb
