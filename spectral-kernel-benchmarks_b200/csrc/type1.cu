// Type-I (DCT-I / DST-I) vertical transforms, see type1.hpp.
//
// A DCT-I of length nz is the first nz outputs of the length-L = 2(nz-1) DFT
// of the column's even extension e (e_z = e_{L-z} = x_z); a DST-I of the
// interior is i times the DFT of the odd extension (o_z = -o_{L-z} = x_z,
// o_0 = o_{nz-1} = 0).  Both hold for complex columns because the transform
// matrices are real.  Each warp walks (row, channel) columns with a grid
// stride: it holds the next column's values in registers while it writes the
// current one's extension into its shared-memory slot, runs warp_fft and
// writes the nz results back over the column (all reads of a column finish
// before its first write, so the transform is in place).  Columns are
// contiguous in HBM, so each warp moves whole sectors; the bound is HBM
// traffic (one read and one write of every transformed value).

#include <algorithm>

#include "fft_device.cuh"
#include "type1.hpp"

namespace skb {
namespace {

constexpr int kWarps = 8;

template <typename T>
__device__ __forceinline__ void store_result(cx<T>* col, int k, cx<T> y, int M, bool sine, bool normalize) {
    using V = cx<T>;
    if (sine) {
        if (k == 0 || k == M) {
            if (normalize) col[k] = V{T(0), T(0)};
            return;
        }
    }
    if (normalize) {
        T s = T(1) / T(M);
        y = V{y.x * s, y.y * s};
        if (!sine && k == M) y = V{y.x * T(0.5), y.y * T(0.5)};
    }
    col[k] = y;
}

template <typename T, int L>
__global__ void __launch_bounds__(kWarps * 32) type1_fft_kernel(cx<T>* __restrict__ data, long long seqs, int storage,
                                                                int first, int channels, unsigned dstMask,
                                                                bool normalize, const cx<T>* __restrict__ tw) {
    using V = cx<T>;
    constexpr int M = L / 2;
    constexpr int nz = M + 1;
    constexpr int kSlots = L + L / 16;  // pad16(L - 1) + 1
    constexpr int kPer = (nz + 31) / 32;  // column values per lane
    // Up to five values per lane are held for the next column while the
    // current one is transformed, so its loads overlap the FFT.
    constexpr bool kPrefetch = kPer <= 5;
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long stride = static_cast<long long>(gridDim.x) * kWarps;
    V* x = reinterpret_cast<V*>(smem_raw) + warp * kSlots;
    auto column = [&](long long sq) {
        const long long row = sq / channels;
        return data + (row * storage + first + (sq - row * channels)) * nz;
    };
    auto load = [&](long long sq, V* v) {
        const V* col = column(sq);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int i = lane + 32 * q;
            v[q] = i < nz ? col[i] : V{T(0), T(0)};
        }
    };
    long long seq = static_cast<long long>(blockIdx.x) * kWarps + warp;
    V cur[kPrefetch ? kPer : 1];
    if constexpr (kPrefetch) {
        if (seq < seqs) load(seq, cur);
    }
    // Warp-uniform loop; only __syncwarp() is used inside.
    for (; seq < seqs; seq += stride) {
        V* col = column(seq);
        const bool sine = (dstMask >> static_cast<int>(seq % channels)) & 1u;
        V nxt[kPrefetch ? kPer : 1];
        auto extend = [&](int i, V v) {
            if (sine && (i == 0 || i == M)) v = V{T(0), T(0)};
            x[pad16(i)] = v;
            if (i > 0 && i < M) x[pad16(L - i)] = sine ? V{-v.x, -v.y} : v;
        };
        if constexpr (kPrefetch) {
            if (seq + stride < seqs) load(seq + stride, nxt);
#pragma unroll
            for (int q = 0; q < kPer; ++q)
                if (lane + 32 * q < nz) extend(lane + 32 * q, cur[q]);
        } else {
            for (int i = lane; i < nz; i += 32) extend(i, col[i]);
        }
        __syncwarp();
        warp_fft<T, L, -1>(x, tw, lane);
        for (int k = lane; k < nz; k += 32) {
            V y = x[pad16(k)];
            if (sine) y = V{-y.y, y.x};  // i * X_k
            store_result<T>(col, k, y, M, sine, normalize);
        }
        __syncwarp();  // the slot is rewritten by the next column
        if constexpr (kPrefetch) {
#pragma unroll
            for (int q = 0; q < kPer; ++q) cur[q] = nxt[q];
        }
    }
}

// Any nz >= 3: each lane forms its outputs as direct sums with the cosine and
// sine of 2 pi m / L read from the twiddle table (m = k z mod L).
template <typename T>
__global__ void __launch_bounds__(kWarps * 32) type1_direct_kernel(cx<T>* __restrict__ data, long long seqs, int nz,
                                                                   int storage, int first, int channels,
                                                                   unsigned dstMask, bool normalize,
                                                                   const cx<T>* __restrict__ tw) {
    using V = cx<T>;
    const int M = nz - 1, L = 2 * M;
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long seq = static_cast<long long>(blockIdx.x) * kWarps + warp;
    if (seq >= seqs) return;
    const long long row = seq / channels;
    const int c = static_cast<int>(seq - row * channels);
    const bool sine = (dstMask >> c) & 1u;
    V* x = reinterpret_cast<V*>(smem_raw) + warp * nz;
    V* col = data + (row * storage + first + c) * nz;
    for (int i = lane; i < nz; i += 32) x[i] = col[i];
    __syncwarp();
    for (int k = lane; k < nz; k += 32) {
        V acc{T(0), T(0)};
        if (!sine) {
            const T sign = (k & 1) ? T(-1) : T(1);
            acc = V{x[0].x + sign * x[M].x, x[0].y + sign * x[M].y};
        }
        int m = 0;  // k z mod L, advanced incrementally
        for (int z = 1; z < M; ++z) {
            m += k;
            if (m >= L) m -= L;
            const V w = __ldg(tw + m);  // (cos, -sin) of 2 pi m / L
            const T f = sine ? T(-2) * w.y : T(2) * w.x;
            acc = V{acc.x + f * x[z].x, acc.y + f * x[z].y};
        }
        store_result<T>(col, k, acc, M, sine, normalize);
    }
}

template <typename T>
__global__ void type1_normalize_kernel(cx<T>* __restrict__ data, long long total, int nz, int storage, int first,
                                       int channels, unsigned dstMask) {
    using V = cx<T>;
    const int M = nz - 1;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total; i += stride) {
        const long long seq = i / nz;
        const int k = static_cast<int>(i - seq * nz);
        const long long row = seq / channels;
        const int c = static_cast<int>(seq - row * channels);
        const bool sine = (dstMask >> c) & 1u;
        V* col = data + (row * storage + first + c) * nz;
        if (sine && (k == 0 || k == M)) {
            col[k] = V{T(0), T(0)};
            continue;
        }
        const V v = col[k];
        T s = T(1) / T(M);
        V y{v.x * s, v.y * s};
        if (!sine && k == M) y = V{y.x * T(0.5), y.y * T(0.5)};
        col[k] = y;
    }
}

template <typename T, int L>
cudaError_t launch_fft(cx<T>* data, long long seqs, int storage, int first, int channels, unsigned mask, bool norm,
                       const cx<T>* tw, cudaStream_t s) {
    const size_t bytes = static_cast<size_t>(kWarps) * (L + L / 16) * sizeof(cx<T>);
    auto kernel = type1_fft_kernel<T, L>;
    // Resident blocks per SM and SM count, per device (each instantiation).
    static int cachedDevice = -1, cachedBlocks = 0;
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    if (device != cachedDevice) {
        if (bytes > 48 * 1024) {
            err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
            if (err != cudaSuccess) return err;
        }
        int perSm = 0, sms = 0;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kWarps * 32, bytes);
        if (err != cudaSuccess) return err;
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (err != cudaSuccess) return err;
        cachedBlocks = std::max(1, perSm) * std::max(1, sms);
        cachedDevice = device;
    }
    const long long blocks = std::min<long long>((seqs + kWarps - 1) / kWarps, cachedBlocks);
    kernel<<<static_cast<unsigned>(blocks), kWarps * 32, bytes, s>>>(data, seqs, storage, first, channels, mask, norm,
                                                                     tw);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_t(void* data, long long rows, int nz, int storage, int first, int channels, unsigned mask,
                     bool norm, const void* twv, cudaStream_t s) {
    auto* d = static_cast<cx<T>*>(data);
    const auto* tw = static_cast<const cx<T>*>(twv);
    const long long seqs = rows * channels;
    if (seqs == 0) return cudaSuccess;
    switch (2 * (nz - 1)) {
        case 8: return launch_fft<T, 8>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 16: return launch_fft<T, 16>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 32: return launch_fft<T, 32>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 64: return launch_fft<T, 64>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 128: return launch_fft<T, 128>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 256: return launch_fft<T, 256>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 512: return launch_fft<T, 512>(d, seqs, storage, first, channels, mask, norm, tw, s);
        case 1024: return launch_fft<T, 1024>(d, seqs, storage, first, channels, mask, norm, tw, s);
        default: break;
    }
    const size_t bytes = static_cast<size_t>(kWarps) * nz * sizeof(cx<T>);
    auto kernel = type1_direct_kernel<T>;
    if (bytes > 227 * 1024) return cudaErrorInvalidValue;
    if (bytes > 48 * 1024) {
        const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (err != cudaSuccess) return err;
    }
    const long long blocks = (seqs + kWarps - 1) / kWarps;
    if (blocks > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    kernel<<<static_cast<unsigned>(blocks), kWarps * 32, bytes, s>>>(d, seqs, nz, storage, first, channels, mask, norm,
                                                                     tw);
    return cudaGetLastError();
}

}  // namespace

bool type1_uses_fft(int nz) {
    const int L = 2 * (nz - 1);
    return L >= 8 && L <= 1024 && (L & (L - 1)) == 0;
}

cudaError_t launch_type1(bool f64, void* data, long long rows, int nz, int storageChannels, int first, int channels,
                         unsigned dstMask, bool normalize, const void* tw, cudaStream_t s) {
    if (nz < 3 || channels <= 0 || first < 0 || first + channels > storageChannels || channels > 32)
        return cudaErrorInvalidValue;
    return f64 ? launch_t<double>(data, rows, nz, storageChannels, first, channels, dstMask, normalize, tw, s)
               : launch_t<float>(data, rows, nz, storageChannels, first, channels, dstMask, normalize, tw, s);
}

cudaError_t launch_type1_normalize(bool f64, void* data, long long rows, int nz, int storageChannels, int first,
                                   int channels, unsigned dstMask, cudaStream_t s) {
    if (nz < 3 || channels <= 0 || first < 0 || first + channels > storageChannels || channels > 32)
        return cudaErrorInvalidValue;
    const long long total = rows * channels * nz;
    if (total == 0) return cudaSuccess;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 32));
    if (f64)
        type1_normalize_kernel<double><<<blocks, 256, 0, s>>>(static_cast<cx<double>*>(data), total, nz,
                                                              storageChannels, first, channels, dstMask);
    else
        type1_normalize_kernel<float><<<blocks, 256, 0, s>>>(static_cast<cx<float>*>(data), total, nz,
                                                             storageChannels, first, channels, dstMask);
    return cudaGetLastError();
}

}  // namespace skb
