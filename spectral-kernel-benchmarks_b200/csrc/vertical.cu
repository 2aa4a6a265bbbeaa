// SIMT grouped vertical GEMM (FP64 / FP32).  See vertical.hpp.
//
// One CTA of 256 threads computes a tile of 32 complex columns of one K^2
// group, all R output rows.  The inner dimension S is streamed through shared
// memory in chunks of 32 with a two-stage cp.async pipeline (chunk c+1 is in
// flight while chunk c is consumed): the chunk of the group's transposed
// matrix At[s][r] (prepared at set-up) and of the input columns in[c][s].  Lane l of
// warp w owns rows r = l + 32k and columns c = w + 8m, so each step of s reads
// a 32-wide contiguous row of At (conflict-free) and a broadcast input value,
// and the final stores of out[c][r] are contiguous across the warp.

#include "vertical.hpp"

#include "fft_device.cuh"

namespace skb {
namespace {

constexpr int kTileCols = 32;
constexpr int kChunk = 32;
constexpr int kThreads = 256;

template <typename T, bool SPLIT>
__device__ __forceinline__ cx<T> load_operand(const ComplexOperand& op, long long i) {
    if (SPLIT) return {reinterpret_cast<const T*>(op.re)[i], reinterpret_cast<const T*>(op.im)[i]};
    return reinterpret_cast<const cx<T>*>(op.re)[i];
}

template <typename T, bool SPLIT>
__device__ __forceinline__ void store_operand(const ComplexOperand& op, long long i, cx<T> v) {
    if (SPLIT) {
        reinterpret_cast<T*>(op.re)[i] = v.x;
        reinterpret_cast<T*>(op.im)[i] = v.y;
    } else {
        reinterpret_cast<cx<T>*>(op.re)[i] = v;
    }
}

// Asynchronous 4/8/16-byte global->shared copy; src_bytes = 0 writes zeros.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src, int src_bytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(src), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Element offset of plan column `col` (member * memberColumns + mode * fields
// + field) in a cell-addressed operand, with its partner (or -1) and
// conjugation.
__device__ __forceinline__ void bin_column(const BinBoundary& bb, int col, long long& base, long long& partner,
                                           bool& conj) {
    // Plan column = member * memberColumns + mode * fields + plan field.
    long long member = 0;
    int rest = col;
    if (bb.memberColumns > 0) {
        member = col / bb.memberColumns;
        rest = static_cast<int>(col - member * bb.memberColumns);
    }
    const int mode = rest / bb.fields;
    const int sub = rest - mode * bb.fields;
    const int field = bb.fieldMap != nullptr ? __ldg(bb.fieldMap + sub) : sub;
    const long long memberStride =
        bb.memberStride != 0 ? bb.memberStride : static_cast<long long>(bb.fields) * bb.zStride;
    const long long off = member * memberStride + static_cast<long long>(field) * bb.zStride;
    base = __ldg(bb.cell + mode) + off;
    const long long p = bb.partner != nullptr ? __ldg(bb.partner + mode) : -1;
    partner = p >= 0 ? p + off : -1;
    conj = bb.conj != nullptr && __ldg(bb.conj + mode) != 0;
}

template <typename T, int KR, bool SPLIT, bool BINS, bool VIRT>
__global__ void __launch_bounds__(kThreads) grouped_gemm_kernel(int R, int S, const T* __restrict__ At,
                                                                GroupTiles tiles, ComplexOperand in,
                                                                ComplexOperand out, BinBoundary inBins,
                                                                BinBoundary outBins) {
    using V = cx<T>;
    constexpr int RP = 32 * KR;
    constexpr size_t xBytes = sizeof(V) * kTileCols * (kChunk + 1);
    constexpr size_t aBytes = sizeof(T) * kChunk * RP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // Per tile column: element offsets of the input and output columns (and
    // the output partner), and the conjugation flags.
    __shared__ long long colIn[kTileCols], colOut[kTileCols], colPartner[kTileCols];
    __shared__ signed char conjIn[kTileCols], conjOut[kTileCols];
    const int tile = blockIdx.x;
    const int g = __ldg(tiles.tileGroup + tile);
    const int c0 = __ldg(tiles.tileColumn + tile);  // first global (member tiles) or virtual column
    const int ncols = __ldg(tiles.tileCount + tile);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (!VIRT && BINS && threadIdx.x < kTileCols) {
        const int c = threadIdx.x;
        long long base = static_cast<long long>(c0 + c) * S, partner = -1;
        bool conj = false;
        if (inBins.cell != nullptr && c < ncols) bin_column(inBins, c0 + c, base, partner, conj);
        colIn[c] = base;
        conjIn[c] = conj ? 1 : 0;
        base = static_cast<long long>(c0 + c) * R;
        partner = -1;
        conj = false;
        if (outBins.cell != nullptr && c < ncols) bin_column(outBins, c0 + c, base, partner, conj);
        colOut[c] = base;
        colPartner[c] = partner;
        conjOut[c] = conj ? 1 : 0;
    }
    if (!VIRT && BINS) __syncthreads();
    // Virtual tiles: warp w copies, multiplies and stores the tile columns
    // w + 8m (m < 4), so its lanes 0..3 resolve exactly those and a warp
    // barrier suffices.
    if (VIRT && lane < kTileCols / 8) {
        const int per = __ldg(tiles.tilePer + tile);
        const int first = __ldg(tiles.tileFirst + tile);
        // Virtual column c0 + c of group g -> global plan column.
        const int c = warp + 8 * lane;
        long long inBase = 0, outBase = 0, partner = -1;
        bool cIn = false, cOut = false;
        if (c < ncols) {
            const int v = c0 + c;
            const int member = v / per;
            const long long col = member * tiles.memberColumns + first + (v - member * per);
            inBase = col * S;
            outBase = col * R;
            long long unused = -1;
            if (BINS && inBins.cell != nullptr) bin_column(inBins, static_cast<int>(col), inBase, unused, cIn);
            if (BINS && outBins.cell != nullptr) bin_column(outBins, static_cast<int>(col), outBase, partner, cOut);
        }
        colIn[c] = inBase;
        conjIn[c] = cIn ? 1 : 0;
        colOut[c] = outBase;
        colPartner[c] = partner;
        conjOut[c] = cOut ? 1 : 0;
    }
    if (VIRT) __syncwarp();
    const T* A = At + g * tiles.matrixStride;
    const int chunks = (S + kChunk - 1) / kChunk;

    auto stageX = [&](int b) { return reinterpret_cast<V(*)[kChunk + 1]>(smem_raw + b * (xBytes + aBytes)); };
    auto stageA = [&](int b) { return reinterpret_cast<T(*)[RP]>(smem_raw + b * (xBytes + aBytes) + xBytes); };

    // Issue the copies of chunk c into stage buffer b (zero-filled padding).
    auto issue = [&](int c, int b) {
        const int s0 = c * kChunk;
        T(*sA)[RP] = stageA(b);
        V(*sX)[kChunk + 1] = stageX(b);
        for (int i = threadIdx.x; i < kChunk * RP; i += kThreads) {
            const int s = i / RP, r = i % RP;
            const bool ok = s0 + s < S && r < R;
            const T* src = ok ? A + (long long)(s0 + s) * R + r : A;
            cp_async<sizeof(T)>(&sA[s][r], src, ok ? int(sizeof(T)) : 0);
        }
        for (int i = threadIdx.x; i < kTileCols * kChunk; i += kThreads) {
            const int c = i / kChunk, s = i % kChunk;
            const bool ok = c < ncols && s0 + s < S;
            const long long idx = ok ? ((VIRT || BINS) ? colIn[c] : (long long)(c0 + c) * S) + s0 + s : 0;
            if (SPLIT) {
                // Split operands: two scalar copies into the complex slot.
                T* slot = reinterpret_cast<T*>(&sX[c][s]);
                cp_async<sizeof(T)>(slot, reinterpret_cast<const T*>(in.re) + idx, ok ? int(sizeof(T)) : 0);
                cp_async<sizeof(T)>(slot + 1, reinterpret_cast<const T*>(in.im) + idx, ok ? int(sizeof(T)) : 0);
            } else {
                cp_async<sizeof(V)>(&sX[c][s], reinterpret_cast<const V*>(in.re) + idx, ok ? int(sizeof(V)) : 0);
            }
        }
        cp_async_commit();
    };

    V acc[KR][kTileCols / 8];
#pragma unroll
    for (int k = 0; k < KR; ++k)
#pragma unroll
        for (int m = 0; m < kTileCols / 8; ++m) acc[k][m] = {T(0), T(0)};

    issue(0, 0);
    for (int c = 0; c < chunks; ++c) {
        if (c + 1 < chunks) {
            issue(c + 1, (c + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        T(*sA)[RP] = stageA(c & 1);
        V(*sX)[kChunk + 1] = stageX(c & 1);
        const int sc = min(kChunk, S - c * kChunk);
#pragma unroll 4
        for (int s = 0; s < sc; ++s) {
            T a[KR];
#pragma unroll
            for (int k = 0; k < KR; ++k) a[k] = sA[s][lane + 32 * k];
#pragma unroll
            for (int m = 0; m < kTileCols / 8; ++m) {
                const V x = sX[warp + 8 * m][s];
#pragma unroll
                for (int k = 0; k < KR; ++k) {
                    acc[k][m].x = fma(a[k], x.x, acc[k][m].x);
                    acc[k][m].y = fma(a[k], x.y, acc[k][m].y);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < kTileCols / 8; ++m) {
        const int c = warp + 8 * m;
        if (c >= ncols) continue;
#pragma unroll
        for (int k = 0; k < KR; ++k) {
            const int r = lane + 32 * k;
            if (r >= R) continue;
            // The matrices are real, so a conjugated input column gives the
            // conjugate product: both flags are applied here, once.
            V v = acc[k][m];
            if (!VIRT && !BINS) {
                store_operand<T, SPLIT>(out, (long long)(c0 + c) * R + r, v);
                continue;
            }
            if (conjIn[c] != conjOut[c]) v.y = -v.y;
            store_operand<T, SPLIT>(out, colOut[c] + r, v);
            if (colPartner[c] >= 0) store_operand<T, SPLIT>(out, colPartner[c] + r, V{v.x, -v.y});
        }
    }
}

template <typename T, int KR>
cudaError_t launch_kr(int R, int S, const void* At, const GroupTiles& tiles, ComplexOperand in, ComplexOperand out,
                      const BinBoundary& inBins, const BinBoundary& outBins, cudaStream_t stream) {
    const bool split = in.im != nullptr;
    if (split != (out.im != nullptr)) return cudaErrorInvalidValue;
    const size_t bytes = 2 * (sizeof(cx<T>) * kTileCols * (kChunk + 1) + sizeof(T) * kChunk * 32 * KR);
    const bool bins = inBins.cell != nullptr || outBins.cell != nullptr;
    using K = void (*)(int, int, const T*, GroupTiles, ComplexOperand, ComplexOperand, BinBoundary, BinBoundary);
    // [split][bins][virtual]
    const K kernels[2][2][2] = {
        {{grouped_gemm_kernel<T, KR, false, false, false>, grouped_gemm_kernel<T, KR, false, false, true>},
         {grouped_gemm_kernel<T, KR, false, true, false>, grouped_gemm_kernel<T, KR, false, true, true>}},
        {{grouped_gemm_kernel<T, KR, true, false, false>, grouped_gemm_kernel<T, KR, true, false, true>},
         {grouped_gemm_kernel<T, KR, true, true, false>, grouped_gemm_kernel<T, KR, true, true, true>}}};
    const K kernel = kernels[split][bins][tiles.virtualColumns];
    if (bytes > 48 * 1024) {
        const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (err != cudaSuccess) return err;
    }
    kernel<<<tiles.tiles, kThreads, bytes, stream>>>(R, S, static_cast<const T*>(At), tiles, in, out, inBins,
                                                     outBins);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_t(int R, int S, const void* At, const GroupTiles& tiles, ComplexOperand in, ComplexOperand out,
                     const BinBoundary& ib, const BinBoundary& ob, cudaStream_t stream) {
    const int kr = (R + 31) / 32;
    switch (kr) {
        case 1: return launch_kr<T, 1>(R, S, At, tiles, in, out, ib, ob, stream);
        case 2: return launch_kr<T, 2>(R, S, At, tiles, in, out, ib, ob, stream);
        case 3: return launch_kr<T, 3>(R, S, At, tiles, in, out, ib, ob, stream);
        case 4: return launch_kr<T, 4>(R, S, At, tiles, in, out, ib, ob, stream);
        case 5: return launch_kr<T, 5>(R, S, At, tiles, in, out, ib, ob, stream);
        case 6: return launch_kr<T, 6>(R, S, At, tiles, in, out, ib, ob, stream);
        case 7:
        case 8:
        case 9: return launch_kr<T, 9>(R, S, At, tiles, in, out, ib, ob, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int gemm_tile_columns(GemmPrecision) { return kTileCols; }

cudaError_t launch_grouped_gemm(GemmPrecision p, int R, int S, const void* matrices, const GroupTiles& tiles,
                                ComplexOperand in, ComplexOperand out, cudaStream_t stream, const BinBoundary* inBins,
                                const BinBoundary* outBins) {
    if (tiles.tiles <= 0) return cudaSuccess;
    const BinBoundary ib = inBins ? *inBins : BinBoundary{};
    const BinBoundary ob = outBins ? *outBins : BinBoundary{};
    switch (p) {
        case GemmPrecision::f64: return launch_t<double>(R, S, matrices, tiles, in, out, ib, ob, stream);
        case GemmPrecision::f32: return launch_t<float>(R, S, matrices, tiles, in, out, ib, ob, stream);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace skb
