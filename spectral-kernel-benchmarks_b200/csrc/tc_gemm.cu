// Tensor-core (tcgen05, sm_100a) grouped vertical GEMM in split TF32x3.
//
// Problem (see vertical.hpp): for each K^2 group g, out[c][r] = sum_s
// A_g[r][s] in[c][s] over the group's complex columns c.  It is issued as the
// transposed real product
//     D[m][n] = sum_k Aop[m][k] * Bop[n][k]
// with m = (column, re/im part) of the data (M = 128 rows = 64 complex
// columns per tile), n = r (N = R padded to a multiple of 16) and k = s.  Both
// operands are K-major: Bop is the group matrix in its natural row-major
// [r][s] layout, Aop is the data row in[c][0..S).
//
// Split precision: x = hi + lo with hi = rna_tf32(x), lo = rna_tf32(x - hi);
// D = Ahi*Blo + Alo*Bhi + Ahi*Bhi accumulated in FP32 in tensor memory, one
// accumulator per 32-wide K chunk, chunk sums added in FP32 registers.  The
// dropped lo*lo term is ~2^-22 relative.
//
// CTA work unit: one group and a run of up to 16 M-tiles of its (member,
// column) list.  The group matrix is split and written once into shared
// memory (all K chunks) and stays resident; data chunks of 32 k stream
// through a three-stage ring filled by producer warps while one MMA lane and
// the epilogue warps work on earlier chunks (warp specialisation below).  Operands use the canonical K-major
// SWIZZLE_128B layout: 8-row atoms of 8 x 128 bytes, 16-byte chunk q of row
// n stored at chunk (q xor n%8).  One elected thread issues the MMAs and
// commits them to the stage's mbarrier; every wait is bounded and reports
// through `error` instead of hanging.

#include <cstdint>

#include "vertical.hpp"

namespace skb {
namespace {

constexpr int kTileRows = 128;    // M
constexpr int kChunkK = 32;       // tf32 elements per 128-byte row
constexpr int kTmemCols = 512;  // two chunk accumulators + the running sum, NP columns each
constexpr int kStageBytes = 2 * kTileRows * 128;  // hi + lo
constexpr long long kWaitLimit = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
// Gives up early once any CTA of the launch has reported an expired wait.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const int* error) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023) == 1023 && *reinterpret_cast<const volatile int*>(error) != 0) return false;
    }
    return false;
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_x8(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_st_x8(uint32_t taddr, const uint32_t (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// K-major SWIZZLE_128B descriptor: SBO = 1024 B between 8-row atoms, LBO
// unused (16 B), descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
           (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
           (static_cast<uint64_t>(2) << 61);
}

// Byte offset of (row, 16-byte chunk q) inside a swizzled operand.
__device__ __forceinline__ uint32_t sw128_offset(int row, int q) {
    return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((q ^ (row & 7)) << 4));
}

struct Split4 {
    float4 hi, lo;
};

__device__ __forceinline__ Split4 split4(float a, float b, float c, float d) {
    Split4 s;
    s.hi = make_float4(tf32_rna(a), tf32_rna(b), tf32_rna(c), tf32_rna(d));
    s.lo = make_float4(tf32_rna(a - s.hi.x), tf32_rna(b - s.hi.y), tf32_rna(c - s.hi.z), tf32_rna(d - s.hi.w));
    return s;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp roles of the pipelined kernel.
constexpr int kProducerWarps = 8;
constexpr int kMmaWarp = kProducerWarps;
constexpr int kEpilogueWarps = 8;
constexpr int kPipeThreads = (kProducerWarps + 1 + kEpilogueWarps) * 32;
constexpr int kStages = 3;
constexpr int kAccumulators = 2;
constexpr int kEpiStride = 17;  // floats per column row of an epilogue warp's transpose buffer
constexpr int kEpiBytes = kEpilogueWarps * 16 * kEpiStride * 4;

struct PipeState {
    uint64_t full[kStages], empty[kStages], accFull[kAccumulators], accEmpty[kAccumulators], done;
    uint32_t tmem;
};

// Where virtual column vc of a group lives: element offset of its first
// value, its Hermitian partner (or -1) and whether the stored value is the
// conjugate.  `len` is the compact column length.
struct ColumnRef {
    long long base, partner;
    bool conj;
};
__device__ __forceinline__ ColumnRef column_ref(const TcGemmArgs& p, const BinBoundary& bb, int vc, int gcols,
                                                long long gfirst, int len) {
    const int member = vc / gcols;
    const int c = static_cast<int>(gfirst) + (vc - member * gcols);  // column within the member (< 2^31)
    if (bb.cell == nullptr) return {(static_cast<long long>(member) * p.memberColumns + c) * len, -1, false};
    const int mode = c / bb.fields;
    const int field = c - mode * bb.fields;
    const long long off = (static_cast<long long>(member) * bb.fields + field) * bb.zStride;
    const long long partner = bb.partner != nullptr ? __ldg(bb.partner + mode) : -1;
    const bool conj = bb.conj != nullptr && __ldg(bb.conj + mode) != 0;
    return {__ldg(bb.cell + mode) + off, partner >= 0 ? partner + off : -1, conj};
}

// Warp-specialised split-TF32x3 grouped GEMM.
//   producer warps 0-7: data chunk (64 columns x 32 k) -> registers -> TF32
//       hi/lo -> swizzled A stage of a 3-deep ring; arrive full[stage].
//   MMA warp 8 (one lane): per chunk, 3 MMAs per k-step into one of two
//       ping-pong TMEM chunk accumulators; commit empty[stage] and accFull.
//   epilogue warps 9-16: add each chunk accumulator into an FP32 running sum
//       kept in TMEM (tcgen05.ld / tcgen05.st), release it (accEmpty), and
//       after the tile's last chunk write the tile's outputs.
// NPH = NP/16: x8 column blocks per epilogue half.
template <int NPH>
__global__ void __launch_bounds__(kPipeThreads, 1) tc_gemm_pipe_kernel(TcGemmArgs p) {
    constexpr int NP = NPH * 16;
    constexpr int HALF = NP / 2;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int KCH = p.KCH, R = p.R, S = p.S;
    unsigned char* sBhi = base;
    unsigned char* sBlo = sBhi + KCH * NP * 128;
    unsigned char* sA = sBlo + KCH * NP * 128;
    PipeState* st = reinterpret_cast<PipeState*>(sA + kStages * kStageBytes);

    const int unit = blockIdx.x;
    const int g = __ldg(p.unitGroup + unit);
    const int vc0 = __ldg(p.unitColumn + unit);
    const int vcN = __ldg(p.unitCount + unit);
    const int gcols = __ldg(p.groupColumns + g);
    const long long gfirst = __ldg(p.groupFirst + g);
    const int tiles = (vcN + 63) / 64;

    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(smem_u32(&st->full[i]), kProducerWarps * 32);
            mbar_init(smem_u32(&st->empty[i]), 1);
        }
        for (int i = 0; i < kAccumulators; ++i) {
            mbar_init(smem_u32(&st->accFull[i]), 1);
            mbar_init(smem_u32(&st->accEmpty[i]), kEpilogueWarps * 32);
        }
        mbar_init(smem_u32(&st->done), 1);
        fence_barrier_init();
    }
    if (warp == kMmaWarp) {
        tmem_alloc(smem_u32(&st->tmem), kTmemCols);
        tmem_relinquish();
    }
    // L2 prefetch of one tile's data columns (S complex each), 128-byte lines.
    auto prefetch_tile = [&](int t) {
        const int tv0 = vc0 + t * 64;
        const int tcount = min(64, vc0 + vcN - tv0);
        const int lines = (S * 8 + 127) / 128 + 1;
        for (int i = tid; i < tcount * lines; i += kProducerWarps * 32) {
            const int cl = i / lines, l = i % lines;
            const char* col =
                reinterpret_cast<const char*>(p.in + column_ref(p, p.inBins, tv0 + cl, gcols, gfirst, S).base);
            const char* line = reinterpret_cast<const char*>(reinterpret_cast<uintptr_t>(col) & ~uintptr_t(127)) + 128 * l;
            if (line < col + S * 8) asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
        }
    };
    if (warp < kProducerWarps) prefetch_tile(0);
    // Resident group matrix, split hi/lo, zero-padded to NP x KCH*32.
    const float* Bg = p.B + static_cast<long long>(g) * R * S;
    for (int item = tid; item < NP * KCH * 8; item += kPipeThreads) {
        const int q = item & 7;
        const int rest = item >> 3;
        const int kc = rest % KCH;
        const int n = rest / KCH;
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int s = kc * kChunkK + q * 4 + j;
            v[j] = (n < R && s < S) ? __ldg(Bg + static_cast<long long>(n) * S + s) : 0.0f;
        }
        const Split4 sp = split4(v[0], v[1], v[2], v[3]);
        const uint32_t off = kc * NP * 128 + sw128_offset(n, q);
        *reinterpret_cast<float4*>(sBhi + off) = sp.hi;
        *reinterpret_cast<float4*>(sBlo + off) = sp.lo;
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = st->tmem;
    bool failed = false;

    if (warp < kProducerWarps) {
        // ---------------------------------------------------------- producer
        // Chunk it+1's loads are issued before chunk it is converted, so two
        // chunks of each warp's loads are in flight.  Warp w converts columns
        // 8w .. 8w+7 of a tile; lane = k within the chunk, so each load
        // instruction reads one column's 32 consecutive complex values (256
        // contiguous bytes) and each shared store fills one 128-byte row.
        const int total = tiles * KCH;
        long long colBase[8];
        unsigned conjMask = 0;  // bit c: column c of the tile is stored conjugated
        int loadTile = -1, loadCount = 0;
        auto load_chunk = [&](int it, float2 (&x)[8]) {
            const int t = it / KCH, kc = it % KCH;
            if (t != loadTile) {
                loadTile = t;
                const int tv0 = vc0 + t * 64;
                loadCount = min(64, vc0 + vcN - tv0);
                conjMask = 0;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int cl = warp * 8 + c;
                    colBase[c] = 0;
                    if (cl < loadCount) {
                        const ColumnRef ref = column_ref(p, p.inBins, tv0 + cl, gcols, gfirst, S);
                        colBase[c] = ref.base;
                        conjMask |= ref.conj ? (1u << c) : 0u;
                    }
                }
                // Pull the following tile's columns towards L2 meanwhile.
                if (t + 1 < tiles) prefetch_tile(t + 1);
            }
            const int s = kc * kChunkK + lane;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                x[c] = make_float2(0.f, 0.f);
                if (warp * 8 + c < loadCount && s < S) {
                    x[c] = __ldg(p.in + colBase[c] + s);
                    if (conjMask & (1u << c)) x[c].y = -x[c].y;
                }
            }
        };
        float2 next[8];
        load_chunk(0, next);
        for (int it = 0; it < total && !failed; ++it) {
            float2 x[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) x[c] = next[c];
            if (it + 1 < total) load_chunk(it + 1, next);
            const int stage = it % kStages;
            const int round = it / kStages;
            if (round > 0 && !mbar_wait(smem_u32(&st->empty[stage]), (round - 1) & 1, p.error)) {
                failed = true;
                break;
            }
            unsigned char* aHi = sA + stage * kStageBytes;
            unsigned char* aLo = aHi + kTileRows * 128;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int cl = warp * 8 + c;
                const float rh = tf32_rna(x[c].x), ih = tf32_rna(x[c].y);
                const float rl = tf32_rna(x[c].x - rh), il = tf32_rna(x[c].y - ih);
                const uint32_t o0 = sw128_offset(2 * cl, lane >> 2) + 4 * (lane & 3);
                const uint32_t o1 = sw128_offset(2 * cl + 1, lane >> 2) + 4 * (lane & 3);
                *reinterpret_cast<float*>(aHi + o0) = rh;
                *reinterpret_cast<float*>(aLo + o0) = rl;
                *reinterpret_cast<float*>(aHi + o1) = ih;
                *reinterpret_cast<float*>(aLo + o1) = il;
            }
            fence_proxy_async();
            mbar_arrive(smem_u32(&st->full[stage]));
        }
    } else if (warp == kMmaWarp) {
        // --------------------------------------------------------------- MMA
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(NP >> 3) << 17) |
                                   (static_cast<uint32_t>(kTileRows >> 4) << 24);
            int it = 0;
            for (int t = 0; t < tiles && !failed; ++t) {
                for (int kc = 0; kc < KCH; ++kc, ++it) {
                    const int stage = it % kStages;
                    const int acc = it % kAccumulators;
                    const int accRound = it / kAccumulators;
                    if (!mbar_wait(smem_u32(&st->full[stage]), (it / kStages) & 1, p.error) ||
                        (accRound > 0 &&
                         !mbar_wait(smem_u32(&st->accEmpty[acc]), (accRound - 1) & 1, p.error))) {
                        failed = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t aH = smem_u32(sA + stage * kStageBytes);
                    const uint32_t aL = aH + kTileRows * 128;
                    const uint32_t bH = smem_u32(sBhi + kc * NP * 128), bL = smem_u32(sBlo + kc * NP * 128);
                    const uint32_t d = tmem + static_cast<uint32_t>(acc * NP);
                    const int ksteps = min(4, (S - kc * kChunkK + 7) / 8);
                    for (int j = 0; j < ksteps; ++j) {
                        const uint32_t off = j * 32;
                        mma_tf32(d, sw128_desc(aH + off), sw128_desc(bL + off), idesc, j > 0 ? 1u : 0u);
                        mma_tf32(d, sw128_desc(aL + off), sw128_desc(bH + off), idesc, 1u);
                        mma_tf32(d, sw128_desc(aH + off), sw128_desc(bH + off), idesc, 1u);
                    }
                    mma_commit(smem_u32(&st->empty[stage]));
                    mma_commit(smem_u32(&st->accFull[acc]));
                }
            }
            // Every issued MMA has completed once this commit lands.
            mma_commit(smem_u32(&st->done));
            if (!mbar_wait(smem_u32(&st->done), 0, p.error)) failed = true;
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        // Running chunk sums live in a third TMEM region (columns 2*NP ..),
        // read-added-stored eight columns at a time, so only 16 values are
        // live per thread.  The final chunk's sum goes straight to global.
        const int quarter = warp & 3;  // TMEM lanes this warp may access
        const int half = (warp - kMmaWarp - 1) >> 2;
        const int part = lane & 1;
        float* ebuf = reinterpret_cast<float*>(st + 1) + (warp - kMmaWarp - 1) * 16 * kEpiStride;
        const uint32_t laneBase = static_cast<uint32_t>(quarter * 32) << 16;
        const uint32_t sumBase = tmem + laneBase + static_cast<uint32_t>(kAccumulators * NP + half * HALF);
        int it = 0;
        for (int t = 0; t < tiles && !failed; ++t) {
            const int tv0 = vc0 + t * 64;
            const int tcount = min(64, vc0 + vcN - tv0);
            // The four columns this lane stores in the transposed epilogue.
            bool storeValid[4], storeConj[4];
            long long storeColumn[4], storePartner[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int sc = quarter * 16 + 4 * k + (lane >> 3);
                storeValid[k] = sc < tcount;
                const ColumnRef ref =
                    storeValid[k] ? column_ref(p, p.outBins, tv0 + sc, gcols, gfirst, R) : ColumnRef{0, -1, false};
                storeColumn[k] = ref.base;
                storePartner[k] = ref.partner;
                storeConj[k] = ref.conj;
            }
            for (int kc = 0; kc < KCH; ++kc, ++it) {
                const int acc = it % kAccumulators;
                if (!mbar_wait(smem_u32(&st->accFull[acc]), (it / kAccumulators) & 1, p.error)) {
                    failed = true;
                    break;
                }
                tc_fence_after();
                const uint32_t accBase = tmem + laneBase + static_cast<uint32_t>(acc * NP + half * HALF);
                const bool first = kc == 0, last = kc == KCH - 1;
                // Blocks of 8 accumulator columns are handled kG at a time:
                // their TMEM loads are issued together and waited for once.
                constexpr int kBlocks = HALF / 8, kG = 3;
#pragma unroll 1
                for (int b0 = 0; b0 < kBlocks; b0 += kG) {
                    uint32_t a[kG][8], b[kG][8];
#pragma unroll
                    for (int i = 0; i < kG; ++i)
                        if (b0 + i < kBlocks) {
                            tmem_ld_x8(accBase + (b0 + i) * 8, a[i]);
                            if (!first) tmem_ld_x8(sumBase + (b0 + i) * 8, b[i]);
                        }
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < kG; ++i) {
                        if (b0 + i >= kBlocks) break;
                        const int blk = b0 + i;
                        float x8[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            x8[j] = first ? __uint_as_float(a[i][j])
                                          : __uint_as_float(b[i][j]) + __uint_as_float(a[i][j]);
                        if (!last) {
                            uint32_t o[8];
#pragma unroll
                            for (int j = 0; j < 8; ++j) o[j] = __float_as_uint(x8[j]);
                            tmem_st_x8(sumBase + blk * 8, o);
                        } else {
                            // Transpose through this warp's shared buffer so
                            // that each store instruction writes 64 contiguous
                            // bytes (8 complex outputs) of four columns.
#pragma unroll
                            for (int j = 0; j < 8; ++j) ebuf[(lane >> 1) * kEpiStride + 2 * j + part] = x8[j];
                            __syncwarp();
                            const int n = half * HALF + blk * 8 + (lane & 7);
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                const int lc = 4 * k + (lane >> 3);
                                if (storeValid[k] && n < R) {
                                    const float re = ebuf[lc * kEpiStride + 2 * (lane & 7)];
                                    const float im = ebuf[lc * kEpiStride + 2 * (lane & 7) + 1];
                                    p.out[storeColumn[k] + n] = make_float2(re, storeConj[k] ? -im : im);
                                    if (storePartner[k] >= 0)
                                        p.out[storePartner[k] + n] = make_float2(re, storeConj[k] ? im : -im);
                                }
                            }
                            __syncwarp();
                        }
                    }
                }
                if (!last) tmem_wait_st();
                tc_fence_before();
                mbar_arrive(smem_u32(&st->accEmpty[acc]));
            }
        }
    }
    if (failed) atomicExch(p.error, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) tmem_dealloc(tmem, kTmemCols);
}

}  // namespace

size_t tc_gemm_smem_bytes(int R, int S) {
    const int NP = (R + 15) / 16 * 16;
    const int KCH = (S + kChunkK - 1) / kChunkK;
    return 1024 + 2 * static_cast<size_t>(KCH) * NP * 128 + kStages * kStageBytes + sizeof(PipeState) + 16 +
           kEpiBytes;
}

bool tc_gemm_supported(int R, int S) {
    const int NP = (R + 15) / 16 * 16;
    return NP >= 16 && (kAccumulators + 1) * NP <= kTmemCols && tc_gemm_smem_bytes(R, S) <= 227 * 1024;
}

int tc_gemm_unit_tiles() { return 16; }

namespace {
template <int NPH>
cudaError_t launch_np(const TcGemmArgs& args, cudaStream_t stream) {
    const size_t bytes = tc_gemm_smem_bytes(args.R, args.S);
    auto kernel = tc_gemm_pipe_kernel<NPH>;
    const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (err != cudaSuccess) return err;
    kernel<<<args.units, kPipeThreads, bytes, stream>>>(args);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_tc_gemm(const TcGemmArgs& args, cudaStream_t stream) {
    if (args.units <= 0) return cudaSuccess;
    if (!tc_gemm_supported(args.R, args.S) || args.NP != (args.R + 15) / 16 * 16) return cudaErrorInvalidValue;
    switch (args.NP / 16) {
        case 1: return launch_np<1>(args, stream);
        case 2: return launch_np<2>(args, stream);
        case 3: return launch_np<3>(args, stream);
        case 4: return launch_np<4>(args, stream);
        case 5: return launch_np<5>(args, stream);
        case 6: return launch_np<6>(args, stream);
        case 7: return launch_np<7>(args, stream);
        case 8: return launch_np<8>(args, stream);
        case 9: return launch_np<9>(args, stream);
        case 10: return launch_np<10>(args, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace skb
