// Tensor-core (tcgen05, sm_100a) grouped vertical GEMM in split TF32x3.
//
// Problem (see vertical.hpp): for each K^2 group g, out[c][r] = sum_s
// A_g[r][s] in[c][s] over the group's complex columns c.  It is issued as the
// transposed real product
//     D[m][n] = sum_k Aop[m][k] * Bop[n][k]
// with m = (column, re/im part) of the data (M = 128 rows = 64 complex
// columns per tile), n = r (N = R padded to a multiple of 16) and k = s.  Both
// operands are K-major: Bop is the group matrix in its row-major [r][s]
// layout, Aop is the data row in[c][0..S).
//
// Split precision, two forms (KIND):
// * TF32x3: x = hi + lo with hi = rna_tf32(x), lo = rna_tf32(x - hi);
//   D = Ahi*Blo + Alo*Bhi + Ahi*Bhi (kind::tf32, K = 8 per MMA).  The dropped
//   lo*lo term is ~2^-22 relative.
// * BF16x3: x = h + m + l, three round-to-nearest BF16 pieces (8 significant
//   bits each, so h + m + l carries all 24 bits of x); D = Al*Bh + Ah*Bl +
//   Am*Bm + Am*Bh + Ah*Bm + Ah*Bh (kind::f16 with BF16 operands, K = 16 per
//   MMA; the dropped m*l, l*m, l*l terms are <= 2^-24 relative).
// Both accumulate in FP32 in tensor memory, one accumulator per 32-wide K
// chunk, chunk sums added in FP32 registers.
//
// Work unit: one group and a run of up to 16 M-tiles of its (member,
// column) list; each CTA (one per SM) walks its share of the units.  The
// group matrix, split and swizzled once at plan time into an operand image
// (tc_gemm_build_images), is bulk-copied into shared memory and stays
// resident for the unit; data chunks of 32 k stream through a three-stage
// ring filled by producer warps while one MMA lane and the epilogue warps
// work on earlier chunks (warp specialisation below).  Operands use the
// canonical K-major SWIZZLE_128B layout: 8-row atoms of 8 x 128 bytes,
// 16-byte chunk q of row n stored at chunk (q xor n%8).  One elected thread
// issues the MMAs and commits them to the stage's mbarrier; every wait is
// bounded and reports through `error` instead of hanging.

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "vertical.hpp"

namespace skb {
namespace {

constexpr int kTileRows = 128;    // M
constexpr int kChunkK = 32;       // tf32 elements per 128-byte row
constexpr int kTmemCols = 512;  // two chunk accumulators of NP columns each (power of two)
constexpr int kStageBytes = 2 * kTileRows * 128;  // hi + lo
constexpr long long kWaitLimit = 1LL << 22;
constexpr long long kTestWaitLimit = 1LL << 14;  // the expired-wait test's wait (expireWaitForTest)

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
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const int* error,
                                          long long limit = kWaitLimit) {
    for (long long i = 0; i < limit; ++i) {
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

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d),
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

// Operand forms of the kernel.
constexpr int kKindTf32x3 = 0;
constexpr int kKindBf16x3 = 1;

struct Split4 {
    float4 hi, lo;
};

// Four values as three BF16 pieces each, packed four to 8 bytes (value e at
// bytes 2e, 2e+1): h = rn(x), m = rn(x - h), l = rn(x - h - m).  Both
// differences are exact in FP32 (each piece holds the leading 8 bits of what
// is left), so h + m + l equals x to within 2^-24 |x|.
struct Split3 {
    uint2 h, m, l;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);  // a in the low half
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ Split3 split3(float a, float b, float c, float d) {
    const float x[4] = {a, b, c, d};
    float h[4], m[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        h[e] = __bfloat162float(__float2bfloat16_rn(x[e]));
        const float r = x[e] - h[e];
        m[e] = __bfloat162float(__float2bfloat16_rn(r));
        l[e] = r - m[e];
    }
    Split3 s;
    s.h = make_uint2(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]));
    s.m = make_uint2(pack_bf16x2(m[0], m[1]), pack_bf16x2(m[2], m[3]));
    s.l = make_uint2(pack_bf16x2(l[0], l[1]), pack_bf16x2(l[2], l[3]));
    return s;
}

// BF16x3 operand rows: a 128-byte row of the first region holds the h piece
// of the chunk's 32 k in bytes 0-63 and the m piece in bytes 64-127; the same
// row of the second region holds the l piece in bytes 0-63 (64-127 unused).
// Piece q (8 bytes, 4 values) of a half-row sits in 16-byte chunk q / 2 of that
// half, at byte 8 (q % 2); chunks are swizzled like every SWIZZLE_128B row.
__device__ __forceinline__ uint32_t bf16_piece_offset(int row, int half, int q) {
    return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + (((4 * half + (q >> 1)) ^ (row & 7)) << 4) +
                                 (q & 1) * 8);
}

__device__ __forceinline__ Split4 split4(float a, float b, float c, float d) {
    Split4 s;
    s.hi = make_float4(tf32_rna(a), tf32_rna(b), tf32_rna(c), tf32_rna(d));
    s.lo = make_float4(tf32_rna(a - s.hi.x), tf32_rna(b - s.hi.y), tf32_rna(c - s.hi.z), tf32_rna(d - s.hi.w));
    return s;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bulk (non-tensor, single-destination) copy global -> this CTA's shared
// memory, completing on `bar` by transaction bytes.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// cp.async of one complex value (8 bytes); srcBytes = 0 writes zeros.
__device__ __forceinline__ void cp_async_value(uint32_t dst, const void* src, int srcBytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Warp roles of the pipelined kernel, one role per warpgroup (4 warps) so
// that each role can set its own register count: warpgroups 0-1 are the
// producers, warpgroup 2 holds the MMA warp (its other three warps have no
// work), warpgroups 3-5 are the epilogue.
constexpr int kProducerWarps = 8;
constexpr int kMmaWarp = kProducerWarps;
constexpr int kEpilogueFirst = kMmaWarp + 4;
constexpr int kEpilogueGroups = 3;  // epilogue warps per TMEM lane quarter
constexpr int kEpilogueWarps = 4 * kEpilogueGroups;
constexpr int kPipeThreads = (kEpilogueFirst + kEpilogueWarps) * 32;
// Registers per thread: the launch gives every thread kLaunchRegs (65,536
// per SM over 768 threads, in steps of 8); the MMA warpgroup hands most of
// its share to the epilogue, which keeps a tile's running sums in registers.
constexpr int kLaunchRegs = 65536 / kPipeThreads / 8 * 8;
constexpr int kProducerRegs = 56;
constexpr int kMmaGroupRegs = 32;
constexpr int kEpilogueRegs = 112;
static_assert(kProducerWarps * 32 * kProducerRegs + 128 * kMmaGroupRegs + kEpilogueWarps * 32 * kEpilogueRegs <=
                  kPipeThreads * kLaunchRegs,
              "register split exceeds the launch's registers");
constexpr int kStages = 3;
constexpr int kAccumulators = 2;
constexpr int kAhead = 2;               // data chunks each producer thread has in flight
constexpr uint32_t kBulkPiece = 32768;  // bytes per bulk copy of a group image

struct PipeState {
    uint64_t full[kStages], empty[kStages], accFull[kAccumulators], accEmpty[kAccumulators], done, unitDone, bFull;
    uint64_t never;  // no thread or copy ever arrives on it (expired-wait test)
    long long colBase[kProducerWarps][8];  // each producer warp's 8 input columns of the current tile
    uint32_t tmem;
};

// Bytes of one group's operand image: hi then lo, each KCH chunks of NP
// swizzled 128-byte rows.
__host__ __device__ constexpr long long image_bytes(int NP, int KCH) { return 2LL * KCH * NP * 128; }

// k (within a 32-wide chunk) held by element e of 16-byte piece q of an
// operand row: pieces pair k = 2q, 2q+1 with k = 2q+16, 2q+17 so that the
// producer warps fill them with conflict-free 16-byte shared-memory accesses.
// The MMA's k-step j (pieces 2j, 2j+1) thus covers k = 4j..4j+3 and
// 4j+16..4j+19.
__host__ __device__ constexpr int kperm(int q, int e) { return 2 * q + (e & 1) + 16 * (e >> 1); }

// Group matrices [g][R][S] -> their shared-memory operand images: TF32 hi/lo
// split, zero-padded to NP x KCH*32, K-major SWIZZLE_128B.  One thread per
// (group, chunk, row, 16-byte piece).
__global__ void tc_gemm_image_kernel(const float* __restrict__ natural, int groups, int R, int S, int NP, int KCH,
                                     int kind, unsigned char* __restrict__ images) {
    const long long total = static_cast<long long>(groups) * KCH * NP * 8;
    const long long bytes = image_bytes(NP, KCH);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int q = static_cast<int>(i & 7);
        long long rest = i >> 3;
        const int n = static_cast<int>(rest % NP);
        rest /= NP;
        const int kc = static_cast<int>(rest % KCH);
        const long long g = rest / KCH;
        const float* m = natural + g * R * S;
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int s = kc * kChunkK + kperm(q, j);
            v[j] = (n < R && s < S) ? m[static_cast<long long>(n) * S + s] : 0.0f;
        }
        unsigned char* img = images + g * bytes;
        if (kind == kKindBf16x3) {
            // Piece q of each half-row: the same k values (kperm(q, e)) as the
            // producer warps put in piece q of a data row.
            const Split3 sp = split3(v[0], v[1], v[2], v[3]);
            const uint32_t base = kc * NP * 128;
            *reinterpret_cast<uint2*>(img + base + bf16_piece_offset(n, 0, q)) = sp.h;
            *reinterpret_cast<uint2*>(img + base + bf16_piece_offset(n, 1, q)) = sp.m;
            *reinterpret_cast<uint2*>(img + bytes / 2 + base + bf16_piece_offset(n, 0, q)) = sp.l;
            // The unused second half of the l row stays zero.
            *reinterpret_cast<uint2*>(img + bytes / 2 + base + bf16_piece_offset(n, 1, q)) = make_uint2(0u, 0u);
            continue;
        }
        const Split4 sp = split4(v[0], v[1], v[2], v[3]);
        const uint32_t off = kc * NP * 128 + sw128_offset(n, q);
        *reinterpret_cast<float4*>(img + off) = sp.hi;
        *reinterpret_cast<float4*>(img + bytes / 2 + off) = sp.lo;
    }
}

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
    const int sub = c - mode * bb.fields;
    const int field = bb.fieldMap != nullptr ? __ldg(bb.fieldMap + sub) : sub;
    const long long memberStride =
        bb.memberStride != 0 ? bb.memberStride : static_cast<long long>(bb.fields) * bb.zStride;
    const long long off = member * memberStride + static_cast<long long>(field) * bb.zStride;
    const long long partner = bb.partner != nullptr ? __ldg(bb.partner + mode) : -1;
    const bool conj = bb.conj != nullptr && __ldg(bb.conj + mode) != 0;
    return {__ldg(bb.cell + mode) + off, partner >= 0 ? partner + off : -1, conj};
}

struct Unit {
    int g, vc0, vcN, gcols, tiles;
    long long gfirst;
};

// The units this CTA walks: [begin, end) with stride `step`.
struct Walk {
    int begin, end, step;
};
__device__ __forceinline__ Walk unit_walk(const TcGemmArgs& p) {
    if (p.ctaFirst != nullptr)
        return {__ldg(p.ctaFirst + blockIdx.x), __ldg(p.ctaFirst + blockIdx.x + 1), 1};
    return {static_cast<int>(blockIdx.x), p.units, static_cast<int>(gridDim.x)};
}
__device__ __forceinline__ Unit unit_at(const TcGemmArgs& p, int u) {
    Unit U;
    U.g = __ldg(p.unitGroup + u);
    U.vc0 = __ldg(p.unitColumn + u);
    U.vcN = __ldg(p.unitCount + u);
    U.gcols = __ldg(p.groupColumns + U.g);
    U.gfirst = __ldg(p.groupFirst + U.g);
    U.tiles = (U.vcN + 63) / 64;
    return U;
}

// Warp-specialised, persistent split-TF32x3 grouped GEMM.  Each CTA (one per
// SM) walks its range of work units (unit_walk); TMEM, the
// barriers and the stage ring live across units, and every role counts chunks
// globally so the barrier phases continue from unit to unit.
//   producer warps 0-7: data chunks (64 columns x 32 k) stream through a
//       3-deep ring of A stages.  Each thread copies its values of a chunk
//       with cp.async into the stage's lo half (raw complex FP32, two chunks
//       in flight), then the warp rewrites its own 2 KB of the stage in place
//       as swizzled TF32 hi/lo rows and arrives full[stage].
//   MMA warp 8 (one lane): per unit, once the previous unit's MMAs have
//       completed, bulk-copies the group's prepared operand image (hi/lo,
//       all K chunks) into shared memory and prefetches the next unit's into
//       L2; per chunk, 3 MMAs per k-step into one of two ping-pong TMEM chunk
//       accumulators; commits empty[stage] and accFull.
//   warps 9-11: no work (they only lend their registers to the epilogue).
//   epilogue warps 12-23: read each chunk accumulator (tcgen05.ld), release
//       it (accEmpty) and add it into an FP32 running sum held in registers;
//       after the tile's last chunk write the tile's outputs: lane pairs
//       (the re and im rows of one column) swap halves with a shuffle so each
//       store instruction writes 16 contiguous bytes of 16 columns.
// NPH = NP/16.
template <int NPH, int KIND>
__global__ void __launch_bounds__(kPipeThreads, 1) tc_gemm_pipe_kernel(TcGemmArgs p) {
    constexpr int NP = NPH * 16;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int KCH = p.KCH, R = p.R, S = p.S;
    const long long imageBytes = image_bytes(NP, KCH);
    unsigned char* sBhi = base;
    unsigned char* sBlo = sBhi + imageBytes / 2;
    unsigned char* sA = sBhi + imageBytes;
    PipeState* st = reinterpret_cast<PipeState*>(sA + kStages * kStageBytes);

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
        mbar_init(smem_u32(&st->unitDone), 1);
        mbar_init(smem_u32(&st->bFull), 1);
        mbar_init(smem_u32(&st->never), 1);
        fence_barrier_init();
    }
    if (warp == kMmaWarp) {
        tmem_alloc(smem_u32(&st->tmem), kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = st->tmem;
    bool failed = false;
    // A bounded wait that expired: stop this role and make the others stop too.
    auto fail = [&] {
        failed = true;
        atomicExch(p.error, 1);
    };

    if (warp < kProducerWarps) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kProducerRegs));
        // ---------------------------------------------------------- producer
        // Issue cursor: unit iu, tile itT, chunk itKc of the tile.
        const Walk W = unit_walk(p);
        int iu = W.begin;
        Unit IU{};
        if (iu < W.end) IU = unit_at(p, iu);
        int itT = 0, itKc = 0, curTile = -1, tileCount = 0;
        long long* colBase = st->colBase[warp];
        unsigned tileMask = 0;  // bit c: column 8*warp+c of the tile is stored conjugated
        int issued = 0, converted = 0, pending = 0;
        unsigned fifo = 0;  // conjugation masks of the chunks in flight, oldest in the low byte
        // L2 prefetch of column 8*warp + lane (lanes 0-7) of tile t of unit V
        // (compact operand only: bin-array columns would first need their
        // cells, a dependent load this warp would wait for).
        auto prefetch_tile = [&](const Unit& V, int t) {
            if (p.inBins.cell != nullptr || lane >= 8) return;
            const int tv0 = V.vc0 + t * 64;
            const int cl = warp * 8 + lane;
            if (cl >= min(64, V.vc0 + V.vcN - tv0)) return;
            const uintptr_t first = reinterpret_cast<uintptr_t>(p.in + column_ref(p, p.inBins, tv0 + cl, V.gcols, V.gfirst, S).base);
            const uintptr_t a = (first + 15) & ~uintptr_t(15), b = (first + S * 8) & ~uintptr_t(15);
            if (b > a) bulk_prefetch_l2(reinterpret_cast<const void*>(a), static_cast<uint32_t>(b - a));
        };
        // Copies of the next chunk of the stream into its stage; false at the
        // end of the stream or on an expired wait.
        auto issue_next = [&]() -> bool {
            if (iu >= W.end || failed) return false;
            const int stage = issued % kStages;
            const int round = issued / kStages;
            if (round > 0 && !mbar_wait(smem_u32(&st->empty[stage]), (round - 1) & 1, p.error)) {
                fail();
                return false;
            }
            if (itT != curTile) {
                // Lanes 0-7 look up one column each; the warp shares them.
                curTile = itT;
                const int tv0 = IU.vc0 + itT * 64;
                tileCount = min(64, IU.vc0 + IU.vcN - tv0);
                const int cl = warp * 8 + lane;
                ColumnRef mine{0, -1, false};
                if (lane < 8 && cl < tileCount) mine = column_ref(p, p.inBins, tv0 + cl, IU.gcols, IU.gfirst, S);
                tileMask = __ballot_sync(0xFFFFFFFFu, lane < 8 && mine.conj) & 0xFFu;
                if (lane < 8) colBase[lane] = mine.base;
                __syncwarp();
                if (itT + 1 < IU.tiles) {
                    prefetch_tile(IU, itT + 1);
                } else if (iu + W.step < W.end) {
                    prefetch_tile(unit_at(p, iu + W.step), 0);
                }
            }
            const uint32_t raw = smem_u32(sA + stage * kStageBytes + kTileRows * 128) + lane * 8;
            const int s = itKc * kChunkK + lane;
#pragma unroll
            for (int cc = 0; cc < 8; ++cc) {
                const bool ok = warp * 8 + cc < tileCount && s < S;
                cp_async_value(raw + (warp * 8 + cc) * 256, ok ? p.in + colBase[cc] + s : p.in, ok ? 8 : 0);
            }
            cp_async_commit();
            fifo |= tileMask << (8 * pending);
            ++pending;
            ++issued;
            if (++itKc == KCH) {
                itKc = 0;
                if (++itT == IU.tiles) {
                    itT = 0;
                    curTile = -1;
                    iu += W.step;
                    if (iu < W.end) IU = unit_at(p, iu);
                }
            }
            return true;
        };
        if (iu < W.end) prefetch_tile(IU, 0);
        for (int k = 0; k < kAhead; ++k)
            if (!issue_next()) break;
        while (pending > 0 && !failed) {
            // The oldest chunk's copies have landed once at most pending-1
            // younger groups are outstanding.
            if (pending > 1)
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            else
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            const int stage = converted % kStages;
            unsigned char* aHi = sA + stage * kStageBytes;
            unsigned char* aLo = aHi + kTileRows * 128;
            const unsigned m = fifo & 0xFFu;
            fifo >>= 8;
            --pending;
            ++converted;
            // This warp's 8 columns sit as raw complex values (column c at
            // byte 256c, value k at 8k) in bytes [2048 warp, +2048) of the lo
            // half, which are also the swizzled rows 16 warp .. +15 they
            // become, so the warp rewrites them in place once all its reads
            // are done.  In pass j a lane takes column 8 warp + 4j + lane/8
            // and the values k = 2q, 2q+1, 2q+16, 2q+17 (q = lane % 8): two
            // 16-byte reads 128 bytes apart, so each 8-lane phase reads 128
            // contiguous bytes, then four 16-byte writes of piece q of the
            // column's re and im rows (hi and lo).  Within each 16-byte piece
            // the k order is the operand order (kperm), shared with the
            // group images, so the MMA sums the same products.
            const int q = lane & 7;
            float4 v[2][2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const unsigned char* src = aLo + (warp * 8 + 4 * j + (lane >> 3)) * 256 + q * 16;
                v[j][0] = *reinterpret_cast<const float4*>(src);
                v[j][1] = *reinterpret_cast<const float4*>(src + 128);
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int cc = 4 * j + (lane >> 3);
                const int cl = warp * 8 + cc;
                const float sgn = (m & (1u << cc)) ? -1.0f : 1.0f;
                if constexpr (KIND == kKindBf16x3) {
                    // Same values and k order as the TF32 pieces; three BF16
                    // pieces of 8 bytes each per row (bf16_piece_offset).
                    const Split3 re = split3(v[j][0].x, v[j][0].z, v[j][1].x, v[j][1].z);
                    const Split3 im = split3(sgn * v[j][0].y, sgn * v[j][0].w, sgn * v[j][1].y, sgn * v[j][1].w);
                    *reinterpret_cast<uint2*>(aHi + bf16_piece_offset(2 * cl, 0, q)) = re.h;
                    *reinterpret_cast<uint2*>(aHi + bf16_piece_offset(2 * cl, 1, q)) = re.m;
                    *reinterpret_cast<uint2*>(aLo + bf16_piece_offset(2 * cl, 0, q)) = re.l;
                    *reinterpret_cast<uint2*>(aHi + bf16_piece_offset(2 * cl + 1, 0, q)) = im.h;
                    *reinterpret_cast<uint2*>(aHi + bf16_piece_offset(2 * cl + 1, 1, q)) = im.m;
                    *reinterpret_cast<uint2*>(aLo + bf16_piece_offset(2 * cl + 1, 0, q)) = im.l;
                } else {
                    const Split4 re = split4(v[j][0].x, v[j][0].z, v[j][1].x, v[j][1].z);
                    const Split4 im = split4(sgn * v[j][0].y, sgn * v[j][0].w, sgn * v[j][1].y, sgn * v[j][1].w);
                    const uint32_t o0 = sw128_offset(2 * cl, q), o1 = sw128_offset(2 * cl + 1, q);
                    *reinterpret_cast<float4*>(aHi + o0) = re.hi;
                    *reinterpret_cast<float4*>(aLo + o0) = re.lo;
                    *reinterpret_cast<float4*>(aHi + o1) = im.hi;
                    *reinterpret_cast<float4*>(aLo + o1) = im.lo;
                }
            }
            fence_proxy_async();
            mbar_arrive(smem_u32(&st->full[stage]));
            issue_next();
        }
        // No copy may still be writing this CTA's shared memory at exit.
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    } else if (warp < kEpilogueFirst) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kMmaGroupRegs));
        // --------------------------------------------------------------- MMA
        if (warp == kMmaWarp && lane == 0) {
            // Instruction descriptor: F32 accumulator, A and B TF32 (2) or
            // BF16 (1), both K-major, N = NP, M = 128.
            constexpr uint32_t kOperandFormat = KIND == kKindBf16x3 ? 1u : 2u;
            const uint32_t idesc = (1u << 4) | (kOperandFormat << 7) | (kOperandFormat << 10) |
                                   (static_cast<uint32_t>(NP >> 3) << 17) |
                                   (static_cast<uint32_t>(kTileRows >> 4) << 24);
            int it = 0, loads = 0, group = -1;
            // Expired-wait test: before this lane has issued any copy or MMA,
            // a bounded wait on a barrier nothing arrives on runs out and takes
            // the same path as any expired wait (error word, every role stops,
            // copies drained, TMEM freed, SKB_ERR_RUNTIME on the host).
            if (p.expireWaitForTest != 0 && !mbar_wait(smem_u32(&st->never), 0, p.error, kTestWaitLimit)) fail();
            const Walk W = unit_walk(p);
            for (int u = W.begin; u < W.end && !failed; u += W.step) {
                const Unit U = unit_at(p, u);
                if (U.g != group) {
                    // The resident image may be replaced once every MMA that
                    // reads it has completed.
                    if (loads > 0) {
                        mma_commit(smem_u32(&st->unitDone));
                        if (!mbar_wait(smem_u32(&st->unitDone), (loads - 1) & 1, p.error)) {
                            fail();
                            break;
                        }
                    }
                    const unsigned char* img = p.B + static_cast<long long>(U.g) * p.imageStride;
                    mbar_expect_tx(smem_u32(&st->bFull), static_cast<uint32_t>(imageBytes));
                    for (uint32_t o = 0; o < imageBytes; o += kBulkPiece)
                        bulk_load(smem_u32(sBhi + o), img + o, min(kBulkPiece, static_cast<uint32_t>(imageBytes - o)),
                                  smem_u32(&st->bFull));
                    // L2 prefetch of the next group's image this CTA will load
                    // (a few units ahead at most).
                    for (int v = u + W.step, seen = 0; v < W.end && seen < 32; v += W.step, ++seen) {
                        const int gn = __ldg(p.unitGroup + v);
                        if (gn != U.g) {
                            bulk_prefetch_l2(p.B + static_cast<long long>(gn) * p.imageStride,
                                             static_cast<uint32_t>(imageBytes));
                            break;
                        }
                    }
                    if (!mbar_wait(smem_u32(&st->bFull), loads & 1, p.error)) {
                        fail();
                        break;
                    }
                    ++loads;
                    group = U.g;
                }
                for (int t = 0; t < U.tiles && !failed; ++t) {
                    for (int kc = 0; kc < KCH; ++kc, ++it) {
                        const int stage = it % kStages;
                        const int acc = it % kAccumulators;
                        const int accRound = it / kAccumulators;
                        if (!mbar_wait(smem_u32(&st->full[stage]), (it / kStages) & 1, p.error) ||
                            (accRound > 0 &&
                             !mbar_wait(smem_u32(&st->accEmpty[acc]), (accRound - 1) & 1, p.error))) {
                            fail();
                            break;
                        }
                        tc_fence_after();
                        const uint32_t aH = smem_u32(sA + stage * kStageBytes);
                        const uint32_t aL = aH + kTileRows * 128;
                        const uint32_t bH = smem_u32(sBhi + kc * NP * 128), bL = smem_u32(sBlo + kc * NP * 128);
                        const uint32_t d = tmem + static_cast<uint32_t>(acc * NP);
                        // k-steps holding any k < S (see kperm).
                        const int left = S - kc * kChunkK;
                        if constexpr (KIND == kKindBf16x3) {
                            // k-step j (K = 16) reads pieces 4j..4j+3 of each
                            // half-row: k = 8j..8j+7 and 16+8j..16+8j+7.
                            const int ksteps = left > 8 ? 2 : 1;
                            for (int j = 0; j < ksteps; ++j) {
                                const uint32_t oh = j * 32, om = 64 + j * 32;
                                mma_bf16(d, sw128_desc(aL + oh), sw128_desc(bH + oh), idesc, j > 0 ? 1u : 0u);
                                mma_bf16(d, sw128_desc(aH + oh), sw128_desc(bL + oh), idesc, 1u);
                                mma_bf16(d, sw128_desc(aH + om), sw128_desc(bH + om), idesc, 1u);
                                mma_bf16(d, sw128_desc(aH + om), sw128_desc(bH + oh), idesc, 1u);
                                mma_bf16(d, sw128_desc(aH + oh), sw128_desc(bH + om), idesc, 1u);
                                mma_bf16(d, sw128_desc(aH + oh), sw128_desc(bH + oh), idesc, 1u);
                            }
                        } else {
                            const int ksteps = left >= 16 ? 4 : (left + 3) / 4;
                            for (int j = 0; j < ksteps; ++j) {
                                const uint32_t off = j * 32;
                                mma_tf32(d, sw128_desc(aH + off), sw128_desc(bL + off), idesc, j > 0 ? 1u : 0u);
                                mma_tf32(d, sw128_desc(aL + off), sw128_desc(bH + off), idesc, 1u);
                                mma_tf32(d, sw128_desc(aH + off), sw128_desc(bH + off), idesc, 1u);
                            }
                        }
                        mma_commit(smem_u32(&st->empty[stage]));
                        mma_commit(smem_u32(&st->accFull[acc]));
                    }
                }
            }
            // Every issued MMA has completed once this commit lands.
            mma_commit(smem_u32(&st->done));
            if (!mbar_wait(smem_u32(&st->done), 0, p.error)) fail();
        }
        __syncwarp();
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kEpilogueRegs));
        // ---------------------------------------------------------- epilogue
        // Twelve warps, three per TMEM lane quarter: warp (quarter, group)
        // owns the 8-column accumulator blocks [group * GB, group * GB + GB)
        // of its 32 TMEM lanes.  The tile's chunk accumulators are added, in
        // chunk order and in FP32, into a running sum held in registers (no
        // TMEM round trip per chunk); each accumulator is released as soon as
        // it has been read, and after the tile's last chunk the sum goes to
        // global memory.  TMEM lane 32*quarter + lane is tile row
        // 2*column + part: this lane holds the real (part 0) or imaginary
        // (part 1) row of column 16*quarter + lane/2.
        constexpr int NB = NP / 8;
        constexpr int GB = (NB + kEpilogueGroups - 1) / kEpilogueGroups;
        // Blocks whose TMEM loads are issued before one wait (fewer at the
        // widest tiles, where the sums leave no room for three).
        constexpr int kG = GB <= 6 ? 3 : 1;
        const int quarter = warp & 3;  // TMEM lanes this warp may access
        const int group = (warp - kEpilogueFirst) >> 2;
        const int blk0 = group * GB;
        const int nblk = max(0, min(NB, blk0 + GB) - blk0);
        const int part = lane & 1;
        const int cl = quarter * 16 + (lane >> 1);
        const uint32_t laneBase = static_cast<uint32_t>(quarter * 32) << 16;
        float sum[GB][8];
        int it = 0;
        const Walk W = unit_walk(p);
        for (int u = W.begin; u < W.end && !failed; u += W.step) {
            const Unit U = unit_at(p, u);
            for (int t = 0; t < U.tiles && !failed; ++t) {
                for (int kc = 0; kc < KCH; ++kc, ++it) {
                    const int acc = it % kAccumulators;
                    if (!mbar_wait(smem_u32(&st->accFull[acc]), (it / kAccumulators) & 1, p.error)) {
                        fail();
                        break;
                    }
                    tc_fence_after();
                    const uint32_t accBase = tmem + laneBase + static_cast<uint32_t>(acc * NP + blk0 * 8);
                    const bool first = kc == 0;
#pragma unroll
                    for (int b0 = 0; b0 < GB; b0 += kG) {
                        uint32_t a[kG][8];
#pragma unroll
                        for (int i = 0; i < kG; ++i)
                            if (b0 + i < GB && b0 + i < nblk) tmem_ld_x8(accBase + (b0 + i) * 8, a[i]);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < kG; ++i) {
                            if (b0 + i >= GB) break;
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                sum[b0 + i][j] = first ? __uint_as_float(a[i][j]) : sum[b0 + i][j] + __uint_as_float(a[i][j]);
                        }
                    }
                    // The accumulator may be overwritten once all its loads have completed.
                    tc_fence_before();
                    mbar_arrive(smem_u32(&st->accEmpty[acc]));
                    if (kc != KCH - 1) continue;
                    // The output column is looked up only now, so that no
                    // register holds it while the chunks are summed.
                    const int tv0 = U.vc0 + t * 64;
                    const bool valid = cl < min(64, U.vc0 + U.vcN - tv0);
                    const ColumnRef ref =
                        valid ? column_ref(p, p.outBins, tv0 + cl, U.gcols, U.gfirst, R) : ColumnRef{0, -1, false};
                    const float sg = ref.conj ? -1.0f : 1.0f;
                    // 16-byte stores need even element offsets (true for bin cells).
                    const bool wide = ((ref.base | (ref.partner < 0 ? 0 : ref.partner)) & 1) == 0;
#pragma unroll
                    for (int i = 0; i < GB; ++i) {
                        if (i >= nblk) break;
                        const float* x8 = sum[i];
                        // Rows n0 .. n0+7 of this column.  The even lane stores
                        // outputs n0+{0,1} and n0+{4,5}, the odd lane n0+{2,3}
                        // and n0+{6,7}, after trading the other part with its
                        // partner, so each store instruction fills whole
                        // 32-byte sectors of 16 columns.
                        const int n0 = (blk0 + i) * 8;
                        float o[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int e = (k & 1) + 4 * (k >> 1);
                            o[k] = __shfl_xor_sync(0xFFFFFFFFu, part ? x8[e] : x8[e + 2], 1);
                        }
                        if (!valid) continue;
#pragma unroll
                        for (int h2 = 0; h2 < 2; ++h2) {
                            const int e = 4 * h2;
                            const int n = n0 + e + 2 * part;
                            const float re0 = part ? o[2 * h2] : x8[e];
                            const float im0 = sg * (part ? x8[e + 2] : o[2 * h2]);
                            const float re1 = part ? o[2 * h2 + 1] : x8[e + 1];
                            const float im1 = sg * (part ? x8[e + 3] : o[2 * h2 + 1]);
                            if (wide && n + 1 < R) {
                                *reinterpret_cast<float4*>(p.out + ref.base + n) = make_float4(re0, im0, re1, im1);
                                if (ref.partner >= 0)
                                    *reinterpret_cast<float4*>(p.out + ref.partner + n) =
                                        make_float4(re0, -im0, re1, -im1);
                            } else {
                                if (n < R) {
                                    p.out[ref.base + n] = make_float2(re0, im0);
                                    if (ref.partner >= 0) p.out[ref.partner + n] = make_float2(re0, -im0);
                                }
                                if (n + 1 < R) {
                                    p.out[ref.base + n + 1] = make_float2(re1, im1);
                                    if (ref.partner >= 0) p.out[ref.partner + n + 1] = make_float2(re1, -im1);
                                }
                            }
                        }
                    }
                }
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
    return 1024 + static_cast<size_t>(image_bytes(NP, KCH)) + kStages * kStageBytes + sizeof(PipeState) + 16;
}

bool tc_gemm_supported(int R, int S) {
    const int NP = (R + 15) / 16 * 16;
    return NP >= 16 && NP <= 160 && kAccumulators * NP <= kTmemCols && tc_gemm_smem_bytes(R, S) <= 227 * 1024;
}

size_t tc_gemm_image_bytes(int R, int S) {
    return static_cast<size_t>(image_bytes((R + 15) / 16 * 16, (S + kChunkK - 1) / kChunkK));
}

cudaError_t tc_gemm_build_images(const float* natural, int groups, int R, int S, int kind, void* images,
                                 cudaStream_t stream) {
    if (groups <= 0) return cudaSuccess;
    const int NP = (R + 15) / 16 * 16;
    const int KCH = (S + kChunkK - 1) / kChunkK;
    const long long items = static_cast<long long>(groups) * KCH * NP * 8;
    const int blocks = static_cast<int>(std::min<long long>((items + 255) / 256, 148LL * 16));
    tc_gemm_image_kernel<<<blocks, 256, 0, stream>>>(natural, groups, R, S, NP, KCH, kind,
                                                     static_cast<unsigned char*>(images));
    return cudaGetLastError();
}

int tc_gemm_unit_tiles() { return 16; }

namespace {
template <int NPH>
cudaError_t launch_np(const TcGemmArgs& args, cudaStream_t stream) {
    // At least half an SM's shared memory, so that two CTAs (each holding
    // all 512 TMEM columns) never share an SM.
    const size_t bytes = std::max<size_t>(tc_gemm_smem_bytes(args.R, args.S), 116 * 1024);
    auto kernel = args.kind == kKindBf16x3 ? tc_gemm_pipe_kernel<NPH, kKindBf16x3>
                                           : tc_gemm_pipe_kernel<NPH, kKindTf32x3>;
    // The warpgroups' setmaxnreg split assumes the kernel was built with
    // exactly kLaunchRegs registers per thread; with fewer, the epilogue's
    // increase could never be granted, so such a build is refused.
    static int launchRegs[2] = {0, 0};
    int& regs = launchRegs[args.kind == kKindBf16x3 ? 1 : 0];
    if (regs == 0) {
        cudaFuncAttributes attr{};
        const cudaError_t aerr = cudaFuncGetAttributes(&attr, kernel);
        if (aerr != cudaSuccess) return aerr;
        regs = attr.numRegs;
    }
    if (regs != kLaunchRegs) return cudaErrorInvalidDeviceFunction;
    const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (err != cudaSuccess) return err;
    // Persistent: one CTA per SM (or per unit, if fewer).
    static int smCount[64] = {};
    int device = 0;
    cudaGetDevice(&device);
    if (device >= 0 && device < 64 && smCount[device] == 0)
        cudaDeviceGetAttribute(&smCount[device], cudaDevAttrMultiProcessorCount, device);
    const int sms = (device >= 0 && device < 64 && smCount[device] > 0) ? smCount[device] : 148;
    const int grid = args.ctaFirst != nullptr ? args.ctas : std::min(args.units, sms);
    kernel<<<grid, kPipeThreads, bytes, stream>>>(args);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_tc_gemm(const TcGemmArgs& args, cudaStream_t stream) {
    if (args.units <= 0) return cudaSuccess;
    if (args.ctaFirst != nullptr && args.ctas <= 0) return cudaErrorInvalidValue;
    if (args.kind != kKindTf32x3 && args.kind != kKindBf16x3) return cudaErrorInvalidValue;
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
