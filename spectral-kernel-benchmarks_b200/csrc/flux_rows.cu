// Fused row stage of the split-precision flux (FP32).
//
// One CTA owns one row y of B consecutive z-planes of one ensemble member and
// does, entirely on chip, what the staged path spreads over three kernels and
// seven real volumes (benchmark.cpp:4405-4424 order):
//   U,V,W rows      <- c2r of the column-transformed bins of input slots 0..2,
//                      kept in registers;
//   for each target t:
//     q_t,x/y/z rows <- c2r of slots 3+3t .. 5+3t;
//     target row     = -scale*(u*q_x + v*q_y + w*q_z)   (pointwise_advection.cpp:143-147)
//     target bins    <- r2c of the target row, kx < keep.
// The c2r / r2c are the same half-length complex FFT formulation as the
// staged row kernels (horizontal.cu), so both paths share their numerics.
// Each warp owns one z-plane and transforms it with warp-synchronous passes
// (warp_fft; for 512-point rows warp_fft_rr, whose first and last passes work
// in registers); every lane keeps the same Nx/64 x-pairs of its plane across
// all transforms, which is what lets U,V,W and the product stay in registers.
// The 3+3T slots are consumed in order, so the bins of slot f+1 are copied
// into a second shared stage with cp.async while slot f is transformed; the
// only CTA-wide barriers are one per slot and one per target.
// Each stage row holds kx = 0..M and is zero beyond keep (written once, never
// copied over), so the c2r pre-processing reads bins k and M-k without range
// tests; the r2c twiddles and the 512-point FFT's lane-ordered twiddle table
// are copied into shared memory once per CTA.

#include "flux_rows.hpp"

#include "async_copy.cuh"
#include "fft_device.cuh"
#include "tensor_map.hpp"

namespace skb {
namespace {

// Per-warp padded sequence region (pad16 of the largest index, plus slack).
template <int M>
constexpr int region() {
    return M + M / 16 + 8;
}
// Stage row stride: kx = 0..M, and a residue mod 16 (in 8-byte words) that
// spreads one cp.async instruction's B planes x 32/B consecutive kx over the
// 16 bank pairs exactly twice (4 for B = 4 and 8, 1 for B = 16).
template <int M, int B>
constexpr int stage_row() {
    constexpr int want = B == 16 ? 1 : 4;
    return M + 1 + ((want - (M + 1) % 16) + 16) % 16;
}
// Output tile [k][b], row stride B, plane b of row k at b ^ swz(k): a warp's
// 16 consecutive kx of one plane and a copy-out instruction's B planes x 32/B
// consecutive kx both touch every bank pair equally often.
// B = 24 (no XOR swizzle stays inside a 24-plane row): rows of 25 slots,
// whose odd stride spreads 16 consecutive kx of one plane over all bank pairs.
template <int B>
constexpr int out_row() {
    return B == 24 ? 25 : B;
}
template <int B>
__device__ __forceinline__ int out_slot(int k, int b) {
    if constexpr (B == 24)
        return k * out_row<B>() + b;
    else
        return k * B + (b ^ ((k / (16 / B)) & (B - 1)));
}
// Entries of the lane-ordered FFT twiddle table (512-point rows only).
template <int M>
constexpr int rr_entries() {
    if constexpr (M == 256) {
        return rr_table_size<M>();
    } else {
        return 0;
    }
}
template <int M, int B>
constexpr size_t rows_smem_words(int keep) {
    return size_t(B) * region<M>() + 2 * size_t(B) * stage_row<M, B>() + size_t(keep) * B + M + rr_entries<M>();
}

// Launch bounds keep 128 registers per thread whatever the CTA width:
// 16 / B CTAs of 32 * B threads fill 512 threads' worth of the register file.
template <int M, int B>
__global__ void __launch_bounds__(32 * B, 16 / B) rows_flux_kernel(RowFluxArgs a) {
    using V = float2;
    constexpr int NT = 32 * B;
    constexpr int PER = M / 32;  // elements of its plane each lane keeps in registers
    constexpr int XP = region<M>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int KP = stage_row<M, B>();
    static_assert(M != 256 || XP >= rr_region_min<256>(), "plane region too small for warp_fft_rr");
    const int keep = a.keep;
    V* xs = reinterpret_cast<V*>(smem_raw);
    V* stage0 = xs + B * XP;
    V* stage1 = stage0 + B * KP;
    V* outTile = stage1 + B * KP;  // [k][b] at out_slot(k, b)
    V* tf = outTile + keep * B;        // twFull[0..M)
    V* tt = tf + M;                    // warp_fft_rr table (M = 256)
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int zChunks = (a.nz + B - 1) / B;
    const int member = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int y = blockIdx.y;
    const V* twHalf = static_cast<const V*>(a.twHalf);
    const V* twFull = static_cast<const V*>(a.twFull);
    const V* in = static_cast<const V*>(a.binsIn.data);
    V* out = static_cast<V*>(a.binsOut.data);
    const long long inRow = a.binsIn.planes;  // stride between kx
    const long long outRow = a.binsOut.planes;
    V* x = xs + warp * XP;  // this warp's plane

    for (int i = tid; i < M; i += NT) tf[i] = twFull[i];
    if constexpr (rr_entries<M>() > 0) rr_fill_table<float, M>(tt, twHalf, tid, NT);
    for (int i = tid; i < 2 * B * (KP - keep); i += NT) {
        const int row = i / (KP - keep);
        stage0[row * KP + keep + i % (KP - keep)] = V{0.f, 0.f};
    }

    // Asynchronous copy of slot f's bins of this row into a plane-major stage
    // [b][k]; consecutive threads read consecutive planes of one kx (the
    // planes-innermost global rows), planes beyond Nz are zero-filled.  NT is a
    // multiple of B, so a thread keeps its plane cb and steps kx by NT / B.
    constexpr int KSTEP = NT / B;
    const int cb = tid % B;
    const int ck = tid / B;
    const bool cok = z0 + cb < a.nz;
    auto issue = [&](int f, V* stage) {
        const long long plane = (static_cast<long long>(member) * a.fieldsIn + f) * a.zStride + z0 + cb;
        const V* src = in + plane + inRow * (a.binsIn.kxStride * y + ck);
        V* dst = stage + cb * KP + ck;
        for (int k = ck; k < keep; k += KSTEP, src += inRow * KSTEP, dst += KSTEP) cp_async8(dst, cok ? src : in, cok ? 8 : 0);
        cp_async_commit();
    };

    // Inverse row transform of slot f into this lane's registers r[]: element
    // lane + 32e of the warp's plane.
    auto inverse_row = [&](int f, V (&r)[PER]) {
        cp_async_wait_all();
        __syncthreads();
        if (f + 1 < a.fieldsIn) issue(f + 1, ((f + 1) & 1) ? stage1 : stage0);
        const V* st = ((f & 1) ? stage1 : stage0) + warp * KP;
        auto load = [&](int k) -> V {
            if (k >= keep) return V{0.f, 0.f};
            V v = st[k];
            if (k == 0 || k == M) v.y = 0.f;
            return v;
        };
        if constexpr (M == 256) {
            // Pre-processed half-length spectrum straight into registers
            // (element k = lane + 32e), then the register-ended FFT.  At k = 0
            // (lane 0, e = 0) the bins 0 and M are real, and the general form
            // reduces to {X0 + XM, X0 - XM} since tf[0] = 1.
            const V* stk = st + lane;
            const V* stm = st + (M - lane);
            const V* tfk = tf + lane;
#pragma unroll
            for (int e = 0; e < PER; ++e) {
                V xk = stk[32 * e];
                V xm = stm[-32 * e];
                if (e == 0 && lane == 0) {
                    xk.y = 0.f;
                    xm.y = 0.f;
                }
                const V s = cadd(xk, cconj(xm));
                const V d = csub(xk, cconj(xm));
                const V t = cmulc(d, tfk[32 * e]);
                r[e] = {s.x - t.y, s.y + t.x};
            }
            warp_fft_rr<float, M, +1>(r, x, tt, lane);
        } else {
            constexpr int pairs = M / 2 + 1;
            for (int k = lane; k < pairs; k += 32) {
                if (k == 0) {
                    const V x0 = load(0);
                    const V xm = load(M);
                    x[pad16(0)] = {x0.x + xm.x, x0.x - xm.x};
                    continue;
                }
                const int kk = M - k;
                const V xk = load(k);
                const V xm = load(kk);
                {
                    const V s = cadd(xk, cconj(xm));
                    const V d = csub(xk, cconj(xm));
                    const V t = cmulc(d, tf[k]);
                    x[pad16(k)] = {s.x - t.y, s.y + t.x};
                }
                if (kk != k) {
                    const V s = cadd(xm, cconj(xk));
                    const V d = csub(xm, cconj(xk));
                    const V t = cmulc(d, tf[kk]);
                    x[pad16(kk)] = {s.x - t.y, s.y + t.x};
                }
            }
            __syncwarp();
            warp_fft<float, M, +1>(x, twHalf, lane);
#pragma unroll
            for (int e = 0; e < PER; ++e) r[e] = x[pad16(lane + 32 * e)];
            __syncwarp();
        }
    };

    issue(0, stage0);
    V u[PER], v[PER], w[PER];
    inverse_row(0, u);
    inverse_row(1, v);
    inverse_row(2, w);
    const float scale = a.scale;
    for (int t = 0; t < a.targets; ++t) {
        V acc[PER], q[PER];
        inverse_row(3 + 3 * t, q);
#pragma unroll
        for (int e = 0; e < PER; ++e) acc[e] = {u[e].x * q[e].x, u[e].y * q[e].y};
        inverse_row(4 + 3 * t, q);
#pragma unroll
        for (int e = 0; e < PER; ++e) acc[e] = {acc[e].x + v[e].x * q[e].x, acc[e].y + v[e].y * q[e].y};
        inverse_row(5 + 3 * t, q);
#pragma unroll
        for (int e = 0; e < PER; ++e)
            acc[e] = {-scale * (acc[e].x + w[e].x * q[e].x), -scale * (acc[e].y + w[e].y * q[e].y)};
        if constexpr (M == 256) {
            warp_fft_rr<float, M, -1>(acc, x, tt, lane);
            // pad16(lane + 32e) = lane + lane/16 + 34e
            V* o = x + lane + (lane >> 4);
#pragma unroll
            for (int e = 0; e < PER; ++e) o[34 * e] = acc[e];
        } else {
#pragma unroll
            for (int e = 0; e < PER; ++e) x[pad16(lane + 32 * e)] = acc[e];
            __syncwarp();
            warp_fft<float, M, -1>(x, twHalf, lane);
        }
        __syncwarp();
        // Real-spectrum split of the half-length FFT, kx < keep, into [k][b].
        const V zz = x[pad16(0)];
        for (int k = lane; k < keep; k += 32) {
            V X;
            if (k == 0) {
                X = {zz.x + zz.y, 0.f};
            } else if (k == M) {
                X = {zz.x - zz.y, 0.f};
            } else {
                const V zk = x[pad16(k)];
                const V zm = cconj(x[pad16(M - k)]);
                const V ev = cscale(cadd(zk, zm), 0.5f);
                const V d = csub(zk, zm);
                const V o = {0.5f * d.y, -0.5f * d.x};
                X = cadd(ev, cmul(tf[k], o));
            }
            outTile[out_slot<B>(k, warp)] = X;
        }
        __syncthreads();
        // Coalesced rows of B planes per kx.
        if (cok) {
            const long long plane = (static_cast<long long>(member) * a.targets + t) * a.zStride + z0 + cb;
            V* dst = out + plane + outRow * (a.binsOut.kxStride * y + ck);
            for (int k = ck; k < keep; k += KSTEP, dst += outRow * KSTEP) *dst = outTile[out_slot<B>(k, cb)];
        }
        // The next outTile write happens after the next inverse_row's barrier.
    }
}

// ---------------------------------------------------------------------------
// 512-point rows, two planes per warp.
//
// The 256-point complex FFT of the half-length formulation is split 16 x 16:
// lane t of a half-warp holds elements t + 16 m (m = 0..15) of its plane's
// sequence; a radix-16 DFT over m in registers, the twiddles W256^(t k2), one
// 16 x 16 transpose through shared memory, and a second radix-16 DFT in
// registers leave output k = t + 16 k1 in register k1 — the same lane-owned
// positions as the input, so U, V, W and the product stay in registers across
// all transforms as in the warp-per-plane kernel, with one shared-memory
// exchange per transform instead of two.  Lanes 0-15 own plane 2w of warp w,
// lanes 16-31 plane 2w + 1.

// Twiddle W16^e with exponent sign SIGN, e in {1, 2, 3, 6, 9} (e = 4 is a
// multiplication by SIGN*i): cos(2 pi e / 16) + SIGN i sin(2 pi e / 16).
template <int SIGN, int E>
__device__ __forceinline__ float2 w16() {
    constexpr float c1 = 0.923879532511286756128f;  // cos(pi/8)
    constexpr float s1 = 0.382683432365089771728f;  // sin(pi/8)
    constexpr float h = 0.707106781186547524401f;   // cos(pi/4)
    constexpr float sg = SIGN < 0 ? -1.0f : 1.0f;
    if constexpr (E == 1) return {c1, sg * s1};
    if constexpr (E == 2) return {h, sg * h};
    if constexpr (E == 3) return {s1, sg * c1};
    if constexpr (E == 6) return {-h, sg * h};
    return {-c1, -sg * s1};  // E == 9
}

// In-place length-16 DFT over v[0..15] (natural order in and out): 16 = 4 x 4,
// input m = m2 + 4 m1, output k = k1 + 4 k2.
template <int SIGN>
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) dft4<SIGN>(v[m2], v[m2 + 4], v[m2 + 8], v[m2 + 12]);
    // v[m2 + 4 k1] *= W16^(m2 k1)
    v[5] = cmul(v[5], w16<SIGN, 1>());
    v[9] = cmul(v[9], w16<SIGN, 2>());
    v[13] = cmul(v[13], w16<SIGN, 3>());
    v[6] = cmul(v[6], w16<SIGN, 2>());
    v[10] = cmul_si<SIGN>(v[10]);
    v[14] = cmul(v[14], w16<SIGN, 6>());
    v[7] = cmul(v[7], w16<SIGN, 3>());
    v[11] = cmul(v[11], w16<SIGN, 6>());
    v[15] = cmul(v[15], w16<SIGN, 9>());
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<SIGN>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4 k1 + k2] holds output k1 + 4 k2: transpose the 4 x 4 block.
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i + 1; j < 4; ++j) {
            const float2 t = v[4 * i + j];
            v[4 * i + j] = v[4 * j + i];
            v[4 * j + i] = t;
        }
}

// 256-point FFT of one half-warp's sequence: v[m] = z[t + 16 m] in, Z[t + 16 k]
// in v[k] out.  xch: this half-warp's 16 x 17 exchange region; tw2[16 k2 + t] =
// exp(-2 pi i t k2 / 256) (conjugated for SIGN > 0).
template <int SIGN>
__device__ __forceinline__ void fft256_pair(float2 (&v)[16], float2* xch, const float2* tw2, int t) {
    dft16<SIGN>(v);
#pragma unroll
    for (int k2 = 1; k2 < 16; ++k2) {
        const float2 w = tw2[16 * k2 + t];
        v[k2] = SIGN < 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
    __syncwarp();  // the previous transform's reads of xch are done
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) xch[17 * t + k2] = v[k2];
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) v[n1] = xch[17 * n1 + t];
    dft16<SIGN>(v);
}

constexpr int kPairM = 256;       // half-length of the 512-point rows
constexpr int kPairXch = 16 * 17;  // exchange words per plane
template <int B>
constexpr int pair_stage_row() {
    // kx = 0..M (the pre-processing reads X[M - k]), and a residue mod 16 (in
    // 8-byte words) that spreads one cp.async instruction's B planes x 32/B
    // kx over the 16 bank pairs exactly twice.
    // (B = 24: an odd stride, at most three accesses per bank pair.)
    constexpr int want = B == 16 || B == 24 ? 1 : 2;
    return kPairM + 1 + ((want - (kPairM + 1) % 16) + 16) % 16;
}
template <int B>
constexpr size_t pair_smem_words(int keep) {
    return 2 * size_t(B) * pair_stage_row<B>() + size_t(B) * kPairXch + size_t(keep) * out_row<B>() + kPairM + kPairM;
}

// TMA form of the stage: rows kx = 0..kTmaRows-1 (the pre-processing reads no
// bin beyond kx = 176, see inverse_row), each row the B planes' values
// (64 or 128 bytes) in the SWIZZLE_64B / SWIZZLE_128B pattern the tensor
// copy writes; rows keep..kTmaRows-1 are zero.  Stages start on 1024-byte
// boundaries (the swizzle pattern's period).
constexpr int kTmaRows = 177;
template <int B>
constexpr size_t tma_stage_bytes() {
    return (size_t(kTmaRows) * B * 8 + 1023) / 1024 * 1024;
}
// W_SMEM: the third velocity row W is kept in a lane-private shared region
// (16 values per thread) instead of registers.
template <int B, int MINB, int NS>
constexpr bool pair_w_in_smem() {
    return B == 8 && MINB == 3 && NS == 2;
}
template <int B, int NS, bool WSM = false>
constexpr size_t pair_tma_smem_bytes(int keep) {
    return 1024 + NS * tma_stage_bytes<B>() +
           sizeof(float2) * (size_t(B) * kPairXch + size_t(keep) * out_row<B>() + kPairM + kPairM +
                             (WSM ? size_t(16) * 16 * B : 0));
}
// Byte offset of (kx k, plane b) in a swizzled TMA stage.
template <int B>
__device__ __forceinline__ unsigned tma_stage_offset(int k, int b) {
    const unsigned off = static_cast<unsigned>((k * B + b) * 8);
    return off ^ (((off >> 7) & (B == 8 ? 3u : 7u)) << 4);
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// A bounded wait on an mbarrier phase (false once the limit is reached).
__device__ __forceinline__ bool stage_wait(unsigned bar, unsigned parity, long long limit = 1LL << 22) {
    for (long long i = 0; i < limit; ++i) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// MINB: resident CTAs per SM the register allocation must allow (2 for B = 8,
// 1 for B = 16: about 240 registers; 3 for the B = 8 form that trades spills
// to L1-cached local memory for occupancy).
// TMA (NS = 2 or 3 stages; 0: cp.async): each slot's stage is filled by one
// tensor copy (thread 0, onto an mbarrier; `tmIn` maps the input bins as
// [cell][plane]) instead of 8-byte cp.async by every thread, NS - 1 slots
// ahead of the one being transformed.  Thread 0's bounded wait on the copy is
// folded into the slot's CTA barrier (__syncthreads_and), so an expired wait
// makes every thread leave together after setting the error word.
template <int B, int MINB, int NS>
__global__ void __launch_bounds__(16 * B, MINB)
    rows_flux_pair_kernel(RowFluxArgs a, const __grid_constant__ CUtensorMap tmIn) {
    using V = float2;
    constexpr bool TMA = NS != 0;
    constexpr int NST = TMA ? NS : 2;  // stages
    constexpr int M = kPairM;
    constexpr int NT = 16 * B;
    constexpr int KP = pair_stage_row<B>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long stageFull[NST];
    __shared__ __align__(8) unsigned long long never;  // nothing arrives on it (expired-wait test)
    const int keep = a.keep;
    unsigned char* tmaBase =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    auto stage_of = [&](int f) -> V* {
        if constexpr (TMA)
            return reinterpret_cast<V*>(tmaBase + (f % NST) * tma_stage_bytes<B>());
        else
            return reinterpret_cast<V*>(smem_raw) + (f & 1) * B * KP;
    };
    V* stage0 = stage_of(0);
    V* xchAll = TMA ? reinterpret_cast<V*>(tmaBase + NST * tma_stage_bytes<B>()) : stage0 + 2 * B * KP;
    V* outTile = xchAll + B * kPairXch;  // [k][b] at out_slot(k, b)
    V* tf = outTile + keep * out_row<B>();  // twFull[0..M)
    V* tw2 = tf + M;                     // tw2[16 k2 + t] = twHalf[(t k2) mod M]
    // Three-CTA two-stage TMA form: W (16 values per thread) lives here, at
    // wsm[16 * e ... ] + tid, which takes the register peak of u, v, w, the
    // product and the current derivative under the 168-register bound.
    constexpr bool WSM = pair_w_in_smem<B, MINB, NS>();
    V* wsm = tw2 + M;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int t = lane & 15;
    const int pl = 2 * warp + (lane >> 4);  // this half-warp's plane within the CTA
    const int zChunks = (a.nz + B - 1) / B;
    const int member = blockIdx.x / zChunks;
    const int z0 = (blockIdx.x % zChunks) * B;
    const int y = blockIdx.y;
    const V* twHalf = static_cast<const V*>(a.twHalf);
    const V* twFull = static_cast<const V*>(a.twFull);
    const V* in = static_cast<const V*>(a.binsIn.data);
    V* out = static_cast<V*>(a.binsOut.data);
    const long long inRow = a.binsIn.planes;
    const long long outRow = a.binsOut.planes;
    V* xch = xchAll + pl * kPairXch;

    for (int i = tid; i < M; i += NT) {
        tf[i] = twFull[i];
        tw2[i] = twHalf[((i & 15) * (i >> 4)) & (M - 1)];
    }
    if constexpr (TMA) {
        // Rows keep..kTmaRows-1 of every stage are zero (the tensor copies
        // write rows 0..keep-1 only; the swizzle stays inside a row).
        for (int i = tid; i < NST * (kTmaRows - keep) * B; i += NT) {
            const int st = i / ((kTmaRows - keep) * B);
            const int j = i % ((kTmaRows - keep) * B);
            reinterpret_cast<V*>(tmaBase + st * tma_stage_bytes<B>())[keep * B + j] = V{0.f, 0.f};
        }
        if (tid == 0) {
            for (int i = 0; i < NST; ++i)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&stageFull[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&never)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    } else {
        for (int i = tid; i < 2 * B * (KP - keep); i += NT) {
            const int row = i / (KP - keep);
            stage0[row * KP + keep + i % (KP - keep)] = V{0.f, 0.f};
        }
    }

    // Slot f's bins of this row into a plane-major stage [b][k] (cp.async, as
    // in the warp-per-plane kernel; planes beyond Nz are zero-filled), or, in
    // the TMA form, into a swizzled [k][b] stage by one tensor copy (planes
    // beyond Nz then hold the next slot's or padding values; those planes'
    // results are never stored).
    constexpr int KSTEP = NT / B;
    const int cb = tid % B;
    const int ck = tid / B;
    const bool cok = z0 + cb < a.nz;
    const int tmaLo = static_cast<int>(tma_stage_offset<B>(t, pl));
    const int tmaHi = static_cast<int>(tma_stage_offset<B>(M - t, pl));
    auto issue = [&](int f) {
        V* stage = stage_of(f);
        if constexpr (TMA) {
            if (tid == 0) {
                const int x = (member * a.fieldsIn + f) * a.zStride + z0;
                const int yc = static_cast<int>(a.binsIn.kxStride * y);
                const unsigned bar = smem_addr(&stageFull[f % NST]);
                // The stage's earlier shared-memory reads precede the copy's writes.
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                             "r"(static_cast<unsigned>(keep * B * 8))
                             : "memory");
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3}], [%4];" ::"r"(smem_addr(stage)),
                    "l"(reinterpret_cast<unsigned long long>(&tmIn)), "r"(x), "r"(yc), "r"(bar)
                    : "memory");
            }
        } else {
            const long long plane = (static_cast<long long>(member) * a.fieldsIn + f) * a.zStride + z0 + cb;
            const V* src = in + plane + inRow * (a.binsIn.kxStride * y + ck);
            V* dst = stage + cb * KP + ck;
            for (int k = ck; k < keep; k += KSTEP, src += inRow * KSTEP, dst += KSTEP) cp_async8(dst, cok ? src : in, cok ? 8 : 0);
            cp_async_commit();
        }
    };

    // c2r of slot f into r[m] = x-pair t + 16 m of this half-warp's plane;
    // false if the TMA form's wait for the slot's copy expired.
    auto inverse_row = [&](int f, V (&r)[16]) -> bool {
        if constexpr (TMA) {
            bool ok = tid != 0 || stage_wait(smem_addr(&stageFull[f % NST]), (f / NST) & 1);
            // Expired-wait test: once slot 0's copy has landed (no copy is then
            // in flight), a short bounded wait on a barrier nothing signals
            // runs out and takes the path of any expired wait.
            if (tid == 0 && ok && f == 0 && a.expireWaitForTest != 0)
                ok = stage_wait(smem_addr(&never), 0, 1LL << 14);
            if (!__syncthreads_and(ok)) {
                if (tid == 0 && a.error != nullptr) atomicExch(a.error, 1);
                return false;
            }
        } else {
            cp_async_wait_all();
            __syncthreads();
        }
        // The stage refilled here was last read in the previous slot, before
        // this barrier.
        if (f + NST - 1 < a.fieldsIn) issue(f + NST - 1);
        const V* st = stage_of(f) + pl * KP;
        const unsigned char* stb = reinterpret_cast<const unsigned char*>(stage_of(f));
        // TMA form: bins k = t + 16 m and M - k sit at this lane's swizzled
        // offsets of m = 0 plus or minus m rows of 16 (16 * B * 8 bytes, a
        // multiple of the swizzle period, so the pattern repeats).
        auto bin = [&](int m, bool mirror) -> V {
            if constexpr (TMA)
                return *reinterpret_cast<const V*>(stb + (mirror ? tmaHi - m * 128 * B : tmaLo + m * 128 * B));
            else
                return st[mirror ? M - t - 16 * m : t + 16 * m];
        };
        // keep <= 176 (checked at launch): bins k >= 176 (m >= 11) and
        // M - k >= 177 (m <= 4) lie beyond the 2/3 band and are zero, so those
        // shared-memory reads are left out.
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int k = t + 16 * m;
            V xk = m < 11 ? bin(m, false) : V{0.f, 0.f};
            V xm = m > 4 ? bin(m, true) : V{0.f, 0.f};
            if (m == 0 && t == 0) {  // bins 0 and M are real
                xk.y = 0.f;
                xm.y = 0.f;
            }
            const V sum = cadd(xk, cconj(xm));
            const V d = csub(xk, cconj(xm));
            const V tt = cmulc(d, tf[k]);
            r[m] = {sum.x - tt.y, sum.y + tt.x};
        }
        fft256_pair<+1>(r, xch, tw2, t);
        return true;
    };

    if constexpr (TMA) __syncthreads();  // barrier init and zero rows before the first copy and reads
    for (int f = 0; f < NST - 1 && f < a.fieldsIn; ++f) issue(f);
    V u[16], v[16], w[16];
    if (!inverse_row(0, u) || !inverse_row(1, v) || !inverse_row(2, w)) return;
    if constexpr (WSM) {
#pragma unroll
        for (int e = 0; e < 16; ++e) wsm[e * NT + tid] = w[e];
    }
    const float scale = a.scale;
    const int src = ((16 - t) & 15) + (lane & 16);  // lane holding Z[M - k]
    for (int tg = 0; tg < a.targets; ++tg) {
        V acc[16], q[16];
        if (!inverse_row(3 + 3 * tg, q)) return;
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[e] = {u[e].x * q[e].x, u[e].y * q[e].y};
        if (!inverse_row(4 + 3 * tg, q)) return;
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[e] = {acc[e].x + v[e].x * q[e].x, acc[e].y + v[e].y * q[e].y};
        if (!inverse_row(5 + 3 * tg, q)) return;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const V we = WSM ? wsm[e * NT + tid] : w[e];
            acc[e] = {-scale * (acc[e].x + we.x * q[e].x), -scale * (acc[e].y + we.y * q[e].y)};
        }
        fft256_pair<-1>(acc, xch, tw2, t);
        // Real-spectrum split, kx < keep, into [k][b].  Z[M - k] for k = t + 16 k1
        // is register 15 - k1 of lane 16 - t (t > 0) or register (16 - k1) mod 16
        // of this lane (t = 0).
#pragma unroll
        for (int k1 = 0; k1 < 11; ++k1) {  // k < 176 >= keep
            const V other = {__shfl_sync(0xFFFFFFFFu, acc[15 - k1].x, src),
                             __shfl_sync(0xFFFFFFFFu, acc[15 - k1].y, src)};
            const int k = t + 16 * k1;
            const V zk = acc[k1];
            const V zm = cconj(t == 0 ? acc[(16 - k1) & 15] : other);
            V X;
            if (k == 0) {
                X = {zk.x + zk.y, 0.f};
            } else {
                const V ev = cscale(cadd(zk, zm), 0.5f);
                const V d = csub(zk, zm);
                const V o = {0.5f * d.y, -0.5f * d.x};
                X = cadd(ev, cmul(tf[k < M ? k : 0], o));
            }
            if (k < keep) outTile[out_slot<B>(k, pl)] = X;
        }
        __syncthreads();
        if (cok) {
            const long long plane = (static_cast<long long>(member) * a.targets + tg) * a.zStride + z0 + cb;
            V* dst = out + plane + outRow * (a.binsOut.kxStride * y + ck);
            for (int k = ck; k < keep; k += KSTEP, dst += outRow * KSTEP) *dst = outTile[out_slot<B>(k, cb)];
        }
        // The next outTile write happens after the next inverse_row's barrier.
    }
}

template <int B, int MINB, int NS>
cudaError_t launch_pair(const RowFluxArgs& a, cudaStream_t stream) {
    constexpr bool TMA = NS != 0;
    const int zChunks = (a.nz + B - 1) / B;
    const dim3 grid(unsigned(zChunks * a.members), unsigned(a.ny));
    auto kernel = rows_flux_pair_kernel<B, MINB, NS>;
    CUtensorMap map{};
    size_t bytes = sizeof(float2) * pair_smem_words<B>(a.keep);
    if constexpr (TMA) {
        // The input bins as [cell][plane]: a cell's planes are contiguous and
        // cells (ky * kxStride + kx) lie `planes` values apart.
        const cudaError_t merr =
            encode_complex_map_2d(&map, a.binsIn.data, static_cast<unsigned long long>(a.binsIn.planes),
                                  static_cast<unsigned long long>(a.ny) * a.binsIn.kxStride,
                                  static_cast<unsigned long long>(a.binsIn.planes) * 8, B, a.keep);
        if (merr != cudaSuccess) return merr;
        bytes = pair_tma_smem_bytes<B, NS, pair_w_in_smem<B, MINB, NS>()>(a.keep);
    }
    const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (err != cudaSuccess) return err;
    kernel<<<grid, 16 * B, bytes, stream>>>(a, map);
    return cudaGetLastError();
}

template <int NS>
cudaError_t launch_pair_form(const RowFluxArgs& a, cudaStream_t stream) {
    if (a.planes == 8) return a.pairs == 2 ? launch_pair<8, 3, NS>(a, stream) : launch_pair<8, 2, NS>(a, stream);
    if (a.planes == 16) return launch_pair<16, 1, NS>(a, stream);
    // 24 planes (12 warps, one CTA per SM, 192-byte pieces): cp.async only,
    // no TMA swizzle pattern fits a 192-byte row.
    if (a.planes == 24) return launch_pair<24, 1, 0>(a, stream);
    return cudaErrorInvalidValue;
}

}  // namespace

template <int M, int B>
cudaError_t launch_m(const RowFluxArgs& a, cudaStream_t stream) {
    const int zChunks = (a.nz + B - 1) / B;
    const dim3 grid(unsigned(zChunks * a.members), unsigned(a.ny));
    auto kernel = rows_flux_kernel<M, B>;
    const size_t bytes = sizeof(float2) * rows_smem_words<M, B>(a.keep);
    if (bytes > 48 * 1024) {
        const cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (err != cudaSuccess) return err;
    }
    kernel<<<grid, 32 * B, bytes, stream>>>(a);
    return cudaGetLastError();
}

template <int M>
cudaError_t launch_planes(const RowFluxArgs& a, cudaStream_t stream) {
    switch (a.planes) {
        case 4: return launch_m<M, 4>(a, stream);
        case 8: return launch_m<M, 8>(a, stream);
        case 16: return launch_m<M, 16>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_rows_flux(const RowFluxArgs& a, cudaStream_t stream) {
    const int M = a.nx / 2;
    if (a.keep < 1 || a.keep > M + 1 || a.fieldsIn != 3 + 3 * a.targets || a.zStride < a.nz) return cudaErrorInvalidValue;
    if (a.pairs != 0 && M == kPairM && a.keep <= 176 && (a.planes == 8 || a.planes == 16 || a.planes == 24)) {
        // The TMA form needs the error word (its copy waits are bounded) and
        // 16-byte aligned cells.
        const bool tma = a.tma != 0 && a.error != nullptr && a.binsIn.planes % 2 == 0 && a.zStride % 2 == 0;
        if (!tma) return launch_pair_form<0>(a, stream);
        return a.tma == 2 ? launch_pair_form<3>(a, stream) : launch_pair_form<2>(a, stream);
    }
    switch (M) {
        case 32: return launch_planes<32>(a, stream);
        case 64: return launch_planes<64>(a, stream);
        case 128: return launch_planes<128>(a, stream);
        case 256: return launch_planes<256>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

bool rows_flux_supported(long long nx) { return nx >= 64 && nx <= 512 && (nx & (nx - 1)) == 0; }

}  // namespace skb
