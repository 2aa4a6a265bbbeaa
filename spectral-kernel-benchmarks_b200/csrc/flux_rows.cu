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
template <int B>
__device__ __forceinline__ int out_slot(int k, int b) {
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
