// Shared-memory batched complex FFT used by the horizontal transform kernels.
//
// Layout: one CTA transforms B independent length-N sequences held in shared
// memory as data[n * B + b] (batch innermost).  B is chosen so a row of B
// complex values is 128 bytes (8 double2 or 16 float2): consecutive threads
// then touch consecutive 8/16-byte words, which makes every pass free of bank
// conflicts and lets the global loads and stores that fill and drain the
// buffer move whole 32-byte sectors when the batch index is the innermost
// global index too (planes are innermost in the WVM layout).
//
// Algorithm: Stockham auto-sort, decimation in time.  Pass p with current
// sub-transform size Ns and radix R: butterfly j reads x[j + r*N/R], multiplies
// by the twiddle w^(r*(j mod Ns)) with w = exp(sign*2*pi*i/(Ns*R)), applies a
// length-R DFT and writes x[(j/Ns)*Ns*R + (j mod Ns) + r*Ns].  Output is in
// natural order.  Every thread owns exactly eight elements per pass (one
// radix-8 butterfly, two radix-4 or four radix-2 butterflies), so a pass reads
// all its inputs into registers, synchronises, and writes in place.
//
// Twiddles come from a table tw[k] = exp(-2*pi*i*k/N), k in [0, N), generated on
// the host in long double and rounded to T (see twiddles.cpp); the inverse
// direction uses their conjugates.

#pragma once

#include <cuda_runtime.h>

namespace skb {

template <typename T>
struct Cx;
template <>
struct Cx<double> {
    using type = double2;
};
template <>
struct Cx<float> {
    using type = float2;
};
template <typename T>
using cx = typename Cx<T>::type;

template <typename V>
__device__ __forceinline__ V cadd(V a, V b) {
    return {a.x + b.x, a.y + b.y};
}
template <typename V>
__device__ __forceinline__ V csub(V a, V b) {
    return {a.x - b.x, a.y - b.y};
}
template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename V>
__device__ __forceinline__ V cmulc(V a, V b) {
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename V>
__device__ __forceinline__ V cconj(V a) {
    return {a.x, -a.y};
}
template <typename V, typename S>
__device__ __forceinline__ V cscale(V a, S s) {
    return {a.x * s, a.y * s};
}
// a * (sign * i); SIGN = -1 for the forward transform, +1 for the inverse.
template <int SIGN, typename V>
__device__ __forceinline__ V cmul_si(V a) {
    if (SIGN < 0) return {a.y, -a.x};
    return {-a.y, a.x};
}

template <int SIGN, typename V>
__device__ __forceinline__ void dft2(V& a, V& b) {
    const V t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

// In-place length-4 DFT with exponent sign SIGN (natural-order output).
template <int SIGN, typename V>
__device__ __forceinline__ void dft4(V& x0, V& x1, V& x2, V& x3) {
    const V c0 = cadd(x0, x2);
    const V c1 = csub(x0, x2);
    const V c2 = cadd(x1, x3);
    const V c3 = cmul_si<SIGN>(csub(x1, x3));
    x0 = cadd(c0, c2);
    x2 = csub(c0, c2);
    x1 = cadd(c1, c3);
    x3 = csub(c1, c3);
}

// In-place length-8 DFT: split into even/odd output halves with the eighth
// roots of unity, then two length-4 DFTs.
template <int SIGN, typename V>
__device__ __forceinline__ void dft8(V* v) {
    using S = decltype(v[0].x);
    const S h = S(0.707106781186547524400844362104849039);
    V a0 = cadd(v[0], v[4]), a1 = cadd(v[1], v[5]), a2 = cadd(v[2], v[6]), a3 = cadd(v[3], v[7]);
    V b0 = csub(v[0], v[4]), b1 = csub(v[1], v[5]), b2 = csub(v[2], v[6]), b3 = csub(v[3], v[7]);
    // b1 *= h*(1 + SIGN*i); b2 *= SIGN*i; b3 *= h*(-1 + SIGN*i)
    const V w1 = {h, S(SIGN) * h};
    const V w3 = {-h, S(SIGN) * h};
    b1 = cmul(b1, w1);
    b2 = cmul_si<SIGN>(b2);
    b3 = cmul(b3, w3);
    dft4<SIGN>(a0, a1, a2, a3);
    dft4<SIGN>(b0, b1, b2, b3);
    v[0] = a0;
    v[2] = a1;
    v[4] = a2;
    v[6] = a3;
    v[1] = b0;
    v[3] = b1;
    v[5] = b2;
    v[7] = b3;
}

template <int SIGN, typename V>
__device__ __forceinline__ V twiddle(const V* __restrict__ tw, int k) {
    const V w = __ldg(tw + k);
    return SIGN < 0 ? w : cconj(w);
}

constexpr int fft_threads(int N) { return N >= 8 ? N / 8 : 1; }

// Transform B sequences of length N in shared memory, element (n, b) at
// data[n * LD + b] (LD = B, or B + 1 where callers also walk along n).  Must
// be called by all fft_threads(N)*B threads (tid in [0, that)); other threads
// of the CTA must still reach the __syncthreads() calls, which is why
// `active` exists.
template <typename T, int N, int B, int SIGN, int LD = B>
__device__ __forceinline__ void fft_smem(cx<T>* data, const cx<T>* __restrict__ tw, int tid, bool active) {
    using V = cx<T>;
    if constexpr (N == 1) {
        return;
    } else if constexpr (N < 8) {
        // Tiny lengths (rows of an 8-point grid): one thread per sequence.
        if (active) {
            V v[N];
            const int b = tid;
#pragma unroll
            for (int n = 0; n < N; ++n) v[n] = data[n * LD + b];
            if constexpr (N == 2) {
                dft2<SIGN>(v[0], v[1]);
            } else {
                V t0 = v[0], t1 = v[1], t2 = v[2], t3 = v[3];
                dft4<SIGN>(t0, t1, t2, t3);
                v[0] = t0;
                v[1] = t1;
                v[2] = t2;
                v[3] = t3;
            }
#pragma unroll
            for (int n = 0; n < N; ++n) data[n * LD + b] = v[n];
        }
        __syncthreads();
    } else {
        const int b = tid % B;
        const int j = tid / B;  // butterfly group in [0, N/8)
        int Ns = 1;
#pragma unroll
        for (int pass = 0; pass < 12; ++pass) {
            if (Ns * 8 > N) break;
            V v[8];
            if (active) {
#pragma unroll
                for (int r = 0; r < 8; ++r) v[r] = data[(j + r * (N / 8)) * LD + b];
                const int k = j % Ns;
                if (Ns > 1) {
                    const int step = k * (N / (Ns * 8));
#pragma unroll
                    for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], twiddle<SIGN>(tw, step * r));
                }
                dft8<SIGN>(v);
            }
            __syncthreads();
            if (active) {
                const int k = j % Ns;
                const int base = (j / Ns) * Ns * 8 + k;
#pragma unroll
                for (int r = 0; r < 8; ++r) data[(base + r * Ns) * LD + b] = v[r];
            }
            __syncthreads();
            Ns *= 8;
        }
        constexpr int rest = [] {
            int ns = 1;
            while (ns * 8 <= N) ns *= 8;
            return N / ns;
        }();
        if constexpr (rest == 4) {
            // Final radix-4 pass: Ns = N/4, two butterflies per thread.
            constexpr int ns = N / 4;
            V v[8];
            if (active) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int jj = j + s * (N / 8);
#pragma unroll
                    for (int r = 0; r < 4; ++r) v[4 * s + r] = data[(jj + r * ns) * LD + b];
#pragma unroll
                    for (int r = 1; r < 4; ++r) v[4 * s + r] = cmul(v[4 * s + r], twiddle<SIGN>(tw, jj * r));
                    dft4<SIGN>(v[4 * s], v[4 * s + 1], v[4 * s + 2], v[4 * s + 3]);
                }
            }
            __syncthreads();
            if (active) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int jj = j + s * (N / 8);
#pragma unroll
                    for (int r = 0; r < 4; ++r) data[(jj + r * ns) * LD + b] = v[4 * s + r];
                }
            }
            __syncthreads();
        } else if constexpr (rest == 2) {
            // Final radix-2 pass: Ns = N/2, four butterflies per thread.
            constexpr int ns = N / 2;
            V v[8];
            if (active) {
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int jj = j + s * (N / 8);
                    v[2 * s] = data[jj * LD + b];
                    v[2 * s + 1] = cmul(data[(jj + ns) * LD + b], twiddle<SIGN>(tw, jj));
                    dft2<SIGN>(v[2 * s], v[2 * s + 1]);
                }
            }
            __syncthreads();
            if (active) {
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int jj = j + s * (N / 8);
                    data[jj * LD + b] = v[2 * s];
                    data[(jj + ns) * LD + b] = v[2 * s + 1];
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-level variant: one warp transforms one length-N sequence held in
// shared memory at x[pad16(n)] (one spare slot per 16 elements: the stride-8
// stores of the first radix-8 pass then spread over all banks of a half-warp,
// while runs of 16 consecutive elements stay contiguous).  Only __syncwarp()
// separates the passes.  Lane l owns butterflies l + 32q.

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

template <typename T, int N, int SIGN>
__device__ __forceinline__ void warp_fft(cx<T>* x, const cx<T>* __restrict__ tw, int lane) {
    using V = cx<T>;
    static_assert(N >= 8 && (N & (N - 1)) == 0, "warp_fft needs a power of two >= 8");
    constexpr int BF = N / 8;
    constexpr int Q = (BF + 31) / 32;
    int Ns = 1;
#pragma unroll
    for (int pass = 0; pass < 12; ++pass) {
        if (Ns * 8 > N) break;
        V v[Q][8];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (j < BF) {
#pragma unroll
                for (int r = 0; r < 8; ++r) v[q][r] = x[pad16(j + r * BF)];
                const int k = j % Ns;
                if (Ns > 1) {
                    const int step = k * (N / (Ns * 8));
#pragma unroll
                    for (int r = 1; r < 8; ++r) v[q][r] = cmul(v[q][r], twiddle<SIGN>(tw, step * r));
                }
                dft8<SIGN>(v[q]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (j < BF) {
                const int k = j % Ns;
                const int base = (j / Ns) * Ns * 8 + k;
#pragma unroll
                for (int r = 0; r < 8; ++r) x[pad16(base + r * Ns)] = v[q][r];
            }
        }
        __syncwarp();
        Ns *= 8;
    }
    constexpr int rest = [] {
        int ns = 1;
        while (ns * 8 <= N) ns *= 8;
        return N / ns;
    }();
    if constexpr (rest == 4) {
        constexpr int ns = N / 4;
        constexpr int Q4 = (ns + 31) / 32;
        V v[Q4][4];
#pragma unroll
        for (int q = 0; q < Q4; ++q) {
            const int jj = lane + 32 * q;
            if (jj < ns) {
#pragma unroll
                for (int r = 0; r < 4; ++r) v[q][r] = x[pad16(jj + r * ns)];
#pragma unroll
                for (int r = 1; r < 4; ++r) v[q][r] = cmul(v[q][r], twiddle<SIGN>(tw, jj * r));
                dft4<SIGN>(v[q][0], v[q][1], v[q][2], v[q][3]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q4; ++q) {
            const int jj = lane + 32 * q;
            if (jj < ns) {
#pragma unroll
                for (int r = 0; r < 4; ++r) x[pad16(jj + r * ns)] = v[q][r];
            }
        }
        __syncwarp();
    } else if constexpr (rest == 2) {
        constexpr int ns = N / 2;
        constexpr int Q2 = (ns + 31) / 32;
        V v[Q2][2];
#pragma unroll
        for (int q = 0; q < Q2; ++q) {
            const int jj = lane + 32 * q;
            if (jj < ns) {
                v[q][0] = x[pad16(jj)];
                v[q][1] = cmul(x[pad16(jj + ns)], twiddle<SIGN>(tw, jj));
                dft2<SIGN>(v[q][0], v[q][1]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q2; ++q) {
            const int jj = lane + 32 * q;
            if (jj < ns) {
                x[pad16(jj)] = v[q][0];
                x[pad16(jj + ns)] = v[q][1];
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Register-ended warp FFT for N in {256, 512}: the sequence enters and leaves
// in registers, element lane + 32e in v[e] (e < N/32).  The first radix-8
// pass reads its butterflies straight from v (butterfly j = lane + 32q needs
// elements j + (N/8)r = lane + 32(q + Qr)), the last pass (radix 4 for 256,
// radix 8 for 512, both with Ns = 64) writes straight back to v (butterfly j
// produces elements j + 64r = lane + 32(q + 2r)), so only the middle pass
// round-trips through the shared region x.  Pass 1 writes element e at
// pad16(e); pass 2 writes element e at e + 8(e/64), so that its stores (the
// butterflies j and j + 8 of a half-warp land 72 = 8 mod 16 words apart) and
// the pass-3 loads (consecutive j) are both free of bank conflicts.  x must
// hold rr_region_min<N>() elements.
//
// Twiddles come from a table in the order the lanes read them (rr_fill_table
// copies them out of the length-N table, so the values are identical):
//   pass 2:  t[8(r-1) + m]       = tw[(N/64) m r],  m = j mod 8, r = 1..7
//   pass 3:  t[56 + 64(r-1) + j] = tw[j r],         j < 64,      r = 1..N/64-1
// A pass-2 read is eight adjacent entries (one wavefront, broadcast), a pass-3
// read 32 adjacent ones, where the strided reads of tw touched up to eight
// lines each.  The table may live in shared or global memory (plain loads).
template <int N>
constexpr int rr_table_size() {
    return 56 + (N / 64 - 1) * 64;
}

template <int N>
constexpr int rr_region_min() {
    return N + 8 * (N / 64 - 1);
}

template <typename T, int N>
__device__ __forceinline__ void rr_fill_table(cx<T>* t, const cx<T>* __restrict__ tw, int tid, int nt) {
    for (int i = tid; i < rr_table_size<N>(); i += nt) {
        int idx;
        if (i < 56) {
            idx = (N / 64) * (i % 8) * (i / 8 + 1);
        } else {
            const int ii = i - 56;
            idx = (ii % 64) * (ii / 64 + 1);
        }
        t[i] = tw[idx];
    }
}

template <int SIGN, typename V>
__device__ __forceinline__ V twiddle_plain(const V* t, int k) {
    const V w = t[k];
    return SIGN < 0 ? w : cconj(w);
}

template <typename T, int N, int SIGN>
__device__ __forceinline__ void warp_fft_rr(cx<T> (&v)[N / 32], cx<T>* x, const cx<T>* t, int lane) {
    using V = cx<T>;
    static_assert(N == 256 || N == 512, "warp_fft_rr handles N = 256 and N = 512");
    constexpr int Q = N / 256;  // radix-8 butterflies per lane in the first / middle passes
    // Addresses as per-lane bases plus compile-time offsets (j < 64, BF = N/8
    // a multiple of 16):
    //   pass-1 stores  pad16(8j + r)   = 8j + j/2 + r
    //   pass-2 loads   pad16(j + BF r) = j + j/16 + (BF + BF/16) r
    //   pass-2 stores  element 64(j/8) + j%8 + 8r at 72(j/8) + j%8 + 8r
    //   pass-3 loads   element j + 64r at j + 72r
    // Pass 1: Ns = 1, radix 8, registers -> x.
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        V b[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) b[r] = v[q + Q * r];
        dft8<SIGN>(b);
        const int j = lane + 32 * q;
        V* o = x + 8 * j + (j >> 1);
#pragma unroll
        for (int r = 0; r < 8; ++r) o[r] = b[r];
    }
    __syncwarp();
    // Pass 2: Ns = 8, radix 8, x -> x.
    {
        V b[Q][8];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            const V* in = x + j + (j >> 4);
#pragma unroll
            for (int r = 0; r < 8; ++r) b[q][r] = in[(N / 8 + N / 128) * r];
            const V* t2 = t + (j % 8);
#pragma unroll
            for (int r = 1; r < 8; ++r) b[q][r] = cmul(b[q][r], twiddle_plain<SIGN>(t2, 8 * (r - 1)));
            dft8<SIGN>(b[q]);
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            V* o = x + 72 * (j / 8) + (j % 8);
#pragma unroll
            for (int r = 0; r < 8; ++r) o[8 * r] = b[q][r];
        }
        __syncwarp();
    }
    // Pass 3: Ns = 64, radix N/64, x -> registers.
    constexpr int R3 = N / 64;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        const V* in = x + j;
        V b[R3];
#pragma unroll
        for (int r = 0; r < R3; ++r) b[r] = in[72 * r];
#pragma unroll
        for (int r = 1; r < R3; ++r) b[r] = cmul(b[r], twiddle_plain<SIGN>(t + 56 + j, 64 * (r - 1)));
        if constexpr (R3 == 4) {
            dft4<SIGN>(b[0], b[1], b[2], b[3]);
        } else {
            dft8<SIGN>(b);
        }
#pragma unroll
        for (int r = 0; r < R3; ++r) v[q + 2 * r] = b[r];
    }
    __syncwarp();
}

}  // namespace skb
