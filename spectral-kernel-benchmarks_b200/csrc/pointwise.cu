// Pointwise advection product target = -scale*(u*qx + v*qy + w*qz)
// (pointwise_advection.cpp:143-147).  shared = [u, v, w] and derivative =
// [qx, qy, qz], each `volume` elements apart.  Grid-stride, two elements per
// thread per iteration with 8/16-byte vector accesses when the arrays allow it.

#include "pointwise.hpp"

namespace skb {
namespace {

template <typename T>
__global__ void pointwise_kernel(long long volume, T scale, const T* __restrict__ shared,
                                 const T* __restrict__ derivative, T* __restrict__ target) {
    const T* u = shared;
    const T* v = shared + volume;
    const T* w = shared + 2 * volume;
    const T* qx = derivative;
    const T* qy = derivative + volume;
    const T* qz = derivative + 2 * volume;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < volume; i += stride)
        target[i] = -scale * (u[i] * qx[i] + v[i] * qy[i] + w[i] * qz[i]);
}

template <typename T, typename V2>
__global__ void pointwise_vec2_kernel(long long pairs, T scale, const V2* __restrict__ u, const V2* __restrict__ v,
                                      const V2* __restrict__ w, const V2* __restrict__ qx,
                                      const V2* __restrict__ qy, const V2* __restrict__ qz, V2* __restrict__ target) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += stride) {
        const V2 a = u[i], b = v[i], c = w[i], x = qx[i], y = qy[i], z = qz[i];
        V2 r;
        r.x = -scale * (a.x * x.x + b.x * y.x + c.x * z.x);
        r.y = -scale * (a.y * x.y + b.y * y.y + c.y * z.y);
        target[i] = r;
    }
}

template <typename T, typename V2>
cudaError_t launch_t(long long volume, double scale, const void* shared, const void* derivative, void* target,
                     int smCount, cudaStream_t stream) {
    const T* s = static_cast<const T*>(shared);
    const T* d = static_cast<const T*>(derivative);
    T* t = static_cast<T*>(target);
    const int threads = 256;
    const bool aligned = volume % 2 == 0 && (reinterpret_cast<uintptr_t>(s) % (2 * sizeof(T))) == 0 &&
                         (reinterpret_cast<uintptr_t>(d) % (2 * sizeof(T))) == 0 &&
                         (reinterpret_cast<uintptr_t>(t) % (2 * sizeof(T))) == 0;
    if (aligned) {
        const long long pairs = volume / 2;
        const long long blocks = std::min<long long>((pairs + threads - 1) / threads, (long long)smCount * 16);
        pointwise_vec2_kernel<T, V2><<<unsigned(std::max(1LL, blocks)), threads, 0, stream>>>(
            pairs, T(scale), reinterpret_cast<const V2*>(s), reinterpret_cast<const V2*>(s + volume),
            reinterpret_cast<const V2*>(s + 2 * volume), reinterpret_cast<const V2*>(d),
            reinterpret_cast<const V2*>(d + volume), reinterpret_cast<const V2*>(d + 2 * volume),
            reinterpret_cast<V2*>(t));
    } else {
        const long long blocks = std::min<long long>((volume + threads - 1) / threads, (long long)smCount * 16);
        pointwise_kernel<T><<<unsigned(std::max(1LL, blocks)), threads, 0, stream>>>(volume, T(scale), s, d, t);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pointwise(bool f64, long long volume, double scale, const void* shared, const void* derivative,
                             void* target, int smCount, cudaStream_t stream) {
    if (volume <= 0) return cudaSuccess;
    return f64 ? launch_t<double, double2>(volume, scale, shared, derivative, target, smCount, stream)
               : launch_t<float, float2>(volume, scale, shared, derivative, target, smCount, stream);
}

}  // namespace skb
