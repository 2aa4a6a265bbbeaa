#include "tensor_map.hpp"

#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

namespace skb {

namespace {
// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library needs no link-time dependency on libcuda.
PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult status{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &status) == cudaSuccess &&
            status == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}
}  // namespace

cudaError_t encode_complex_map_2d(CUtensorMap* map, const void* base, unsigned long long inner,
                                  unsigned long long outer, unsigned long long rowBytes, unsigned boxInner,
                                  unsigned boxOuter) {
    if (map == nullptr || base == nullptr || inner == 0 || outer == 0) return cudaErrorInvalidValue;
    if ((reinterpret_cast<std::uintptr_t>(base) & 15) != 0 || (rowBytes & 15) != 0 || rowBytes < inner * 8)
        return cudaErrorInvalidValue;
    if (boxInner != 8 && boxInner != 16) return cudaErrorInvalidValue;
    if (boxOuter < 1 || boxOuter > 256 || inner >= (1ULL << 32) || outer >= (1ULL << 32)) return cudaErrorInvalidValue;
    const auto fn = encoder();
    if (fn == nullptr) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {rowBytes};
    const cuuint32_t box[2] = {boxInner, boxOuter};
    const cuuint32_t elementStrides[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_INT64, 2, const_cast<void*>(base), dims, strides, box,
                          elementStrides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          boxInner == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace skb
