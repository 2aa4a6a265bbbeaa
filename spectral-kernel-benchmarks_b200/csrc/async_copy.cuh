// cp.async helpers (sm_80+ asynchronous global -> shared copies).
#pragma once

#include <cuda_runtime.h>

namespace skb {

// Copy `srcBytes` (0 or 8) bytes from global to shared; the rest of the 8
// destination bytes is zero-filled, so srcBytes = 0 writes a zero without a
// global access.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int srcBytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(srcBytes) : "memory");
}
// 4-byte form, same zero-fill rule (srcBytes 0 or 4).
__device__ __forceinline__ void cp_async4(void* dst, const void* src, int srcBytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

}  // namespace skb
