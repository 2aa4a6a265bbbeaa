// Dense 2-D c2r inverse that allocates nothing: its scratch is a fixed array
// in device memory that this library declares, not memory it asks for.
//
// Who needs it: callers that may not allocate device memory once they are
// running.  A host that enforces its own device-memory budget through its own
// allocator (a serving process that reserves HBM for its caches at start-up,
// a framework plugin whose host forbids cudaMalloc and cudaFree in its compute
// callbacks) cannot let a library call cudaMalloc: the call may fail once the
// budget is reserved, and cudaFree synchronises the whole device, stalling
// every other stream of the host.  skb_fft_inverse_device creates nothing per
// call either, but its handle allocates at creation; this entry point needs no
// handle at all.
//
// The scratch is `g_scratch`, a file-scope device array of kScratchBytes
// (64 MiB).  Every GPU that loads this library holds it until the process
// exits.  Host code cannot use the array's name as a device address (on the
// host it names a stand-in object), so the first call on each device, with
// that device current, looks the address up with cudaGetSymbolAddress and
// keeps it; that first call may also make the CUDA driver load this file's
// device code, so make it before any stream capture begins.  The kept address
// belongs to the device's current context: a host that calls cudaDeviceReset
// on a device ends that context, and this entry point must not be called on
// that device again in the same process.
//
// Each call writes, in stream order, the three twiddle tables and then every
// entry of the intermediate column spectrum it reads, so nothing in the array
// has to start at zero and no call depends on what an earlier call left there.
// All calls share the one array: two calls whose GPU work overlaps (on
// different streams, or from different host threads) race on it and corrupt
// each other's results.  Serialise them, for instance on one stream.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "horizontal.hpp"
#include "noalloc.hpp"
#include "runtime.hpp"

namespace skb {
namespace {

constexpr std::size_t kScratchBytes = std::size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setupMutex;
void* g_scratchAddress[kMaxDevices] = {};

// Device address of g_scratch on the current device (looked up once).
void* scratch_address() {
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices)
        throw Error(-1, "device ordinal " + std::to_string(device) + " is beyond the " +
                            std::to_string(kMaxDevices) + " devices the static scratch supports");
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (g_scratchAddress[device] == nullptr) {
        void* address = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&address, g_scratch);
        if (err != cudaSuccess || address == nullptr)
            throw Error(-2, std::string("cudaGetSymbolAddress of the static scratch array failed: ") +
                                cudaGetErrorString(err));
        g_scratchAddress[device] = address;
    }
    return g_scratchAddress[device];
}

// Byte counts saturate at SIZE_MAX instead of wrapping, so a workload whose
// Nz * fields (both unbounded) overflows the product is refused like any other
// workload that needs more than the array holds.
std::size_t mul_sat(std::size_t a, std::size_t b) {
    std::size_t r = 0;
    return __builtin_mul_overflow(a, b, &r) ? SIZE_MAX : r;
}

std::size_t add_sat(std::size_t a, std::size_t b) {
    std::size_t r = 0;
    return __builtin_add_overflow(a, b, &r) ? SIZE_MAX : r;
}

std::size_t round_up(std::size_t bytes) { return bytes > SIZE_MAX - 255 ? SIZE_MAX : (bytes + 255) & ~std::size_t(255); }

// tw[k] = exp(-2 pi i k / n) for k in [0, n), the table layout the transform
// kernels read.  sincospi of the exact dyadic argument 2k/n, rounded to T.
template <typename V>
__global__ void fill_twiddles_kernel(V* tw, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s, c;
    sincospi(2.0 * static_cast<double>(k) / static_cast<double>(n), &s, &c);
    tw[k].x = static_cast<decltype(tw[k].x)>(c);
    tw[k].y = static_cast<decltype(tw[k].y)>(-s);
}

void fill_twiddles(Precision p, void* tw, int n, cudaStream_t s) {
    const int threads = 256;
    const int blocks = (n + threads - 1) / threads;
    if (p == Precision::f64)
        fill_twiddles_kernel<<<blocks, threads, 0, s>>>(static_cast<double2*>(tw), n);
    else
        fill_twiddles_kernel<<<blocks, threads, 0, s>>>(static_cast<float2*>(tw), n);
    check_cuda(cudaGetLastError(), "twiddle table kernel");
}

}  // namespace

std::size_t static_inverse_scratch_limit() { return kScratchBytes; }

std::size_t static_inverse_scratch_bytes(const Workload& w, Precision p) {
    const std::size_t complexBytes = 2 * element_bytes(p);
    const std::size_t half = std::max<std::uint64_t>(1, w.nx / 2);
    const std::size_t planes = mul_sat(w.nz, w.fields);
    const std::size_t columns = mul_sat(mul_sat(mul_sat(complexBytes, w.ny), w.nxHalf()), planes);
    std::size_t total = round_up(mul_sat(complexBytes, half));
    total = add_sat(total, round_up(mul_sat(complexBytes, w.nx)));
    total = add_sat(total, round_up(mul_sat(complexBytes, w.ny)));
    return add_sat(total, round_up(columns));
}

void inverse_dense_static(const Workload& w, Precision p, const void* wvm, void* real, cudaStream_t s) {
    validate_workload(w);
    if (!supported_length(static_cast<long long>(w.nx)) || !supported_length(static_cast<long long>(w.ny)))
        throw Error(-1, "unsupported: the cuda provider transforms power-of-two Nx and Ny in [2, 1024]; got " +
                            std::to_string(w.nx) + "x" + std::to_string(w.ny));
    const std::size_t need = static_inverse_scratch_bytes(w, p);
    if (need > kScratchBytes)
        throw Error(-1, "workload " + std::to_string(w.nx) + "x" + std::to_string(w.ny) + "x" +
                            std::to_string(w.nz) + " with " + std::to_string(w.fields) + " fields needs " +
                            std::to_string(need) + " bytes of scratch; the allocation-free inverse has a fixed " +
                            std::to_string(kScratchBytes) +
                            "-byte array (use skb_fft_inverse_device with a provider handle instead)");
    unsigned char* base = static_cast<unsigned char*>(scratch_address());
    const std::size_t complexBytes = 2 * element_bytes(p);
    const int half = static_cast<int>(std::max<std::uint64_t>(1, w.nx / 2));
    void* twHalf = base;
    void* twFull = base + round_up(complexBytes * half);
    void* twCol = static_cast<unsigned char*>(twFull) + round_up(complexBytes * w.nx);
    void* bins = static_cast<unsigned char*>(twCol) + round_up(complexBytes * w.ny);

    fill_twiddles(p, twHalf, half, s);
    fill_twiddles(p, twFull, static_cast<int>(w.nx), s);
    fill_twiddles(p, twCol, static_cast<int>(w.ny), s);
    const int keep = static_cast<int>(w.nxHalf());
    const long long planes = static_cast<long long>(w.planes());
    const DenseBins in{const_cast<void*>(wvm), planes, keep};
    const DenseBins mid{bins, planes, keep};
    check_cuda(launch_columns_dense(p, +1, static_cast<int>(w.ny), keep, planes, in, mid, twCol, s),
               "column c2c kernel");
    check_cuda(launch_rows_inverse(p, static_cast<int>(w.nx), static_cast<int>(w.ny), planes, keep, mid, real,
                                   twHalf, twFull, s),
               "row c2r kernel");
}

}  // namespace skb
