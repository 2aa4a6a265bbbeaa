// Host runtime shared by every C-ABI handle: status errors, owned device
// buffers, and the horizontal / vertical plans (set-up tables + scratch) that
// the providers and the flux pipeline are built from.

#pragma once

#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "horizontal.hpp"
#include "model.hpp"
#include "vertical.hpp"

namespace skb {

// Error carrying one of the SKB_ERR_* status codes.
class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const noexcept { return code_; }

private:
    int code_;
};

[[noreturn]] void throw_cuda(cudaError_t err, const char* what);
inline void check_cuda(cudaError_t err, const char* what) {
    if (err != cudaSuccess) throw_cuda(err, what);
}

using Clock = std::chrono::steady_clock;
inline double seconds_since(Clock::time_point t) {
    return std::chrono::duration<double>(Clock::now() - t).count();
}

// Owned device allocation.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t bytes) { allocate(bytes); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
        o.ptr_ = nullptr;
        o.bytes_ = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr_ = o.ptr_;
            bytes_ = o.bytes_;
            o.ptr_ = nullptr;
            o.bytes_ = 0;
        }
        return *this;
    }
    void allocate(size_t bytes);
    void release() noexcept;
    template <typename T = void>
    T* get() const {
        return static_cast<T*>(ptr_);
    }
    size_t bytes() const noexcept { return bytes_; }
    void upload(const void* src, size_t bytes, cudaStream_t stream = nullptr);

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

template <typename T>
DeviceBuffer upload_vector(const std::vector<T>& v) {
    DeviceBuffer b(v.size() * sizeof(T) + (v.empty() ? sizeof(T) : 0));
    if (!v.empty()) b.upload(v.data(), v.size() * sizeof(T));
    return b;
}

int sm_count();
size_t element_bytes(Precision p);

// Upload a double table in the plan's precision.
DeviceBuffer upload_real_table(const std::vector<double>& values, Precision p);

// Horizontal plan: twiddles, column tables and the dense bin scratch for a
// grid, a kept kx band and a maximum plane count.
class HorizontalPlan {
public:
    HorizontalPlan(const Workload& w, Precision p, bool pruned, std::uint64_t maxPlanes);

    const Workload& workload() const { return w_; }
    Precision precision() const { return p_; }
    int keep() const { return keep_; }
    std::uint64_t modes() const { return modeCount_; }
    ModeTables tables() const;
    DenseBins scratch(std::uint64_t planes) const {
        return {bins_.get(), static_cast<long long>(planes), static_cast<long long>(keep_)};
    }

    // x then y (forward) into views; y then x (inverse) from views.
    void forward(const void* real, std::uint64_t planes, const ViewSet& views, double scale, cudaStream_t s) const;
    void inverse(const ViewSet& views, void* real, cudaStream_t s) const;
    void forward_rows(const void* real, std::uint64_t planes, cudaStream_t s) const;
    void forward_columns(const ViewSet& views, double scale, cudaStream_t s) const;
    void inverse_columns(const ViewSet& views, cudaStream_t s) const;
    void inverse_rows(void* real, std::uint64_t planes, cudaStream_t s) const;
    // Full-grid dense forms (keep = Nx/2+1): WVM spectrum with `planes` planes.
    void forward_dense(const void* real, void* wvm, std::uint64_t planes, cudaStream_t s) const;
    void inverse_dense(const void* wvm, void* real, std::uint64_t planes, cudaStream_t s) const;
    void gather_dense(const void* wvm, std::uint64_t planes, const ViewSet& views, double scale,
                      cudaStream_t s) const;
    // Column stages against caller-owned bin arrays (kxStride = keep()).
    // zStride: bin planes per view (0 = Nz); values above Nz need the FP32 warp kernels.
    void inverse_columns_into(const ViewSet& views, DenseBins out, cudaStream_t s, int zStride = 0) const;
    void forward_columns_from(DenseBins in, const ViewSet& views, double scale, cudaStream_t s,
                              int zStride = 0) const;
    // Band form of the column stages (fused flux), in place on dense bins
    // whose slot f starts at plane f * zStride: valid when band_exact(), i.e.
    // the retained cells of every column (with the kx = 0 partners) are the
    // band min(ky, Ny - ky) <= band[kx].  FP32 only.
    bool band_exact() const { return bandExact_; }
    void inverse_columns_band(DenseBins bins, int slots, int zStride, cudaStream_t s) const;
    void forward_columns_band(DenseBins bins, int slots, double scale, int zStride, cudaStream_t s) const;
    // Kernel form of each band stage (kBandDefault / kBandWarp, columns_warp.hpp).
    void set_band_forms(int inverseForm, int forwardForm) {
        bandFormInverse_ = inverseForm;
        bandFormForward_ = forwardForm;
    }
    int band_form_inverse() const { return bandFormInverse_; }
    int band_form_forward() const { return bandFormForward_; }
    const void* twiddlesHalf() const { return twHalf_.get(); }
    const void* twiddlesFull() const { return twFull_.get(); }
    void embed_dense(const ViewSet& views, void* wvm, std::uint64_t planes, cudaStream_t s) const;

    double allocationSeconds = 0.0, planningSeconds = 0.0;
    std::uint64_t persistentBytes = 0, scratchBytes = 0;

private:
    Workload w_;
    Precision p_;
    int keep_ = 0;
    std::uint64_t maxPlanes_ = 0;
    std::uint64_t modeCount_ = 0;
    DeviceBuffer twHalf_, twFull_, twCol_;
    DeviceBuffer cellMap_, gatherMap_, colStart_, colKy_, colMode_, modeKx_, modeKy_, modeConj_;
    DeviceBuffer bins_;
    DeviceBuffer band_;
    bool bandExact_ = false;
    int bandFormInverse_ = 0, bandFormForward_ = 0;
};

// Vertical plan for one direction: the group matrices prepared for the chosen
// GEMM form and the tile / work-unit tables of every group and member.
class VerticalPlan {
public:
    // rowsOut x inner matrices per group, natural layout A[g][r][s]
    // (forward: F[g][j][z], inverse: I[g][z][j]); one matrix for all groups
    // when `natural` holds a single rowsOut x inner block.
    VerticalPlan(GemmPrecision p, int rowsOut, int inner, const std::vector<ModeGroup>& groups,
                 std::uint64_t fields, std::uint64_t members, const std::vector<double>& natural);
    // `members` <= the capacity given at construction (0 = all): the first
    // `members` ensemble members are computed.
    // inBins / outBins (tensor-core form only): operands in the fused flux's
    // dense bin array instead of compact [column][len] arrays.
    void execute(ComplexOperand in, ComplexOperand out, cudaStream_t s, std::uint64_t members = 0,
                 const BinBoundary* inBins = nullptr, const BinBoundary* outBins = nullptr) const;
    // Raises if a bounded device wait of the tensor-core form expired.
    void check_device_error() const;
    // Tensor-core form: the next launches wait on a device barrier that
    // nothing signals, so their bounded wait expires (tests the error path).
    void set_expire_wait_for_test(bool on) { expireWaitForTest_ = on; }
    GemmPrecision precision() const { return p_; }
    // The split TF32x3 and BF16x3 forms run on the tcgen05 tensor cores.
    bool tensor_core() const { return p_ == GemmPrecision::tf32x3 || p_ == GemmPrecision::bf16x3; }
    std::uint64_t columns() const { return columns_; }
    std::uint64_t matrixBytes() const { return matrices_.bytes(); }
    std::uint64_t persistentBytes() const;
    int launches() const { return 1; }
    // Tensor-core form: M-tiles (64 columns) per work unit; the unit tables are
    // rebuilt for a new size (device work must not be in flight on them).
    void set_unit_tiles(int tiles);
    int unit_tiles() const { return unitTiles_; }
    int rows_out() const { return R_; }
    int inner() const { return S_; }
    std::uint64_t groups() const { return groupColumnsHost_.size(); }

private:
    void build_units(int tiles);
    GemmPrecision p_;
    int R_, S_;
    std::uint64_t columns_ = 0;
    std::uint64_t members_ = 1;
    long long memberColumns_ = 0;
    long long matrixStride_ = 0;  // SIMT form: elements between group matrices (0: one common matrix)
    DeviceBuffer matrices_;
    // SIMT tiles: one member-major table whose first tilePrefix_[m - 1] tiles
    // cover m members, or (virtual numbering) one table per member count.
    struct TileTable {
        DeviceBuffer group, column, count, per, first;
        int tiles = 0;
    };
    std::vector<TileTable> tileTables_;
    std::vector<int> tilePrefix_;  // tiles launched for 1..members members
    bool virtualTiles_ = false;    // SIMT tile numbering (GroupTiles::virtualColumns)
    long long imageStride_ = 0;  // tensor-core form: bytes between group images (0: one common image)
    // Tensor-core work units, one table per active member count 1..members.
    struct UnitTable {
        DeviceBuffer group, column, count, first;  // first: per-CTA unit ranges (ctas + 1 entries)
        int units = 0, ctas = 0;
    };
    std::vector<UnitTable> unitTables_;
    std::vector<int> groupColumnsHost_;  // complex columns per member in each group
    int unitTiles_ = 0;
    DeviceBuffer groupColumns_, groupFirst_, error_;
    bool expireWaitForTest_ = false;
};

}  // namespace skb
