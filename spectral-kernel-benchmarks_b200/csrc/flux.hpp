// The composed 15 -> 4 (or 12 -> 3) antialiased flux on the device.
//
// Order and normalisation follow runProductionLifetimeFluxBenchmark's
// streamed graph (src/benchmark.cpp:4328-4424): inverse vertical GEMM of all
// input fields, inverse pruned horizontal of [U,V,W] once, then per target the
// inverse of its derivative triple, the pointwise product
// -1/(Nx*Ny)^2 (u qx + v qy + w qz), the forward pruned horizontal with
// retention, and finally the forward vertical GEMM of the targets.  Input slot
// map (benchmark.cpp:4138): slots 0..2 are [U,V,W]; slots 3+3t..5+3t are
// [q_t,x, q_t,y, q_t,z].  Ensemble members are independent and batched into
// every launch.

#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "autotune.hpp"
#include "flux_rows.hpp"
#include "runtime.hpp"

namespace skb {

enum class FluxMode { fp64_plain = 0, fp32 = 1, split_tf32x3 = 2, split_bf16x3 = 3 };

// Externally supplied vertical operators (the authoritative WVM path,
// src/authoritative_spectral_flux.cpp and src/spectral_flux_fixture.cpp of
// the reference): two families (wave-f = 0, wave-g = 1) over explicit operator
// groups, and the family each input slot and each target uses.
struct FluxFamilies {
    std::vector<ModeGroup> groups;               // contiguous runs of the retained modes, in order
    std::array<std::vector<double>, 2> forward;  // family: [group][j][z]
    std::array<std::vector<double>, 2> inverse;  // family: [group][z][j]
    std::vector<int> inputFamily;                // per input slot: 0 or 1
    std::vector<int> targetFamily;               // per target: 0 or 1
};

struct FluxConfig {
    std::uint64_t n = 0, nz = 0, targets = 4, members = 1;
    FluxMode mode = FluxMode::fp64_plain;
    int family = 1;  // SKB_FAMILY_K2_ROTATION or SKB_FAMILY_STURM_LIOUVILLE
    std::uint64_t familySeed = 0;
    std::shared_ptr<const FluxFamilies> families;  // overrides `family` when set
};

class FluxPipeline {
public:
    explicit FluxPipeline(const FluxConfig& cfg);
    ~FluxPipeline();

    // Device arrays of the pipeline's I/O precision (double for fp64_plain,
    // float otherwise): modal input [member][mode][3+3T][j], output
    // [member][mode][T][j].
    void execute(const void* modalIn, void* modalOut, cudaStream_t s);
    // The first `members` (<= capacity) ensemble members only, for partial batches.
    void execute(const void* modalIn, void* modalOut, cudaStream_t s, std::uint64_t members);

    // One evaluation with CUDA events between stages; per stage the summed
    // device milliseconds, launches and algorithmic bytes / flops.
    struct StageTime {
        std::string name;
        double ms = 0.0;
        std::uint64_t launches = 0;
        double bytes = 0.0, flops = 0.0;
    };
    std::vector<StageTime> profile(const void* modalIn, void* modalOut, cudaStream_t s);
    void capture(const void* modalIn, void* modalOut, cudaStream_t s);
    // Project autotuner: measures every missing launch-shape choice of the
    // fused path on these buffers (the input is read; the output receives the
    // flux), applies and caches them (autotune.hpp), and drops any captured
    // graph (capture again after tuning).  Cached choices are already applied
    // when a pipeline is created.  Returns the choices in force.
    std::vector<TuneEntry> autotune(const void* modalIn, void* modalOut, cudaStream_t s);
    double tunedSeconds = 0.0;
    // Raises if a bounded device wait inside a tensor-core kernel expired.
    void check_device_errors() const;
    // Failure-path test of the row kernel's TMA forms (RowFluxArgs::expireWaitForTest).
    void set_rows_expire_wait_for_test(bool enable) { rowsExpireWaitForTest_ = enable; }
    void replay(cudaStream_t s);

    std::uint64_t modes() const { return modes_; }
    std::uint64_t nj() const { return nj_; }
    std::uint64_t fieldsIn() const { return fieldsIn_; }
    std::uint64_t inputElements() const { return cfg_.members * modes_ * fieldsIn_ * nj_; }
    std::uint64_t outputElements() const { return cfg_.members * modes_ * cfg_.targets * nj_; }
    bool f64() const { return cfg_.mode == FluxMode::fp64_plain; }
    const FluxConfig& config() const { return cfg_; }
    std::uint64_t launchesPerExecution() const { return launches_; }

    double allocationSeconds = 0.0, planningSeconds = 0.0;
    std::uint64_t persistentBytes = 0, scratchBytes = 0;
    std::string familyId;

private:
    FluxConfig cfg_;
    Workload wOut_;
    std::uint64_t modes_ = 0, nj_ = 0, fieldsIn_ = 0, volume_ = 0;
    std::unique_ptr<HorizontalPlan> horizontal_;
    std::unique_ptr<VerticalPlan> inverseGemm_, forwardGemm_;
    DeviceBuffer physIn_, shared_, deriv_, target_, physOut_;
    // Fused split-precision path: column-transformed bins of every input slot
    // and of every target.
    bool fused_ = false;
    std::uint64_t zStride_ = 0;  // bin planes per slot (Nz padded to a multiple of 8)
    DeviceBuffer binsIn_, binsOut_;
    // Dense boundary: the GEMMs read / write the retained values at their
    // cells of the bin arrays (no compact intermediate, no mode map in the
    // column kernels).  Per mode: cell offsets in binsIn_ (with the kx = 0
    // partner) and in binsOut_, and the conjugation flag.
    bool dense_ = false;
    DeviceBuffer cellIn_, partnerIn_, cellOut_, modeConj_;
    std::uint64_t launches_ = 0;
    struct Recorder;
    void runFused(const void* modalIn, void* modalOut, cudaStream_t s, Recorder* rec, std::uint64_t members);
    std::vector<TuneEntry> apply_tuned(const void* modalIn, void* modalOut, cudaStream_t s, double* seconds);
    RowFluxArgs row_args(std::uint64_t members) const;
    // The vertical GEMMs of both directions: one plan, or with external
    // families one plan per family over that family's fields.  `dense`:
    // the bin arrays of the fused path, else the compact physical buffers.
    void gemm_inverse(const void* modalIn, cudaStream_t s, std::uint64_t members, bool dense);
    void gemm_forward(void* modalOut, cudaStream_t s, std::uint64_t members, bool dense);
    struct FamilyPlan {
        std::unique_ptr<VerticalPlan> plan;
        DeviceBuffer fieldMap;  // plan field -> input slot or target
        int fields = 0;
    };
    std::vector<const VerticalPlan*> gemm_plans() const;
    double matrix_bytes(bool inverse) const;
    bool families_ = false;
    std::array<FamilyPlan, 2> inverseFamily_, forwardFamily_;
    // Per mode: element offset of (member 0, field 0) in the compact arrays.
    DeviceBuffer cellModalIn_, cellModalOut_, cellPhysIn_, cellPhysOut_;
    int rowsPlanes_ = 8;  // z-planes per CTA of the fused row kernel
    int rowsPairs_ = 0;   // 512-point rows: two planes per warp (RowFluxArgs::pairs)
    int rowsTma_ = 0;     // two-planes-per-warp rows: stages filled by TMA tensor copies (RowFluxArgs::tma)
    bool rowsExpireWaitForTest_ = false;  // RowFluxArgs::expireWaitForTest
    DeviceBuffer rowsError_;  // set by the fused row kernel when a bounded wait expires
    void run(const void* modalIn, void* modalOut, cudaStream_t s, Recorder* rec, std::uint64_t members);
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graphExec_ = nullptr;
};

}  // namespace skb
