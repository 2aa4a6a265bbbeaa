// The spectral-pipeline round trip: pruned r2c with retention, K^2 vertical
// forward, synthetic modal work, vertical inverse, embedding and c2r, in the
// order of runSpectralPipelineBenchmark's reference computation
// (benchmark.cpp:3072-3110).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace skb {

struct PipelineStage {
    std::string name;
    double ms = 0.0, bytes = 0.0;
    std::uint64_t launches = 0;
};

class SpectralPipeline {
public:
    // FP64: FP64 transforms and SIMT FP64 GEMMs (the plain drop-in).
    // FP32: FP32 transforms and split-TF32x3 tensor-core GEMMs.
    SpectralPipeline(const Workload& w, Precision p);
    ~SpectralPipeline();
    SpectralPipeline(const SpectralPipeline&) = delete;
    SpectralPipeline& operator=(const SpectralPipeline&) = delete;

    // Real [field][z][y][x] in and out (unnormalised c2r), device arrays of the
    // handle's precision.
    void execute(const void* realIn, void* realOut, cudaStream_t s) const;
    std::vector<PipelineStage> profile(const void* realIn, void* realOut, cudaStream_t s) const;
    void check_device_error() const;
    const Workload& workload() const { return w_; }
    Precision precision() const { return p_; }

    double allocationSeconds = 0.0, planningSeconds = 0.0;
    std::uint64_t persistentBytes = 0, scratchBytes = 0;

private:
    struct Marks;
    void run(const void* realIn, void* realOut, cudaStream_t s, Marks* marks) const;
    Workload w_;
    Precision p_;
    std::uint64_t modes_ = 0, nj_ = 0;
    std::unique_ptr<HorizontalPlan> horizontal_;
    std::unique_ptr<VerticalPlan> forward_, inverse_;
    DeviceBuffer retained_, modal_, weights_;
};

// syntheticModalWorkWeights (model.cpp:246-267), [mode][field][j].
std::vector<double> synthetic_modal_weights(const Workload& w, const std::vector<RetainedMode>& modes);

// out[i] = weights[i] * in[i] for `count` complex values (in place allowed).
cudaError_t launch_modal_work(Precision p, const void* weights, const void* in, void* out, long long count,
                              cudaStream_t s);

}  // namespace skb
