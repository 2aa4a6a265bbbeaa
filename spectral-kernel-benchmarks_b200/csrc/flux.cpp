#include "flux.hpp"

#include "pointwise.hpp"

namespace skb {

FluxPipeline::FluxPipeline(const FluxConfig& cfg) : cfg_(cfg) {
    if (cfg.n < 2 || cfg.nz < 2) throw Error(-1, "flux requires n >= 2 and Nz >= 2");
    if (cfg.targets != 4 && cfg.targets != 3) throw Error(-1, "flux targets must be 4 (15 -> 4) or 3 (12 -> 3)");
    if (cfg.members == 0) throw Error(-1, "flux requires at least one ensemble member");
    if (3 * cfg.members > static_cast<std::uint64_t>(kMaxViews))
        throw Error(-1, "at most " + std::to_string(kMaxViews / 3) + " ensemble members per flux handle");
    if (cfg.mode == FluxMode::split_tf32x3 || cfg.mode == FluxMode::split_bf16x3)
        throw Error(-2, "unsupported: split tensor-core flux mode is not built in this library");
    const auto planStart = Clock::now();
    wOut_ = Workload{cfg.n, cfg.n, cfg.nz, cfg.targets, 1.0, 1.0, true};
    fieldsIn_ = 3 + 3 * cfg.targets;
    const auto modes = retained_modes(wOut_);
    const auto groups = squared_wavenumber_groups(modes);
    modes_ = modes.size();
    nj_ = wOut_.nj();
    volume_ = cfg.n * cfg.n * cfg.nz;
    VerticalFamily fam = cfg.family == 2 ? sturm_liouville_family(wOut_, groups, cfg.familySeed)
                                         : k2_rotation_family(wOut_, groups);
    familyId = fam.id;
    const auto fwdT = transpose_family(fam, true);
    const auto invT = transpose_family(fam, false);
    planningSeconds = seconds_since(planStart);

    const auto allocStart = Clock::now();
    const Precision hp = f64() ? Precision::f64 : Precision::f32;
    const GemmPrecision gp = f64() ? GemmPrecision::f64 : GemmPrecision::f32;
    const size_t es = element_bytes(hp);
    // Admission by device memory: refuse before allocating what cannot fit.
    const std::uint64_t maxPlanes = 3 * cfg.members * cfg.nz;
    std::uint64_t need = 2 * es * cfg.members * modes_ * cfg.nz * (fieldsIn_ + cfg.targets)  // physIn, physOut
                         + es * volume_ * cfg.members * 7                                   // 3+3+1 volumes
                         + 2 * es * cfg.n * (cfg.n / 2 + 1) * maxPlanes;                    // bin scratch bound
    size_t freeBytes = 0, totalBytes = 0;
    check_cuda(cudaMemGetInfo(&freeBytes, &totalBytes), "cudaMemGetInfo");
    if (need > freeBytes)
        throw Error(-4, "flux workload needs " + std::to_string(need) + " device bytes; " +
                            std::to_string(freeBytes) + " are free");
    horizontal_ = std::make_unique<HorizontalPlan>(Workload{cfg.n, cfg.n, cfg.nz, 3, 1.0, 1.0, true}, hp, true,
                                                   maxPlanes);
    inverseGemm_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(cfg.nz), static_cast<int>(nj_), groups,
                                                  fieldsIn_, cfg.members, invT);
    forwardGemm_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(nj_), static_cast<int>(cfg.nz), groups,
                                                  cfg.targets, cfg.members, fwdT);
    physIn_.allocate(2 * es * cfg.members * modes_ * fieldsIn_ * cfg.nz);
    physOut_.allocate(2 * es * cfg.members * modes_ * cfg.targets * cfg.nz);
    shared_.allocate(es * 3 * cfg.members * volume_);
    deriv_.allocate(es * 3 * cfg.members * volume_);
    target_.allocate(es * cfg.members * volume_);
    allocationSeconds = seconds_since(allocStart) + horizontal_->allocationSeconds;
    planningSeconds += horizontal_->planningSeconds;
    persistentBytes = horizontal_->persistentBytes + inverseGemm_->persistentBytes() + forwardGemm_->persistentBytes();
    scratchBytes = horizontal_->scratchBytes + physIn_.bytes() + physOut_.bytes() + shared_.bytes() +
                   deriv_.bytes() + target_.bytes();
    // 2 GEMMs, 2 launches per inverse / forward horizontal, members pointwise per target.
    launches_ = 2 + 2 + cfg.targets * (2 + cfg.members + 2);
}

FluxPipeline::~FluxPipeline() {
    if (graphExec_ != nullptr) cudaGraphExecDestroy(graphExec_);
    if (graph_ != nullptr) cudaGraphDestroy(graph_);
}

void FluxPipeline::execute(const void* modalIn, void* modalOut, cudaStream_t s) {
    const auto H = modes_, nz = cfg_.nz, T = cfg_.targets, M = cfg_.members;
    const size_t ces = 2 * element_bytes(horizontal_->precision());  // complex element bytes
    auto* physIn = physIn_.get<unsigned char>();
    auto* physOut = physOut_.get<unsigned char>();
    inverseGemm_->execute({const_cast<void*>(modalIn), nullptr}, {physIn_.get(), nullptr}, s);

    auto triple = [&](std::uint64_t firstField) {
        ViewSet v{};
        v.count = static_cast<int>(3 * M);
        for (std::uint64_t m = 0; m < M; ++m)
            for (std::uint64_t f = 0; f < 3; ++f)
                v.v[3 * m + f] = {physIn + ces * ((m * H * fieldsIn_ + firstField + f) * nz), nullptr,
                                  static_cast<long long>(fieldsIn_ * nz)};
        return v;
    };
    horizontal_->inverse(triple(0), shared_.get(), s);
    const double scale = 1.0 / (static_cast<double>(cfg_.n * cfg_.n) * static_cast<double>(cfg_.n * cfg_.n));
    const size_t es = element_bytes(horizontal_->precision());
    const int sms = sm_count();
    for (std::uint64_t t = 0; t < T; ++t) {
        horizontal_->inverse(triple(3 + 3 * t), deriv_.get(), s);
        for (std::uint64_t m = 0; m < M; ++m) {
            check_cuda(launch_pointwise(f64(), static_cast<long long>(volume_), scale,
                                        shared_.get<unsigned char>() + es * 3 * m * volume_,
                                        deriv_.get<unsigned char>() + es * 3 * m * volume_,
                                        target_.get<unsigned char>() + es * m * volume_, sms, s),
                       "pointwise advection kernel");
        }
        ViewSet out{};
        out.count = static_cast<int>(M);
        for (std::uint64_t m = 0; m < M; ++m)
            out.v[m] = {physOut + ces * ((m * H * T + t) * nz), nullptr, static_cast<long long>(T * nz)};
        horizontal_->forward(target_.get(), M * nz, out, 1.0, s);
    }
    forwardGemm_->execute({physOut_.get(), nullptr}, {modalOut, nullptr}, s);
}

void FluxPipeline::capture(const void* modalIn, void* modalOut, cudaStream_t s) {
    if (graphExec_ != nullptr) {
        cudaGraphExecDestroy(graphExec_);
        graphExec_ = nullptr;
    }
    if (graph_ != nullptr) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        execute(modalIn, modalOut, s);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g != nullptr) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(s, &graph_), "cudaStreamEndCapture");
    check_cuda(cudaGraphInstantiate(&graphExec_, graph_, 0), "cudaGraphInstantiate");
}

void FluxPipeline::replay(cudaStream_t s) {
    if (graphExec_ == nullptr) throw Error(-3, "no captured flux graph to replay");
    check_cuda(cudaGraphLaunch(graphExec_, s), "cudaGraphLaunch");
}

}  // namespace skb
