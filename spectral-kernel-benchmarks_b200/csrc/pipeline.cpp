#include "pipeline.hpp"

#include <algorithm>
#include <chrono>

namespace skb {

std::vector<double> synthetic_modal_weights(const Workload& w, const std::vector<RetainedMode>& modes) {
    const std::uint64_t nj = w.nj();
    std::vector<double> out(modes.size() * w.fields * nj);
    // |value|, written so that the most negative value cannot overflow.
    auto magnitude = [](std::int64_t v) {
        return v < 0 ? static_cast<std::uint64_t>(-(v + 1)) + 1 : static_cast<std::uint64_t>(v);
    };
    for (std::size_t m = 0; m < modes.size(); ++m) {
        const std::uint64_t k = magnitude(modes[m].k), l = magnitude(modes[m].l);
        for (std::uint64_t f = 0; f < w.fields; ++f)
            for (std::uint64_t j = 0; j < nj; ++j) {
                const std::uint64_t key = (17 * k + 29 * l + 7 * j + 11 * f) % 97;
                out[(m * w.fields + f) * nj + j] = 0.75 + 0.5 * static_cast<double>(key) / 96.0;
            }
    }
    return out;
}

SpectralPipeline::SpectralPipeline(const Workload& w, Precision p) : w_(w), p_(p) {
    validate_workload(w);
    using Clock = std::chrono::steady_clock;
    const auto t0 = Clock::now();
    const auto modes = retained_modes(w);
    const auto groups = squared_wavenumber_groups(modes);
    modes_ = modes.size();
    nj_ = w.nj();
    if (nj_ == 0) throw Error(-1, "spectral pipeline requires Nz >= 2");
    const VerticalFamily fam = k2_rotation_family(w, groups);
    const auto weights = synthetic_modal_weights(w, modes);
    planningSeconds = std::chrono::duration<double>(Clock::now() - t0).count();
    const auto t1 = Clock::now();
    horizontal_ = std::make_unique<HorizontalPlan>(w, p, true, w.planes());
    const GemmPrecision gp = p == Precision::f64 ? GemmPrecision::f64 : GemmPrecision::tf32x3;
    forward_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(nj_), static_cast<int>(w.nz), groups, w.fields, 1,
                                              fam.forward);
    inverse_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(w.nz), static_cast<int>(nj_), groups, w.fields, 1,
                                              fam.inverse);
    const size_t es = element_bytes(p);
    retained_.allocate(2 * es * modes_ * w.planes());
    modal_.allocate(2 * es * modes_ * w.fields * nj_);
    weights_ = upload_real_table(weights, p);
    allocationSeconds = std::chrono::duration<double>(Clock::now() - t1).count() + horizontal_->allocationSeconds;
    planningSeconds += horizontal_->planningSeconds;
    persistentBytes = horizontal_->persistentBytes + forward_->persistentBytes() + inverse_->persistentBytes() +
                      weights_.bytes();
    scratchBytes = horizontal_->scratchBytes + retained_.bytes() + modal_.bytes();
}

SpectralPipeline::~SpectralPipeline() = default;

struct SpectralPipeline::Marks {
    cudaStream_t s;
    std::vector<cudaEvent_t> events;
    std::vector<PipelineStage> stages;
    explicit Marks(cudaStream_t stream) : s(stream) { mark(); }
    ~Marks() {
        for (auto e : events) cudaEventDestroy(e);
    }
    void mark() {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        check_cuda(cudaEventRecord(e, s), "cudaEventRecord");
        events.push_back(e);
    }
    void end(const char* name, double bytes, std::uint64_t launches) {
        stages.push_back({name, 0.0, bytes, launches});
        mark();
    }
};

void SpectralPipeline::run(const void* realIn, void* realOut, cudaStream_t s, Marks* marks) const {
    const std::uint64_t fields = w_.fields, nz = w_.nz, planes = w_.planes();
    const size_t es = element_bytes(p_), ces = 2 * es;
    ViewSet views{};
    views.count = static_cast<int>(fields);
    for (std::uint64_t f = 0; f < fields; ++f)
        views.v[f] = {static_cast<unsigned char*>(retained_.get()) + ces * f * nz, nullptr,
                      static_cast<long long>(planes)};
    const double realBytes = double(planes) * w_.nx * w_.ny * es, retBytes = double(modes_) * planes * ces;
    const double modalBytes = double(modes_) * fields * nj_ * ces;
    horizontal_->forward(realIn, planes, views, 1.0, s);
    if (marks) marks->end("pruned_forward", realBytes + retBytes, 2);
    forward_->execute({retained_.get(), nullptr}, {modal_.get(), nullptr}, s);
    if (marks) marks->end("vertical_forward", retBytes + modalBytes + double(forward_->matrixBytes()), 1);
    check_cuda(launch_modal_work(p_, weights_.get(), modal_.get(), modal_.get(),
                                 static_cast<long long>(modes_ * fields * nj_), s),
               "modal work kernel");
    if (marks) marks->end("modal_work", 2 * modalBytes + double(modes_) * fields * nj_ * es, 1);
    inverse_->execute({modal_.get(), nullptr}, {retained_.get(), nullptr}, s);
    if (marks) marks->end("vertical_inverse", retBytes + modalBytes + double(inverse_->matrixBytes()), 1);
    horizontal_->inverse(views, realOut, s);
    if (marks) marks->end("pruned_inverse", realBytes + retBytes, 2);
}

void SpectralPipeline::execute(const void* realIn, void* realOut, cudaStream_t s) const {
    run(realIn, realOut, s, nullptr);
}

std::vector<PipelineStage> SpectralPipeline::profile(const void* realIn, void* realOut, cudaStream_t s) const {
    Marks marks(s);
    run(realIn, realOut, s, &marks);
    check_cuda(cudaEventSynchronize(marks.events.back()), "cudaEventSynchronize");
    for (size_t i = 0; i < marks.stages.size(); ++i) {
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, marks.events[i], marks.events[i + 1]), "cudaEventElapsedTime");
        marks.stages[i].ms = ms;
    }
    return marks.stages;
}

void SpectralPipeline::check_device_error() const {
    forward_->check_device_error();
    inverse_->check_device_error();
}

}  // namespace skb
