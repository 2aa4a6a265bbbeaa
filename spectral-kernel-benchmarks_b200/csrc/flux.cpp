#include "flux.hpp"

#include <chrono>
#include <functional>

#include "autotune.hpp"
#include "columns_warp.hpp"
#include "flux_rows.hpp"
#include "pointwise.hpp"

namespace skb {

FluxPipeline::FluxPipeline(const FluxConfig& cfg) : cfg_(cfg) {
    if (cfg.n < 2 || cfg.nz < 2) throw Error(-1, "flux requires n >= 2 and Nz >= 2");
    if (cfg.targets != 4 && cfg.targets != 3) throw Error(-1, "flux targets must be 4 (15 -> 4) or 3 (12 -> 3)");
    if (cfg.members == 0) throw Error(-1, "flux requires at least one ensemble member");
    if (3 * cfg.members > static_cast<std::uint64_t>(kMaxViews))
        throw Error(-1, "at most " + std::to_string(kMaxViews / 3) + " ensemble members per flux handle");
    const auto planStart = Clock::now();
    wOut_ = Workload{cfg.n, cfg.n, cfg.nz, cfg.targets, 1.0, 1.0, true};
    fieldsIn_ = 3 + 3 * cfg.targets;
    const auto modes = retained_modes(wOut_);
    modes_ = modes.size();
    nj_ = wOut_.nj();
    volume_ = cfg.n * cfg.n * cfg.nz;
    families_ = cfg.families != nullptr;
    const auto groups = families_ ? cfg.families->groups : squared_wavenumber_groups(modes);
    VerticalFamily fam;
    if (families_) {
        const FluxFamilies& F = *cfg.families;
        if (cfg.targets != 4) throw Error(-1, "operator families are defined for the 15 -> 4 flux");
        std::uint64_t next = 0;
        for (const auto& g : groups) {
            if (g.first != next || g.count == 0) throw Error(-1, "operator groups must be contiguous runs of modes");
            next += g.count;
        }
        if (next != modes_) throw Error(-1, "operator groups must cover every retained mode");
        const std::uint64_t matrix = groups.size() * nj_ * cfg.nz;
        for (int f = 0; f < 2; ++f)
            if (F.forward[f].size() != matrix || F.inverse[f].size() != matrix)
                throw Error(-1, "operator family matrices must be groups x Nj x Nz");
        if (F.inputFamily.size() != fieldsIn_ || F.targetFamily.size() != cfg.targets)
            throw Error(-1, "the family map needs one entry per input slot and per target");
        for (const int v : F.inputFamily)
            if (v != 0 && v != 1) throw Error(-1, "family indices must be 0 (wave-f) or 1 (wave-g)");
        for (const int v : F.targetFamily)
            if (v != 0 && v != 1) throw Error(-1, "family indices must be 0 (wave-f) or 1 (wave-g)");
        familyId = "external wave-f + wave-g operator families";
    } else {
        fam = cfg.family == 2 ? sturm_liouville_family(wOut_, groups, cfg.familySeed)
                              : k2_rotation_family(wOut_, groups);
        familyId = fam.id;
    }
    planningSeconds = seconds_since(planStart);

    const auto allocStart = Clock::now();
    const Precision hp = f64() ? Precision::f64 : Precision::f32;
    const bool split = cfg.mode == FluxMode::split_tf32x3 || cfg.mode == FluxMode::split_bf16x3;
    const GemmPrecision gp = f64()                                ? GemmPrecision::f64
                             : cfg.mode == FluxMode::split_tf32x3 ? GemmPrecision::tf32x3
                             : cfg.mode == FluxMode::split_bf16x3 ? GemmPrecision::bf16x3
                                                                  : GemmPrecision::f32;
    const size_t es = element_bytes(hp);
    fused_ = split && rows_flux_supported(static_cast<long long>(cfg.n));
    // Admission by device memory: refuse before allocating what cannot fit.
    const std::uint64_t maxPlanes = fused_ ? 1 : 3 * cfg.members * cfg.nz;
    const std::uint64_t binPlanes = fused_ ? cfg.members * cfg.nz * (fieldsIn_ + cfg.targets) : maxPlanes;
    std::uint64_t need = 2 * es * cfg.members * modes_ * cfg.nz * (fieldsIn_ + cfg.targets)  // physIn, physOut
                         + (fused_ ? 0 : es * volume_ * cfg.members * 7)                   // 3+3+1 volumes
                         + 2 * es * cfg.n * (cfg.n / 2 + 1) * binPlanes * 9 / 8;           // bin scratch bound
    size_t freeBytes = 0, totalBytes = 0;
    check_cuda(cudaMemGetInfo(&freeBytes, &totalBytes), "cudaMemGetInfo");
    if (need > freeBytes)
        throw Error(-4, "flux workload needs " + std::to_string(need) + " device bytes; " +
                            std::to_string(freeBytes) + " are free");
    horizontal_ = std::make_unique<HorizontalPlan>(Workload{cfg.n, cfg.n, cfg.nz, 3, 1.0, 1.0, true}, hp, true,
                                                   maxPlanes);
    if (!families_) {
        inverseGemm_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(cfg.nz), static_cast<int>(nj_), groups,
                                                      fieldsIn_, cfg.members, fam.inverse);
        forwardGemm_ = std::make_unique<VerticalPlan>(gp, static_cast<int>(nj_), static_cast<int>(cfg.nz), groups,
                                                      cfg.targets, cfg.members, fam.forward);
    } else {
        const FluxFamilies& F = *cfg.families;
        for (int f = 0; f < 2; ++f) {
            std::vector<int> in, out;
            for (std::uint64_t i = 0; i < fieldsIn_; ++i)
                if (F.inputFamily[i] == f) in.push_back(static_cast<int>(i));
            for (std::uint64_t t = 0; t < cfg.targets; ++t)
                if (F.targetFamily[t] == f) out.push_back(static_cast<int>(t));
            if (!in.empty()) {
                inverseFamily_[f].plan = std::make_unique<VerticalPlan>(
                    gp, static_cast<int>(cfg.nz), static_cast<int>(nj_), groups, in.size(), cfg.members, F.inverse[f]);
                inverseFamily_[f].fieldMap = upload_vector(in);
                inverseFamily_[f].fields = static_cast<int>(in.size());
            }
            if (!out.empty()) {
                forwardFamily_[f].plan = std::make_unique<VerticalPlan>(
                    gp, static_cast<int>(nj_), static_cast<int>(cfg.nz), groups, out.size(), cfg.members, F.forward[f]);
                forwardFamily_[f].fieldMap = upload_vector(out);
                forwardFamily_[f].fields = static_cast<int>(out.size());
            }
        }
        std::vector<long long> mi(modes_), mo(modes_), pi(modes_), po(modes_);
        for (std::uint64_t m = 0; m < modes_; ++m) {
            mi[m] = static_cast<long long>(m * fieldsIn_ * nj_);
            mo[m] = static_cast<long long>(m * cfg.targets * nj_);
            pi[m] = static_cast<long long>(m * fieldsIn_ * cfg.nz);
            po[m] = static_cast<long long>(m * cfg.targets * cfg.nz);
        }
        cellModalIn_ = upload_vector(mi);
        cellModalOut_ = upload_vector(mo);
        cellPhysIn_ = upload_vector(pi);
        cellPhysOut_ = upload_vector(po);
    }
    dense_ = fused_ && horizontal_->band_exact();
    if (!dense_) {
        physIn_.allocate(2 * es * cfg.members * modes_ * fieldsIn_ * cfg.nz);
        physOut_.allocate(2 * es * cfg.members * modes_ * cfg.targets * cfg.nz);
    }
    if (fused_) {
        // Bin planes per slot padded to a multiple of 8 (64 bytes of FP32
        // complex), so every 8-plane run a column or row CTA moves starts on a
        // 64-byte boundary.
        zStride_ = (cfg.nz + 7) / 8 * 8;
        const std::uint64_t keep = static_cast<std::uint64_t>(horizontal_->keep());
        binsIn_.allocate(2 * es * cfg.n * keep * cfg.members * fieldsIn_ * zStride_);
        binsOut_.allocate(2 * es * cfg.n * keep * cfg.members * cfg.targets * zStride_);
        rowsError_.allocate(sizeof(int));
        check_cuda(cudaMemset(rowsError_.get(), 0, sizeof(int)), "cudaMemset");
        if (dense_) {
            const long long inStored = static_cast<long long>(cfg.members * fieldsIn_ * zStride_);
            const long long outStored = static_cast<long long>(cfg.members * cfg.targets * zStride_);
            std::vector<long long> cellIn(modes_), partnerIn(modes_), cellOut(modes_);
            std::vector<unsigned char> conj(modes_);
            for (std::uint64_t m = 0; m < modes_; ++m) {
                const auto& md = modes[m];
                const long long cell = static_cast<long long>(md.ky * keep + md.kx);
                cellIn[m] = cell * inStored;
                cellOut[m] = cell * outStored;
                partnerIn[m] = (md.kx == 0 && md.ky != 0 && 2 * md.ky != cfg.n)
                                   ? static_cast<long long>((cfg.n - md.ky) * keep) * inStored
                                   : -1;
                conj[m] = md.conj ? 1 : 0;
            }
            cellIn_ = upload_vector(cellIn);
            partnerIn_ = upload_vector(partnerIn);
            cellOut_ = upload_vector(cellOut);
            modeConj_ = upload_vector(conj);
        }
    } else {
        shared_.allocate(es * 3 * cfg.members * volume_);
        deriv_.allocate(es * 3 * cfg.members * volume_);
        target_.allocate(es * cfg.members * volume_);
    }
    allocationSeconds = seconds_since(allocStart) + horizontal_->allocationSeconds;
    planningSeconds += horizontal_->planningSeconds;
    persistentBytes = horizontal_->persistentBytes + cellModalIn_.bytes() + cellModalOut_.bytes() +
                      cellPhysIn_.bytes() + cellPhysOut_.bytes();
    for (const VerticalPlan* g : gemm_plans()) persistentBytes += g->persistentBytes();
    scratchBytes = horizontal_->scratchBytes + physIn_.bytes() + physOut_.bytes() + shared_.bytes() +
                   deriv_.bytes() + target_.bytes() + binsIn_.bytes() + binsOut_.bytes();
    // Staged: 2 GEMMs, 2 launches per inverse / forward horizontal, members pointwise per target.
    // Fused: GEMM, embed+columns, fused rows, columns+retention, GEMM.  With
    // operator families each GEMM is one launch per family.
    launches_ = (fused_ ? 5 : 2 + 2 + cfg.targets * (2 + cfg.members + 2)) + (families_ ? 2 : 0);
    apply_tuned(nullptr, nullptr, nullptr, nullptr);
}

// Tuned launch shapes of the fused path (autotune.hpp):
//   work-unit size (M-tiles per unit) of each tensor-core GEMM, 4 / 8 / 16 / 32;
//   the 512-point row kernel's form (one plane per warp, or two planes per
//   warp with the 16 x 16 FFT) and its z-planes per CTA, 4 / 8 / 16;
//   kernel form of each 512-point band column stage, direct / warp-per-plane /
//   persistent direct.
// With buffers, missing choices are measured on them (tune_pick); without,
// only cached choices are applied.  Returns the choices in force.
std::vector<TuneEntry> FluxPipeline::apply_tuned(const void* modalIn, void* modalOut, cudaStream_t s,
                                                 double* seconds) {
    std::vector<TuneEntry> chosen;
    if (!fused_ || !dense_) return chosen;
    const auto start = std::chrono::steady_clock::now();
    const bool measure = modalIn != nullptr;
    const std::string dev = " | " + device_tag();
    const std::uint64_t M = cfg_.members, T = cfg_.targets;
    const std::string shape = " n=" + std::to_string(cfg_.n) + " nz=" + std::to_string(cfg_.nz) +
                              " targets=" + std::to_string(T) + " members=" + std::to_string(M);
    const long long keep = horizontal_->keep();
    const long long inStored = static_cast<long long>(M * fieldsIn_ * zStride_);
    const long long outStored = static_cast<long long>(M * T * zStride_);
    const DenseBins binsIn{binsIn_.get(), inStored, keep};
    const DenseBins binsOut{binsOut_.get(), outStored, keep};
    const BinBoundary gemmOut{cellIn_.get<long long>(), partnerIn_.get<long long>(), modeConj_.get<unsigned char>(),
                              static_cast<int>(fieldsIn_), static_cast<int>(zStride_)};
    const BinBoundary gemmIn{cellOut_.get<long long>(), nullptr, modeConj_.get<unsigned char>(), static_cast<int>(T),
                             static_cast<int>(zStride_)};
    auto pick = [&](const std::string& key, const std::vector<int>& candidates, const std::function<void(int)>& apply,
                    const std::function<void()>& run) {
        int value = 0;
        double ms = 0.0;
        if (measure) {
            value = tune_pick(key, candidates, [&](int c) {
                apply(c);
                run();
            }, s, 1, 3, &ms);
        } else if (!tune_lookup(key, value)) {
            return;
        }
        apply(value);
        chosen.push_back({key, value, ms});
    };
    auto unitTiles = [&](VerticalPlan& g) {
        return [&g, s](int c) {
            if (g.unit_tiles() == c) return;
            // The unit tables are replaced: no launch may still read them.
            if (s != nullptr) check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            g.set_unit_tiles(c);
        };
    };
    auto gemmKey = [&](const char* dir, const VerticalPlan& g) {
        return std::string("flux.tc_gemm.unit_tiles ") + dir + (g.precision() == GemmPrecision::bf16x3 ? " bf16x3" : "") +
               shape + " R=" + std::to_string(g.rows_out()) +
               " S=" + std::to_string(g.inner()) + " groups=" + std::to_string(g.groups()) + dev;
    };
    const std::vector<int> tileCandidates{4, 8, 16, 32};
    if (!families_) pick(gemmKey("inverse", *inverseGemm_), tileCandidates, unitTiles(*inverseGemm_), [&] {
        inverseGemm_->execute({const_cast<void*>(modalIn), nullptr}, {binsIn_.get(), nullptr}, s, M, nullptr,
                              &gemmOut);
    });
    if (!families_) pick(gemmKey("forward", *forwardGemm_), tileCandidates, unitTiles(*forwardGemm_), [&] {
        forwardGemm_->execute({binsOut_.get(), nullptr}, {modalOut, nullptr}, s, M, &gemmIn, nullptr);
    });
    if (cfg_.n == 512) {
        // Row kernel form first (two planes per warp needs 8 or 16 planes per
        // CTA), then the planes per CTA among those the form takes.
        // pairs 2: the 8-plane form compiled for three CTAs per SM (168
        // registers, a few spilled) instead of two.
        pick("flux.rows.pairs" + shape + dev, {0, 1, 2},
             [&](int c) {
                 rowsPairs_ = c;
                 if (c != 0 && rowsPlanes_ < 8) rowsPlanes_ = 8;
             },
             [&] { check_cuda(launch_rows_flux(row_args(M), s), "fused row flux kernel"); });
    }
    if (cfg_.n == 512 && rowsPairs_ != 0) {
        // Two-planes-per-warp forms: stage fills by per-thread cp.async (0) or
        // by one TMA tensor copy per slot, one (1) or two (2) slots ahead.
        pick("flux.rows.tma" + shape + dev, {0, 1, 2}, [&](int c) { rowsTma_ = c; },
             [&] { check_cuda(launch_rows_flux(row_args(M), s), "fused row flux kernel"); });
    }
    pick("flux.rows.planes_per_cta" + shape + dev, rowsPairs_ != 0 ? std::vector<int>{8, 16, 24} : std::vector<int>{4, 8, 16},
         [&](int c) { rowsPlanes_ = c; },
         [&] { check_cuda(launch_rows_flux(row_args(M), s), "fused row flux kernel"); });
    if (cfg_.n == 512) {
        // Both forms run in place on the bin arrays; repeated runs leave values
        // the final execution below overwrites.
        const std::vector<int> forms{kBandDefault,  kBandWarp,     kBandPersist,  kBandDirect4, kBand16,
                                     kBand32,       kBand16Pipe16, kBand16Pipe32, kBand16Pipe64};
        pick("flux.columns_band.form inverse" + shape + dev, forms,
             [&](int c) { horizontal_->set_band_forms(c, horizontal_->band_form_forward()); },
             [&] { horizontal_->inverse_columns_band(binsIn, static_cast<int>(M * fieldsIn_), static_cast<int>(zStride_), s); });
        pick("flux.columns_band.form forward" + shape + dev, forms,
             [&](int c) { horizontal_->set_band_forms(horizontal_->band_form_inverse(), c); },
             [&] {
                 horizontal_->forward_columns_band(binsOut, static_cast<int>(M * T), 1.0, static_cast<int>(zStride_), s);
             });
    }
    if (measure) run(modalIn, modalOut, s, nullptr, M);
    if (seconds != nullptr) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    return chosen;
}

std::vector<TuneEntry> FluxPipeline::autotune(const void* modalIn, void* modalOut, cudaStream_t s) {
    if (modalIn == nullptr || modalOut == nullptr) throw Error(-1, "autotune needs the input and output buffers");
    // A captured graph holds the old launch shapes.
    if (graphExec_ != nullptr) {
        cudaGraphExecDestroy(graphExec_);
        graphExec_ = nullptr;
    }
    if (graph_ != nullptr) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    double seconds = 0.0;
    auto chosen = apply_tuned(modalIn, modalOut, s, &seconds);
    check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    planningSeconds += seconds;
    tunedSeconds = seconds;
    return chosen;
}

FluxPipeline::~FluxPipeline() {
    if (graphExec_ != nullptr) cudaGraphExecDestroy(graphExec_);
    if (graph_ != nullptr) cudaGraphDestroy(graph_);
}

// Optional stage timing: events recorded on the stream between stages.
struct FluxPipeline::Recorder {
    cudaStream_t stream;
    std::vector<cudaEvent_t> events;
    std::vector<int> stageOf;
    std::vector<StageTime> stages;
    explicit Recorder(cudaStream_t s) : stream(s) { mark(-1); }
    ~Recorder() {
        for (auto e : events) cudaEventDestroy(e);
    }
    int stage(const std::string& name) {
        for (size_t i = 0; i < stages.size(); ++i)
            if (stages[i].name == name) return static_cast<int>(i);
        stages.push_back({name});
        return static_cast<int>(stages.size() - 1);
    }
    void mark(int stageIndex) {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        check_cuda(cudaEventRecord(e, stream), "cudaEventRecord");
        events.push_back(e);
        stageOf.push_back(stageIndex);
    }
    void end(const std::string& name, std::uint64_t launches, double bytes, double flops) {
        const int i = stage(name);
        stages[i].launches += launches;
        stages[i].bytes += bytes;
        stages[i].flops += flops;
        mark(i);
    }
    std::vector<StageTime> finish() {
        check_cuda(cudaEventSynchronize(events.back()), "cudaEventSynchronize");
        for (size_t k = 1; k < events.size(); ++k) {
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, events[k - 1], events[k]), "cudaEventElapsedTime");
            stages[stageOf[k]].ms += ms;
        }
        return stages;
    }
};

void FluxPipeline::execute(const void* modalIn, void* modalOut, cudaStream_t s) {
    run(modalIn, modalOut, s, nullptr, cfg_.members);
}

void FluxPipeline::execute(const void* modalIn, void* modalOut, cudaStream_t s, std::uint64_t members) {
    if (members == 0 || members > cfg_.members)
        throw Error(-1, "active members must be between 1 and the handle's capacity");
    run(modalIn, modalOut, s, nullptr, members);
}

std::vector<FluxPipeline::StageTime> FluxPipeline::profile(const void* modalIn, void* modalOut, cudaStream_t s) {
    Recorder rec(s);
    run(modalIn, modalOut, s, &rec, cfg_.members);
    return rec.finish();
}

RowFluxArgs FluxPipeline::row_args(std::uint64_t members) const {
    const double n = static_cast<double>(cfg_.n);
    const long long keep = horizontal_->keep();
    RowFluxArgs a{};
    a.nx = static_cast<int>(cfg_.n);
    a.ny = static_cast<int>(cfg_.n);
    a.nz = static_cast<int>(cfg_.nz);
    a.zStride = static_cast<int>(zStride_);
    a.keep = static_cast<int>(keep);
    a.members = static_cast<int>(members);
    a.fieldsIn = static_cast<int>(fieldsIn_);
    a.targets = static_cast<int>(cfg_.targets);
    a.scale = static_cast<float>(1.0 / (n * n * n * n));
    a.binsIn = {binsIn_.get(), static_cast<long long>(cfg_.members * fieldsIn_ * zStride_), keep};
    a.binsOut = {binsOut_.get(), static_cast<long long>(cfg_.members * cfg_.targets * zStride_), keep};
    a.twHalf = horizontal_->twiddlesHalf();
    a.twFull = horizontal_->twiddlesFull();
    a.planes = rowsPlanes_;
    a.pairs = rowsPairs_;
    a.tma = rowsTma_;
    a.error = static_cast<int*>(rowsError_.get());
    a.expireWaitForTest = rowsExpireWaitForTest_ ? 1 : 0;
    return a;
}

void FluxPipeline::runFused(const void* modalIn, void* modalOut, cudaStream_t s, Recorder* rec,
                            std::uint64_t members) {
    const auto H = modes_, nz = cfg_.nz, T = cfg_.targets, M = members;
    const size_t ces = 2 * sizeof(float);
    const double n = static_cast<double>(cfg_.n);
    const long long keep = horizontal_->keep();
    auto* physIn = physIn_.get<unsigned char>();
    auto* physOut = physOut_.get<unsigned char>();
    const double binsPlane = n * keep * ces, compactPlane = double(H) * ces;
    const double gemmIn = double(M) * H * fieldsIn_ * (nj_ + nz) * ces + matrix_bytes(true);
    const double gemmOut = double(M) * H * T * (nj_ + nz) * ces + matrix_bytes(false);
    const long long inPlanes = static_cast<long long>(M * fieldsIn_ * nz);
    const long long outPlanes = static_cast<long long>(M * T * nz);
    // Stored planes (stride between kx in the bin arrays) include the z-padding.
    const long long inStored = static_cast<long long>(cfg_.members * fieldsIn_ * zStride_);
    const long long outStored = static_cast<long long>(cfg_.members * T * zStride_);
    const DenseBins binsIn{binsIn_.get(), inStored, keep};
    const DenseBins binsOutArr{binsOut_.get(), outStored, keep};
    // Tensor-core products per real multiply-add: 3 (TF32 hi/lo) or 6 (BF16 h/m/l).
    const bool bf16 = cfg_.mode == FluxMode::split_bf16x3;
    const double splitTerms = bf16 ? 6.0 : 3.0;
    auto gemmStage = [bf16](bool inverse) {
        return inverse ? (bf16 ? "gemm_inverse_bf16x3" : "gemm_inverse_tf32x3")
                       : (bf16 ? "gemm_forward_bf16x3" : "gemm_forward_tf32x3");
    };
    if (dense_) {
        // GEMM -> retained cells of binsIn -> in-place inverse columns.
        gemm_inverse(modalIn, s, M, true);
        if (rec) rec->end(gemmStage(true), 1, gemmIn, splitTerms * 4.0 * nz * nj_ * double(M) * H * fieldsIn_);
        horizontal_->inverse_columns_band(binsIn, static_cast<int>(M * fieldsIn_), static_cast<int>(zStride_), s);
        if (rec) rec->end("columns_inverse_embed", 1, double(inPlanes) * (compactPlane + binsPlane), 0.0);
    } else {
        gemm_inverse(modalIn, s, M, false);
        if (rec) rec->end(gemmStage(true), 1, gemmIn, splitTerms * 4.0 * nz * nj_ * double(M) * H * fieldsIn_);
        ViewSet inViews{};
        inViews.count = static_cast<int>(M * fieldsIn_);
        for (std::uint64_t m = 0; m < M; ++m)
            for (std::uint64_t f = 0; f < fieldsIn_; ++f)
                inViews.v[m * fieldsIn_ + f] = {physIn + ces * ((m * H * fieldsIn_ + f) * nz), nullptr,
                                                static_cast<long long>(fieldsIn_ * nz)};
        horizontal_->inverse_columns_into(inViews, binsIn, s, static_cast<int>(zStride_));
        if (rec) rec->end("columns_inverse_embed", 1, double(inPlanes) * (compactPlane + binsPlane), 0.0);
    }

    const RowFluxArgs a = row_args(M);
    check_cuda(launch_rows_flux(a, s), "fused row flux kernel");
    if (rec) rec->end("rows_flux_fused", 1, double(inPlanes + outPlanes) * binsPlane, 0.0);

    if (dense_) {
        // In-place forward columns keep the retained cells; the GEMM reads them there.
        horizontal_->forward_columns_band(binsOutArr, static_cast<int>(M * T), 1.0, static_cast<int>(zStride_), s);
        if (rec) rec->end("columns_forward_gather", 1, double(outPlanes) * (binsPlane + compactPlane), 0.0);
        gemm_forward(modalOut, s, M, true);
        if (rec) rec->end(gemmStage(false), 1, gemmOut, splitTerms * 4.0 * nz * nj_ * double(M) * H * T);
        return;
    }
    ViewSet outViews{};
    outViews.count = static_cast<int>(M * T);
    for (std::uint64_t m = 0; m < M; ++m)
        for (std::uint64_t t = 0; t < T; ++t)
            outViews.v[m * T + t] = {physOut + ces * ((m * H * T + t) * nz), nullptr, static_cast<long long>(T * nz)};
    horizontal_->forward_columns_from(a.binsOut, outViews, 1.0, s, static_cast<int>(zStride_));
    if (rec) rec->end("columns_forward_gather", 1, double(outPlanes) * (binsPlane + compactPlane), 0.0);

    gemm_forward(modalOut, s, M, false);
    if (rec) rec->end(gemmStage(false), 1, gemmOut, splitTerms * 4.0 * nz * nj_ * double(M) * H * T);
}

void FluxPipeline::run(const void* modalIn, void* modalOut, cudaStream_t s, Recorder* rec, std::uint64_t members) {
    if (fused_) {
        runFused(modalIn, modalOut, s, rec, members);
        return;
    }
    const auto H = modes_, nz = cfg_.nz, T = cfg_.targets, M = members;
    const size_t es = element_bytes(horizontal_->precision());
    const size_t ces = 2 * es;  // complex element bytes
    const double n = static_cast<double>(cfg_.n);
    const double keep = horizontal_->keep();
    auto* physIn = physIn_.get<unsigned char>();
    auto* physOut = physOut_.get<unsigned char>();
    // Algorithmic bytes of one plane through each horizontal stage.
    const double binsPlane = n * keep * ces, realPlane = n * n * es, compactPlane = double(H) * ces;
    const double gemmIn = double(M) * H * fieldsIn_ * (nj_ + nz) * ces + matrix_bytes(true);
    const double gemmOut = double(M) * H * T * (nj_ + nz) * ces + matrix_bytes(false);

    gemm_inverse(modalIn, s, M, false);
    if (rec) rec->end("gemm_inverse", 1, gemmIn, 4.0 * nz * nj_ * double(M) * H * fieldsIn_);

    auto triple = [&](std::uint64_t firstField) {
        ViewSet v{};
        v.count = static_cast<int>(3 * M);
        for (std::uint64_t m = 0; m < M; ++m)
            for (std::uint64_t f = 0; f < 3; ++f)
                v.v[3 * m + f] = {physIn + ces * ((m * H * fieldsIn_ + firstField + f) * nz), nullptr,
                                  static_cast<long long>(fieldsIn_ * nz)};
        return v;
    };
    const double triplePlanes = 3.0 * M * nz;
    auto inverseTriple = [&](std::uint64_t firstField, void* real) {
        const ViewSet v = triple(firstField);
        horizontal_->inverse_columns(v, s);
        if (rec) rec->end("columns_inverse_embed", 1, triplePlanes * (compactPlane + binsPlane), 0.0);
        horizontal_->inverse_rows(real, 3 * M * nz, s);
        if (rec) rec->end("rows_inverse_c2r", 1, triplePlanes * (binsPlane + realPlane), 0.0);
    };
    inverseTriple(0, shared_.get());
    const double scale = 1.0 / (n * n * n * n);
    const int sms = sm_count();
    for (std::uint64_t t = 0; t < T; ++t) {
        inverseTriple(3 + 3 * t, deriv_.get());
        for (std::uint64_t m = 0; m < M; ++m) {
            check_cuda(launch_pointwise(f64(), static_cast<long long>(volume_), scale,
                                        shared_.get<unsigned char>() + es * 3 * m * volume_,
                                        deriv_.get<unsigned char>() + es * 3 * m * volume_,
                                        target_.get<unsigned char>() + es * m * volume_, sms, s),
                       "pointwise advection kernel");
        }
        if (rec) rec->end("pointwise", M, 7.0 * es * double(volume_) * M, 6.0 * double(volume_) * M);
        ViewSet out{};
        out.count = static_cast<int>(M);
        for (std::uint64_t m = 0; m < M; ++m)
            out.v[m] = {physOut + ces * ((m * H * T + t) * nz), nullptr, static_cast<long long>(T * nz)};
        horizontal_->forward_rows(target_.get(), M * nz, s);
        if (rec) rec->end("rows_forward_r2c", 1, double(M) * nz * (realPlane + binsPlane), 0.0);
        horizontal_->forward_columns(out, 1.0, s);
        if (rec) rec->end("columns_forward_gather", 1, double(M) * nz * (binsPlane + compactPlane), 0.0);
    }
    gemm_forward(modalOut, s, M, false);
    if (rec) rec->end("gemm_forward", 1, gemmOut, 4.0 * nz * nj_ * double(M) * H * T);
}

std::vector<const VerticalPlan*> FluxPipeline::gemm_plans() const {
    std::vector<const VerticalPlan*> out;
    if (inverseGemm_) out.push_back(inverseGemm_.get());
    if (forwardGemm_) out.push_back(forwardGemm_.get());
    for (int f = 0; f < 2; ++f) {
        if (inverseFamily_[f].plan) out.push_back(inverseFamily_[f].plan.get());
        if (forwardFamily_[f].plan) out.push_back(forwardFamily_[f].plan.get());
    }
    return out;
}

double FluxPipeline::matrix_bytes(bool inverse) const {
    if (!families_) return static_cast<double>(inverse ? inverseGemm_->matrixBytes() : forwardGemm_->matrixBytes());
    double bytes = 0.0;
    for (const auto& f : inverse ? inverseFamily_ : forwardFamily_)
        if (f.plan) bytes += static_cast<double>(f.plan->matrixBytes());
    return bytes;
}

void FluxPipeline::gemm_inverse(const void* modalIn, cudaStream_t s, std::uint64_t M, bool dense) {
    const ComplexOperand in{const_cast<void*>(modalIn), nullptr};
    const ComplexOperand out{dense ? binsIn_.get() : physIn_.get(), nullptr};
    if (!families_) {
        if (!dense) {
            inverseGemm_->execute(in, out, s, M);
            return;
        }
        const BinBoundary bins{cellIn_.get<long long>(), partnerIn_.get<long long>(), modeConj_.get<unsigned char>(),
                               static_cast<int>(fieldsIn_), static_cast<int>(zStride_)};
        inverseGemm_->execute(in, out, s, M, nullptr, &bins);
        return;
    }
    for (const auto& f : inverseFamily_) {
        if (!f.plan) continue;
        const int* map = f.fieldMap.get<int>();
        const BinBoundary modal{cellModalIn_.get<long long>(), nullptr, nullptr, f.fields, static_cast<int>(nj_),
                                static_cast<long long>(modes_ * fieldsIn_ * nj_), map};
        const BinBoundary target =
            dense ? BinBoundary{cellIn_.get<long long>(), partnerIn_.get<long long>(), modeConj_.get<unsigned char>(),
                                f.fields, static_cast<int>(zStride_), static_cast<long long>(fieldsIn_ * zStride_), map}
                  : BinBoundary{cellPhysIn_.get<long long>(), nullptr, nullptr, f.fields, static_cast<int>(cfg_.nz),
                                static_cast<long long>(modes_ * fieldsIn_ * cfg_.nz), map};
        f.plan->execute(in, out, s, M, &modal, &target);
    }
}

void FluxPipeline::gemm_forward(void* modalOut, cudaStream_t s, std::uint64_t M, bool dense) {
    const ComplexOperand in{dense ? binsOut_.get() : physOut_.get(), nullptr};
    const ComplexOperand out{modalOut, nullptr};
    const std::uint64_t T = cfg_.targets;
    if (!families_) {
        if (!dense) {
            forwardGemm_->execute(in, out, s, M);
            return;
        }
        const BinBoundary bins{cellOut_.get<long long>(), nullptr, modeConj_.get<unsigned char>(), static_cast<int>(T),
                               static_cast<int>(zStride_)};
        forwardGemm_->execute(in, out, s, M, &bins, nullptr);
        return;
    }
    for (const auto& f : forwardFamily_) {
        if (!f.plan) continue;
        const int* map = f.fieldMap.get<int>();
        const BinBoundary source =
            dense ? BinBoundary{cellOut_.get<long long>(), nullptr, modeConj_.get<unsigned char>(), f.fields,
                                static_cast<int>(zStride_), static_cast<long long>(T * zStride_), map}
                  : BinBoundary{cellPhysOut_.get<long long>(), nullptr, nullptr, f.fields, static_cast<int>(cfg_.nz),
                                static_cast<long long>(modes_ * T * cfg_.nz), map};
        const BinBoundary modal{cellModalOut_.get<long long>(), nullptr, nullptr, f.fields, static_cast<int>(nj_),
                                static_cast<long long>(modes_ * T * nj_), map};
        f.plan->execute(in, out, s, M, &source, &modal);
    }
}

void FluxPipeline::check_device_errors() const {
    for (const VerticalPlan* g : gemm_plans()) g->check_device_error();
    if (rowsError_.bytes() != 0) {
        int flag = 0;
        check_cuda(cudaMemcpy(&flag, rowsError_.get(), sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
        if (flag != 0) throw Error(-2, "fused row kernel: a bounded wait for a stage copy expired");
    }
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
