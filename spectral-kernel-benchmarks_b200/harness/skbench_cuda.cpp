// skbench-cuda: the skbench command line (list / validate / run / compare)
// over the cuda provider in libskb_cuda.so.
//
// It mirrors the reference CLI (src/main.cpp:11-246): the same commands, the
// same profiles (src/benchmark.cpp:1039-1056), kernel names `fft` (alias
// `2d-rfft`), `pruned-horizontal`, `vertical-gemm`, `pointwise-advection`,
// `production-lifetime-flux`, `spectral-pipeline` and
// `constant-stratification-vertical`, the spectral-kernel-benchmark-v1 JSON report
// and nine-column CSV, and exit codes 0 (passed), 1 (a correctness check
// failed) and 2 (bad arguments or a provider error).  Everything it runs goes
// through the C ABI of include/skb_cuda.h; primitive timings are CUDA events
// on the provider's stream around device-resident calls, adapter timings are
// host wall-clock around the host-array calls (copies included).

#include <sys/utsname.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

#include "direct.hpp"
#include "fixture.hpp"
#include "report.hpp"
#include "skb_cuda.h"

using namespace skbh;

namespace {

// --------------------------------------------------------------- errors

void ok(int rc) {
    if (rc == SKB_OK) return;
    const std::string what = skb_last_error();
    if (rc == SKB_ERR_INVALID_ARGUMENT) throw std::invalid_argument(what);
    if (rc == SKB_ERR_LOGIC) throw std::logic_error(what);
    throw std::runtime_error(what);
}

// ------------------------------------------------------------- profiles

struct Profile {
    std::string name, purpose;
    skb_workload w;
    std::uint64_t warmups, samples;
};

std::vector<Profile> profiles() {
    auto wl = [](std::uint64_t n, std::uint64_t nz, std::uint64_t f) { return skb_workload{n, n, nz, f, 1.0, 1.0, 1}; };
    return {
        {"smoke", "Small deterministic correctness and CLI exercise; performance is not meaningful.", wl(8, 7, 2), 1, 2},
        {"quick", "First production FFT vertical slice from WVM issue #129.", wl(256, 65, 3), 3, 15},
        {"exhaustive", "Initial larger reference shape from WVM issue #129.", wl(512, 129, 4), 3, 20},
        {"wvm-historical-256-nz65-f3", "Historical issue #129 medium workload, three fields.", wl(256, 65, 3), 3, 15},
        {"wvm-historical-256-nz65-f4", "Historical issue #129 medium workload, four fields.", wl(256, 65, 4), 3, 15},
        {"wvm-historical-512-nz129-f3", "Historical issue #129 large workload, three fields.", wl(512, 129, 3), 3, 20},
        {"wvm-historical-512-nz129-f4", "Historical issue #129 large workload, four fields.", wl(512, 129, 4), 3, 20},
        {"wvm-current-256-nz129-f1", "Current WVM 256-cubed-class workload, one field.", wl(256, 129, 1), 3, 15},
        {"wvm-current-256-nz129-f3", "Current WVM 256-cubed-class workload, three fields.", wl(256, 129, 3), 3, 15},
        {"wvm-current-256-nz129-f4", "Current WVM 256-cubed-class workload, four fields.", wl(256, 129, 4), 3, 15},
        {"wvm-current-512-nz257-f1", "Current WVM 512-cubed-class workload, one field.", wl(512, 257, 1), 3, 20},
        {"wvm-current-512-nz257-f3", "Current WVM 512-cubed-class workload, three fields.", wl(512, 257, 3), 3, 20},
        {"wvm-current-512-nz257-f4", "Current WVM 512-cubed-class workload, four fields.", wl(512, 257, 4), 3, 20},
        {"wvm-large-512-nz513-f4", "Large-vertical nonhydrostatic decision workload, four fields.", wl(512, 513, 4), 3,
         20},
        {"wvm-large-1024-nz129-f4", "Large-horizontal nonhydrostatic decision workload, four fields.",
         wl(1024, 129, 4), 3, 20}};
}

Profile profile_named(const std::string& name) {
    for (const auto& p : profiles())
        if (p.name == name) return p;
    throw std::invalid_argument("Unknown profile: " + name);
}

// --------------------------------------------------------- device memory

struct DeviceBuffer {
    void* p = nullptr;
    std::uint64_t bytes = 0;
    explicit DeviceBuffer(std::uint64_t n) : bytes(n) { ok(skb_device_alloc(std::max<std::uint64_t>(n, 1), &p)); }
    ~DeviceBuffer() {
        if (p) skb_device_free(p);
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    template <typename T>
    void upload(const std::vector<T>& v, void* stream) {
        ok(skb_copy_to_device(p, v.data(), v.size() * sizeof(T), stream));
        ok(skb_stream_synchronize(stream));
    }
    template <typename T>
    std::vector<T> download(std::uint64_t count, void* stream) const {
        std::vector<T> v(count);
        ok(skb_copy_to_host(v.data(), p, count * sizeof(T), stream));
        ok(skb_stream_synchronize(stream));
        return v;
    }
};

// ---------------------------------------------------------------- timing

struct Timer {
    skb_timer* t = nullptr;
    Timer() { ok(skb_timer_create(&t)); }
    ~Timer() { skb_timer_destroy(t); }
};

// W untimed calls, then S calls each bracketed by events on `stream`.
std::vector<double> measure_device(std::uint64_t warmups, std::uint64_t samples, void* stream,
                                   const std::function<void()>& call) {
    Timer timer;
    for (std::uint64_t i = 0; i < warmups; ++i) call();
    ok(skb_stream_synchronize(stream));
    std::vector<double> out;
    for (std::uint64_t i = 0; i < samples; ++i) {
        ok(skb_timer_start(timer.t, stream));
        call();
        ok(skb_timer_stop(timer.t, stream));
        double ms = 0;
        ok(skb_timer_elapsed_ms(timer.t, &ms));
        out.push_back(ms * 1e-3);
    }
    return out;
}

// Host wall clock around blocking calls.
std::vector<double> measure_host(std::uint64_t warmups, std::uint64_t samples, const std::function<void()>& call) {
    using Clock = std::chrono::steady_clock;
    for (std::uint64_t i = 0; i < warmups; ++i) call();
    std::vector<double> out;
    for (std::uint64_t i = 0; i < samples; ++i) {
        const auto t0 = Clock::now();
        call();
        out.push_back(std::chrono::duration<double>(Clock::now() - t0).count());
    }
    return out;
}

Timing series(const std::string& scope, const std::string& stage, const std::string& direction,
              std::uint64_t bytes, std::vector<double> seconds, StageState state = StageState::executed) {
    return {scope, stage, direction, state, bytes, std::move(seconds)};
}

Metric metric(const std::string& name, double maxRel, double relL2, double tol) {
    return {name, maxRel, relL2, tol, std::isfinite(maxRel) && maxRel <= tol && std::isfinite(relL2)};
}

// ----------------------------------------------------------- environment

std::string read_first(const char* path, const char* key) {
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line))
        if (line.rfind(key, 0) == 0) {
            const auto colon = line.find(':');
            if (colon != std::string::npos) return line.substr(line.find_first_not_of(" \t", colon + 1));
        }
    return "";
}

Environment environment() {
    Environment e;
    char buf[256] = {};
    const std::time_t now = std::time(nullptr);
    std::strftime(buf, sizeof buf, "%Y-%m-%dT%H:%M:%SZ", std::gmtime(&now));
    e.timestampUtc = buf;
    if (gethostname(buf, sizeof buf) == 0) e.hostname = buf;
    utsname u{};
    if (uname(&u) == 0) e.operatingSystem = std::string(u.sysname) + " " + u.release + " " + u.machine;
    int devices = 0;
    if (skb_device_count(&devices) == SKB_OK) e.machineModel = std::to_string(devices) + " CUDA device(s), sm_100a build";
    e.cpuBrand = read_first("/proc/cpuinfo", "model name");
    e.totalCores = std::thread::hardware_concurrency();
    e.performanceCores = e.totalCores;
    e.physicalMemoryBytes = std::uint64_t(sysconf(_SC_PHYS_PAGES)) * std::uint64_t(sysconf(_SC_PAGESIZE));
    e.compiler = "g++";
    e.compilerVersion = __VERSION__;
    e.compilerFlags = "-std=c++20 -O2 (harness); nvcc -gencode arch=compute_100a,code=sm_100a -O3 (provider)";
    e.buildType = "Release";
    return e;
}

// --------------------------------------------------------- report set-up

struct Options {
    std::string kernel = "fft", profile = "smoke", providers = "cuda", precision = "fp64";
    std::string gemm = "fp64", family = "k2-grouped", fluxMode = "split-tf32x3", output, fluxFixture;
    std::uint64_t members = 1, targets = 4, warmups = 0, samples = 0, seed = 129;
    bool warmupsSet = false, samplesSet = false, autotune = false;
    std::uint64_t nx = 0, ny = 0, nz = 0, fields = 0;
    // The reference's streaming-provider knobs (RunOptions boundaryPolicy,
    // streamingTileWidth, streamingInversePolicy; skbench.hpp:522-532, 952-954):
    // checked as the reference checks them and recorded, with no effect here.
    std::string boundaryPolicy, inversePolicy = "full-zero";
    std::uint64_t tileWidth = 1;
};

// Checks the streaming-provider knobs against the values the reference accepts
// for the kernel (benchmark.cpp:2978-2985, 3962-3970, 5398-5403;
// pruned_fftw_provider.cpp:626-643; authoritative_spectral_flux.cpp:333-338).
void check_streaming_options(const Options& o) {
    const std::vector<std::string> inverse{"full-zero", "active-reset", "compact-preserved", "full-preserved"};
    if (std::find(inverse.begin(), inverse.end(), o.inversePolicy) == inverse.end())
        throw std::invalid_argument("--streaming-inverse-policy: expected full-zero, active-reset, compact-preserved "
                                    "or full-preserved; got '" + o.inversePolicy + "'.");
    if (o.inversePolicy != "full-zero") {
        if (o.kernel != "production-lifetime-flux")
            throw std::invalid_argument("--streaming-inverse-policy other than full-zero applies to "
                                        "production-lifetime-flux only.");
        if (o.fluxFixture.empty())
            throw std::invalid_argument("--streaming-inverse-policy other than full-zero needs a prepared fixture "
                                        "(--spectral-flux-fixture).");
    }
    if (!o.fluxFixture.empty() && o.tileWidth != 1 && o.tileWidth != 16)
        throw std::invalid_argument("--streaming-tile-width: the authoritative flux graph runs with 16-plane tiles; "
                                    "got " + std::to_string(o.tileWidth) + ".");
    if (o.boundaryPolicy.empty()) return;
    std::vector<std::string> allowed;
    if (o.kernel == "production-lifetime-flux") allowed = {"wvm-direct", "streaming-pruned-compact-split"};
    if (o.kernel == "spectral-pipeline")
        allowed = {"wvm-direct", "plane-major-fused-split", "streaming-pruned-compact-split"};
    if (!allowed.empty() && std::find(allowed.begin(), allowed.end(), o.boundaryPolicy) == allowed.end()) {
        std::string list;
        for (const auto& a : allowed) list += (list.empty() ? "" : ", ") + a;
        throw std::invalid_argument("--boundary-policy for " + o.kernel + ": expected one of " + list + "; got '" +
                                    o.boundaryPolicy + "'.");
    }
}

std::vector<skb_retained_mode> retained_modes(const skb_workload& w) {
    std::uint64_t count = 0;
    ok(skb_retained_modes(&w, nullptr, 0, &count));
    std::vector<skb_retained_mode> modes(count);
    ok(skb_retained_modes(&w, modes.data(), count, &count));
    return modes;
}

std::vector<skb_mode_group> k2_groups(const skb_workload& w) {
    std::uint64_t count = 0;
    ok(skb_squared_wavenumber_groups(&w, nullptr, 0, &count));
    std::vector<skb_mode_group> groups(count);
    ok(skb_squared_wavenumber_groups(&w, groups.data(), count, &count));
    return groups;
}

Report base_report(const Options& o, const Profile& prof, const skb_workload& w) {
    Report r;
    r.profile = prof.name;
    r.seed = o.seed;
    r.warmups = o.warmups;
    r.samples = o.samples;
    r.nx = w.nx;
    r.ny = w.ny;
    r.nz = w.nz;
    r.fields = w.fields;
    r.nj = w.nz < 2 ? 0 : 2 * (w.nz - 1) / 3;
    r.antialias = w.antialias != 0;
    const auto modes = retained_modes(w);
    r.nkl = modes.size();
    char modeHash[64] = {}, groupHash[64] = {}, wvmHash[64] = {};
    ok(skb_order_hashes(&w, modeHash, groupHash, wvmHash));
    r.retainedModeOrderHash = modeHash;
    r.wvmFullSpectrumOrderHash = wvmHash;
    r.verticalGroupOrderHash = groupHash;
    const std::uint64_t planes = w.nz * w.fields, half = w.nx / 2 + 1;
    const std::uint64_t s = o.precision == "fp32" ? 4 : 8;
    r.realBytes = planes * w.nx * w.ny * s;
    r.fullSpectrumBytes = planes * w.ny * half * 2 * s;
    r.retainedSpectrumBytes = modes.size() * planes * 2 * s;
    r.modalSpectrumBytes = modes.size() * w.fields * r.nj * 2 * s;
    r.scalarTypeId = o.precision == "fp32" ? "float32" : "float64";
    r.scalarBits = o.precision == "fp32" ? 32 : 64;
    const std::time_t now = std::time(nullptr);
    char buf[64];
    std::strftime(buf, sizeof buf, "%Y%m%dT%H%M%SZ", std::gmtime(&now));
    r.runId = std::string(buf) + "-" + o.kernel + "-" + prof.name + "-cuda";
    r.environment = environment();
    return r;
}

void fill_info(ProviderRecord& rec, const skb_provider_info& info) {
    rec.version = info.version;
    rec.libraryIdentity = info.library_identity;
    rec.allocationSeconds = info.allocation_seconds;
    rec.planningSeconds = info.planning_seconds;
    rec.otherSetupSeconds = info.other_setup_seconds;
    rec.persistentBytes = info.persistent_bytes;
    rec.scratchBytes = info.scratch_bytes;
    rec.planningBytes = info.planning_bytes;
    rec.forward.destroysNativeInput = info.destroys_native_input != 0;
    rec.inverse.destroysNativeInput = info.destroys_native_input != 0;
}

int precision_code(const Options& o) {
    if (o.precision == "fp64") return SKB_PRECISION_FP64;
    if (o.precision == "fp32") return SKB_PRECISION_FP32;
    throw std::invalid_argument("precision must be 'fp64' or 'fp32'.");
}

template <typename T>
std::vector<T> narrow(const std::vector<double>& v) {
    return std::vector<T>(v.begin(), v.end());
}

// The values the device actually received: rounded to float for FP32 runs.
std::vector<double> as_used(const std::vector<double>& v, bool f32) {
    if (!f32) return v;
    std::vector<double> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = double(float(v[i]));
    return out;
}

std::vector<double> widen_real(const DeviceBuffer& b, std::uint64_t count, bool f32, void* stream) {
    if (!f32) return b.download<double>(count, stream);
    const auto f = b.download<float>(count, stream);
    return std::vector<double>(f.begin(), f.end());
}

std::vector<cplx> widen_complex(const DeviceBuffer& b, std::uint64_t count, bool f32, void* stream) {
    const auto r = widen_real(b, 2 * count, f32, stream);
    std::vector<cplx> out(count);
    for (std::uint64_t i = 0; i < count; ++i) out[i] = cplx(r[2 * i], r[2 * i + 1]);
    return out;
}

// Sampled direct-DFT check of a WVM spectrum: `probes` bins (ky, kx, plane)
// spread over the spectrum, each a direct long double sum over the plane.
Metric spectrum_probes(const skb_workload& w, const std::vector<double>& real, const std::vector<cplx>& spectrum,
                       std::uint64_t probes, double tol, const std::string& name) {
    const std::uint64_t half = w.nx / 2 + 1, planes = w.nz * w.fields;
    const auto rx = unit_roots(w.nx, -1), ry = unit_roots(w.ny, -1);
    std::mt19937_64 rng(7);
    std::vector<cplx> got, want;
    for (std::uint64_t i = 0; i < probes; ++i) {
        const std::uint64_t ky = rng() % w.ny, kx = rng() % half, p = rng() % planes;
        lcplx s = 0;
        const double* f = real.data() + p * w.nx * w.ny;
        for (std::uint64_t y = 0; y < w.ny; ++y) {
            lcplx row = 0;
            for (std::uint64_t x = 0; x < w.nx; ++x) row += static_cast<long double>(f[y * w.nx + x]) * rx[(kx * x) % w.nx];
            s += row * ry[(ky * y) % w.ny];
        }
        const std::uint64_t field = p / w.nz, z = p % w.nz;
        want.emplace_back(double(s.real()), double(s.imag()));
        got.push_back(spectrum[((ky * half + kx) * w.fields + field) * w.nz + z]);
    }
    return metric(name, max_relative_error(got.data(), want.data(), got.size()),
                  relative_l2_error(got.data(), want.data(), got.size()), tol);
}

// ------------------------------------------------------------ kernels

ProviderRecord run_fft(const Options& o, const skb_workload& w, Report& report) {
    const int prec = precision_code(o);
    const bool f32 = prec == SKB_PRECISION_FP32;
    const double tol = f32 ? 1e-5 : 1e-12;
    const std::uint64_t s = f32 ? 4 : 8, planes = w.nz * w.fields, half = w.nx / 2 + 1;
    const std::uint64_t realN = planes * w.nx * w.ny, specN = planes * w.ny * half;
    std::vector<double> input(realN);
    ok(skb_make_fixture(&w, 2, o.seed, input.data()));

    skb_fft_provider* h = nullptr;
    ok(skb_fft_create(&w, prec, &h));
    std::unique_ptr<skb_fft_provider, int (*)(skb_fft_provider*)> guard(h, skb_fft_destroy);
    void* stream = skb_fft_stream(h);
    skb_provider_info info{};
    ok(skb_fft_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    rec.algorithmId = "stockham-radix8-smem-rows-then-columns";
    rec.nativeRepresentationId = "wvm-frequency-major-interleaved-hermitian-half-spectrum";
    rec.modeOrderId = "wvm-full-spectrum";
    rec.planningConfiguration = std::string(f32 ? "float32" : "float64") + "; batched row r2c + column c2c kernels";
    for (auto* d : {&rec.forward, &rec.inverse}) {
        d->nativePlacement = "out-of-place device arrays";
        d->adapterPlacement = "out-of-place host arrays";
    }
    rec.forward.nativeInputRepresentationId = "real [field][z][y][x]";
    rec.forward.nativeOutputRepresentationId = "WVM [ky][kx][field][z]";
    rec.inverse.nativeInputRepresentationId = "WVM [ky][kx][field][z]";
    rec.inverse.nativeOutputRepresentationId = "real [field][z][y][x]";

    DeviceBuffer dReal(realN * s), dSpec(specN * 2 * s), dBack(realN * s);
    if (f32) dReal.upload(narrow<float>(input), stream);
    else dReal.upload(input, stream);
    const std::uint64_t bytes = realN * s + specN * 2 * s;
    rec.timings.push_back(series("primitive", "raw FFT", "forward", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_fft_forward_device(h, dReal.p, dSpec.p, stream));
                                 })));
    rec.timings.push_back(series("primitive", "raw FFT", "inverse", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_fft_inverse_device(h, dSpec.p, dBack.p, stream));
                                 })));
    // Adapter: host FP64 arrays in and out, copies (and FP32 staging) included.
    std::vector<skb_complex> hostSpec(specN);
    std::vector<double> hostBack(realN);
    rec.timings.push_back(series("adapter-total", "WVM-compatible full-spectrum adapter", "forward", bytes,
                                 measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_fft_forward(h, input.data(), hostSpec.data()));
                                 })));
    rec.timings.push_back(series("adapter-total", "WVM-compatible full-spectrum adapter", "inverse", bytes,
                                 measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_fft_inverse(h, hostSpec.data(), hostBack.data()));
                                 })));
    rec.ledger = {{"row r2c", StageState::executed, "half-length complex FFT per row, planes innermost"},
                  {"column c2c", StageState::executed, "Ny-point FFT per kx column, in place in the output"},
                  {"spectrum-order permutation", StageState::fused, "rows write WVM order directly"}};

    // Correctness: forward against direct DFT probes, round trip against the input.
    ok(skb_fft_forward_device(h, dReal.p, dSpec.p, stream));
    ok(skb_fft_inverse_device(h, dSpec.p, dBack.p, stream));
    ok(skb_stream_synchronize(stream));
    const auto spec = widen_complex(dSpec, specN, f32, stream);
    const auto back = widen_real(dBack, realN, f32, stream);
    const std::vector<double> used = as_used(input, f32);
    rec.correctness.push_back(spectrum_probes(w, used, spec, 64, tol, "forward vs direct DFT (64 sampled bins)"));
    const double scale = 1.0 / double(w.nx * w.ny);
    rec.correctness.push_back(metric("inverse(forward(x)) / (Nx*Ny) vs x",
                                     max_relative_error(back.data(), used.data(), realN, scale),
                                     relative_l2_error(back.data(), used.data(), realN, scale), tol));
    (void)report;
    return rec;
}

ProviderRecord run_pruned(const Options& o, const skb_workload& w, Report& report) {
    const int prec = precision_code(o);
    const bool f32 = prec == SKB_PRECISION_FP32;
    const double tol = f32 ? 1e-5 : 1e-12;
    const std::uint64_t s = f32 ? 4 : 8, planes = w.nz * w.fields;
    const std::uint64_t realN = planes * w.nx * w.ny;
    const auto modes = retained_modes(w);
    const std::uint64_t retN = modes.size() * planes;
    std::vector<double> input(realN);
    ok(skb_make_fixture(&w, 2, o.seed, input.data()));

    skb_pruned_provider* h = nullptr;
    ok(skb_pruned_create(&w, prec, &h));
    std::unique_ptr<skb_pruned_provider, int (*)(skb_pruned_provider*)> guard(h, skb_pruned_destroy);
    void* stream = skb_pruned_stream(h);
    skb_provider_info info{};
    ok(skb_pruned_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    rec.algorithmId = "pruned-rows-then-active-kx-columns-with-fused-retention";
    rec.nativeRepresentationId = "retained [mode][field][z] interleaved";
    rec.modeOrderId = "radial-two-thirds-sorted(radius,k,l)";
    rec.planningConfiguration = "active kx " + std::to_string(info.active_kx) + " of " + std::to_string(info.full_kx) +
                                "; omitted column transforms " +
                                std::to_string(info.omitted_column_transforms_per_direction);
    for (auto* d : {&rec.forward, &rec.inverse}) {
        d->nativePlacement = "out-of-place device arrays";
        d->adapterPlacement = "out-of-place host arrays";
    }
    rec.forward.nativeOutputRepresentationId = rec.inverse.nativeInputRepresentationId = rec.nativeRepresentationId;

    DeviceBuffer dReal(realN * s), dRet(retN * 2 * s), dBack(realN * s);
    if (f32) dReal.upload(narrow<float>(input), stream);
    else dReal.upload(input, stream);
    std::vector<skb_field_view> views(w.fields);
    for (std::uint64_t f = 0; f < w.fields; ++f)
        views[f] = {static_cast<char*>(dRet.p) + f * w.nz * 2 * s, nullptr, planes};
    const std::uint64_t bytes = realN * s + retN * 2 * s;
    rec.timings.push_back(series("primitive", "raw pruned FFT", "forward", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_forward_device(h, dReal.p, views.data(), w.fields, 1.0, stream));
                                 })));
    rec.timings.push_back(series("primitive", "raw pruned FFT", "inverse", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_inverse_device(h, views.data(), w.fields, dBack.p, stream));
                                 })));
    rec.timings.push_back(series("primitive-component", "pruned row FFT batch", "forward", 0,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_forward_rows_device(h, dReal.p, stream));
                                 })));
    rec.timings.push_back(series("primitive-component", "retained-support column FFT batch", "forward", 0,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_forward_columns_device(h, views.data(), w.fields, 1.0, stream));
                                 })));
    rec.timings.push_back(series("primitive-component", "retained-support inverse column FFT batch", "inverse", 0,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_inverse_columns_device(h, views.data(), w.fields, stream));
                                 })));
    rec.timings.push_back(series("primitive-component", "pruned inverse row FFT batch", "inverse", 0,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pruned_inverse_rows_device(h, dBack.p, stream));
                                 })));
    std::vector<skb_complex> hostRet(retN);
    std::vector<double> hostBack(realN);
    rec.timings.push_back(series("adapter-total", "pruned retained adapter", "forward", bytes,
                                 measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_pruned_forward(h, input.data(), hostRet.data()));
                                 })));
    rec.timings.push_back(series("adapter-total", "pruned retained adapter", "inverse", bytes,
                                 measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_pruned_inverse(h, hostRet.data(), hostBack.data()));
                                 })));
    rec.ledger = {{"row r2c", StageState::executed, "all rows, only the active kx band written"},
                  {"column c2c", StageState::executed, "active kx columns only"},
                  {"retention gather / embed", StageState::fused, "inside the column kernels"},
                  {"kx = 0 Hermitian repair", StageState::fused, "inside the inverse column kernel"}};

    // Correctness: forward vs sampled direct retained values; inverse(forward)
    // round trip of the retained band.
    ok(skb_pruned_forward_device(h, dReal.p, views.data(), w.fields, 1.0, stream));
    ok(skb_stream_synchronize(stream));
    const auto ret = widen_complex(dRet, retN, f32, stream);
    const std::vector<double> used = as_used(input, f32);
    {
        const auto rx = unit_roots(w.nx, -1), ry = unit_roots(w.ny, -1);
        std::mt19937_64 rng(11);
        std::vector<cplx> got, want;
        for (int i = 0; i < 64; ++i) {
            const std::uint64_t m = rng() % modes.size(), p = rng() % planes;
            const auto& md = modes[m];
            lcplx acc = 0;
            const double* f = used.data() + p * w.nx * w.ny;
            for (std::uint64_t y = 0; y < w.ny; ++y) {
                lcplx row = 0;
                for (std::uint64_t x = 0; x < w.nx; ++x)
                    row += static_cast<long double>(f[y * w.nx + x]) * rx[(md.stored_kx * x) % w.nx];
                acc += row * ry[(md.stored_ky * y) % w.ny];
            }
            cplx v(double(acc.real()), double(acc.imag()));
            if (md.conjugates_stored_value) v = std::conj(v);
            want.push_back(v);
            got.push_back(ret[m * planes + p]);
        }
        rec.correctness.push_back(metric("forward vs direct retained DFT (64 sampled modes)",
                                         max_relative_error(got.data(), want.data(), got.size()),
                                         relative_l2_error(got.data(), want.data(), got.size()), tol));
    }
    ok(skb_pruned_inverse_device(h, views.data(), w.fields, dBack.p, stream));
    ok(skb_pruned_forward_device(h, dBack.p, views.data(), w.fields, 1.0 / double(w.nx * w.ny), stream));
    ok(skb_stream_synchronize(stream));
    const auto again = widen_complex(dRet, retN, f32, stream);
    rec.correctness.push_back(metric("forward(inverse(R)) / (Nx*Ny) vs R", max_relative_error(again.data(), ret.data(), retN),
                                     relative_l2_error(again.data(), ret.data(), retN), tol));
    (void)report;
    return rec;
}

int gemm_code(const std::string& g) {
    if (g == "fp64") return SKB_GEMM_FP64;
    if (g == "fp32") return SKB_GEMM_FP32;
    if (g == "tf32x3") return SKB_GEMM_TF32X3;
    if (g == "bf16x3") return SKB_GEMM_BF16X3;
    throw std::invalid_argument("vertical-gemm-precision must be 'fp64', 'fp32', 'tf32x3' or 'bf16x3'.");
}

ProviderRecord run_vertical(const Options& o, const skb_workload& w, Report& report) {
    const int gemm = gemm_code(o.gemm);
    const bool f32 = gemm != SKB_GEMM_FP64;
    const double tol = gemm == SKB_GEMM_FP64 ? 1e-12 : (gemm == SKB_GEMM_TF32X3 || gemm == SKB_GEMM_BF16X3) ? 1e-6 : 1e-5;
    const std::uint64_t s = f32 ? 4 : 8, nz = w.nz, nj = nz < 2 ? 0 : 2 * (nz - 1) / 3;
    const auto modes = retained_modes(w);
    const int family = o.family == "common" ? SKB_FAMILY_COMMON_DCT2 : SKB_FAMILY_K2_ROTATION;
    if (o.family != "common" && o.family != "k2-grouped")
        throw std::invalid_argument("vertical-gemm-family must be 'common' or 'k2-grouped'.");
    std::vector<skb_mode_group> groups;
    if (family == SKB_FAMILY_COMMON_DCT2) groups = {{0, 0, modes.size()}};
    else groups = k2_groups(w);
    std::vector<double> fwd(groups.size() * nj * nz), inv(groups.size() * nz * nj);
    std::uint64_t familyGroups = 0;
    char id[128] = {};
    ok(skb_vertical_family(&w, family, o.seed, fwd.data(), inv.data(), fwd.size(), &familyGroups, id));
    report.verticalMatrixFamilyId = id;
    report.verticalGroupCount = groups.size();
    report.verticalMatrixFamilySourceBytes = 2 * fwd.size() * sizeof(double);
    {
        std::vector<double> sizes;
        for (const auto& g : groups) sizes.push_back(double(g.mode_count));
        report.minGroupModes = std::uint64_t(*std::min_element(sizes.begin(), sizes.end()));
        report.maxGroupModes = std::uint64_t(*std::max_element(sizes.begin(), sizes.end()));
        report.medianGroupModes = median(sizes);
        report.minGroupColumns = report.minGroupModes * w.fields;
        report.maxGroupColumns = report.maxGroupModes * w.fields;
        report.medianGroupColumns = report.medianGroupModes * double(w.fields);
    }

    skb_vertical_provider* h = nullptr;
    ok(skb_vertical_create(&w, groups.data(), groups.size(), fwd.data(), inv.data(), SKB_LAYOUT_INTERLEAVED,
                           SKB_BUFFERS_BIDIRECTIONAL, gemm, &h));
    std::unique_ptr<skb_vertical_provider, int (*)(skb_vertical_provider*)> guard(h, skb_vertical_destroy);
    void* stream = skb_vertical_stream(h);
    skb_provider_info info{};
    ok(skb_vertical_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    rec.algorithmId = gemm == SKB_GEMM_TF32X3   ? "grouped-gemm-tcgen05-tf32x3"
                      : gemm == SKB_GEMM_BF16X3 ? "grouped-gemm-tcgen05-bf16x3"
                                                : "grouped-gemm-simt-cp-async";
    rec.nativeRepresentationId = "complex columns [mode][field][z|j] interleaved";
    rec.modeOrderId = "radial-two-thirds-sorted(radius,k,l); K^2 groups contiguous";
    rec.planningConfiguration = std::string(id) + "; " + o.gemm + "; " + std::to_string(groups.size()) + " groups";
    rec.gemmCallsPerExecution = 1;
    for (auto* d : {&rec.forward, &rec.inverse}) {
        d->nativePlacement = "out-of-place device arrays";
        d->adapterPlacement = "provider-owned device buffers loaded from host";
    }

    const std::uint64_t cols = modes.size() * w.fields;
    std::mt19937_64 rng(o.seed ^ 0x9e3779b97f4a7c15ULL);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> phys(cols * nz * 2), modal(cols * nj * 2);
    for (auto& v : phys) v = u(rng);
    for (auto& v : modal) v = u(rng);
    DeviceBuffer dPhys(phys.size() * s), dModal(modal.size() * s), dPhysOut(phys.size() * s), dModalOut(modal.size() * s);
    if (f32) {
        dPhys.upload(narrow<float>(phys), stream);
        dModal.upload(narrow<float>(modal), stream);
    } else {
        dPhys.upload(phys, stream);
        dModal.upload(modal, stream);
    }
    const std::uint64_t matrixBytes = groups.size() * nz * nj * s;
    const std::uint64_t bytes = matrixBytes + cols * (nz + nj) * 2 * s;
    rec.timings.push_back(series("primitive", "raw vertical GEMM", "forward", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_vertical_forward_device(h, dPhys.p, nullptr, dModalOut.p, nullptr, stream));
                                 })));
    rec.timings.push_back(series("primitive", "raw vertical GEMM", "inverse", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_vertical_inverse_device(h, dModal.p, nullptr, dPhysOut.p, nullptr, stream));
                                 })));
    rec.ledger = {{"matrix preparation", StageState::setupOnly, "family transposed / tiled once at creation"},
                  {"packing and representation conversion", StageState::elided, "columns used in place"}};

    // 17 sampled columns recomputed on the host in long double.
    ok(skb_vertical_forward_device(h, dPhys.p, nullptr, dModalOut.p, nullptr, stream));
    ok(skb_vertical_inverse_device(h, dModal.p, nullptr, dPhysOut.p, nullptr, stream));
    ok(skb_stream_synchronize(stream));
    const auto gotF = widen_real(dModalOut, modal.size(), f32, stream);
    const auto gotI = widen_real(dPhysOut, phys.size(), f32, stream);
    const auto physUsed = as_used(phys, f32);
    const auto modalUsed = as_used(modal, f32);
    std::vector<std::uint64_t> groupOf(modes.size());
    for (std::uint64_t g = 0; g < groups.size(); ++g)
        for (std::uint64_t m = 0; m < groups[g].mode_count; ++m) groupOf[groups[g].first_mode + m] = g;
    std::vector<cplx> aF, eF, aI, eI;
    for (int probe = 0; probe < 17; ++probe) {
        const std::uint64_t col = (probe * (cols - 1)) / 16, m = col / w.fields;
        const std::uint64_t g = family == SKB_FAMILY_COMMON_DCT2 ? 0 : groupOf[m];
        for (std::uint64_t j = 0; j < nj; ++j) {
            long double re = 0, im = 0;
            for (std::uint64_t z = 0; z < nz; ++z) {
                const long double a = fwd[(g * nj + j) * nz + z];
                re += a * physUsed[2 * (col * nz + z)];
                im += a * physUsed[2 * (col * nz + z) + 1];
            }
            eF.emplace_back(double(re), double(im));
            aF.emplace_back(gotF[2 * (col * nj + j)], gotF[2 * (col * nj + j) + 1]);
        }
        for (std::uint64_t z = 0; z < nz; ++z) {
            long double re = 0, im = 0;
            for (std::uint64_t j = 0; j < nj; ++j) {
                const long double a = inv[(g * nz + z) * nj + j];
                re += a * modalUsed[2 * (col * nj + j)];
                im += a * modalUsed[2 * (col * nj + j) + 1];
            }
            eI.emplace_back(double(re), double(im));
            aI.emplace_back(gotI[2 * (col * nz + z)], gotI[2 * (col * nz + z) + 1]);
        }
    }
    rec.correctness.push_back(metric("forward, 17 probe columns", max_relative_error(aF.data(), eF.data(), aF.size()),
                                     relative_l2_error(aF.data(), eF.data(), aF.size()), tol));
    rec.correctness.push_back(metric("inverse, 17 probe columns", max_relative_error(aI.data(), eI.data(), aI.size()),
                                     relative_l2_error(aI.data(), eI.data(), aI.size()), tol));
    return rec;
}

ProviderRecord run_pointwise(const Options& o, const skb_workload& w, Report& report) {
    const int prec = precision_code(o);
    const bool f32 = prec == SKB_PRECISION_FP32;
    const double tol = f32 ? 1e-6 : 1e-15;
    const std::uint64_t s = f32 ? 4 : 8, V = w.nx * w.ny * w.nz;
    const double scale = 1.0 / double(w.nx * w.ny) / double(w.nx * w.ny);
    skb_pointwise_executor* h = nullptr;
    ok(skb_pointwise_create(V, scale, prec, &h));
    std::unique_ptr<skb_pointwise_executor, int (*)(skb_pointwise_executor*)> guard(h, skb_pointwise_destroy);
    void* stream = skb_pointwise_stream(h);
    std::mt19937_64 rng(o.seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> shared(3 * V), deriv(3 * V);
    for (auto& v : shared) v = u(rng);
    for (auto& v : deriv) v = u(rng);
    DeviceBuffer dS(3 * V * s), dD(3 * V * s), dT(V * s);
    if (f32) {
        dS.upload(narrow<float>(shared), stream);
        dD.upload(narrow<float>(deriv), stream);
    } else {
        dS.upload(shared, stream);
        dD.upload(deriv, stream);
    }
    ProviderRecord rec;
    rec.algorithmId = "fused-three-term-product-vectorised";
    rec.nativeRepresentationId = "real volumes [field][z][y][x]";
    rec.planningConfiguration = "scale = 1/(Nx*Ny)^2";
    rec.forward.nativePlacement = "out-of-place device arrays";
    rec.inverse.nativePlacement = "unsupported";
    rec.timings.push_back(series("primitive", "pointwise advection", "pointwise", 7 * V * s,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pointwise_execute_device(h, dS.p, dD.p, dT.p, stream));
                                 })));
    ok(skb_pointwise_execute_device(h, dS.p, dD.p, dT.p, stream));
    ok(skb_stream_synchronize(stream));
    const auto got = widen_real(dT, V, f32, stream);
    std::vector<double> want(V);
    for (std::uint64_t i = 0; i < V; ++i) {
        auto val = [&](const std::vector<double>& v, std::uint64_t k) { return f32 ? double(float(v[k])) : v[k]; };
        want[i] = -scale * (val(shared, i) * val(deriv, i) + val(shared, V + i) * val(deriv, V + i) +
                            val(shared, 2 * V + i) * val(deriv, 2 * V + i));
    }
    rec.correctness.push_back(metric("target vs host expression", max_relative_error(got.data(), want.data(), V, 1.0),
                                     relative_l2_error(got.data(), want.data(), V, 1.0),
                                     f32 ? tol : 1e-15 * 4));
    (void)report;
    return rec;
}

// The spectral-pipeline round trip composed on the host with the direct
// transforms (benchmark.cpp:3072-3110 order) for the correctness check.
std::vector<double> host_pipeline(const skb_workload& w, const std::vector<double>& real) {
    const auto modes = retained_modes(w);
    const auto groups = k2_groups(w);
    const std::uint64_t nz = w.nz, nj = 2 * (nz - 1) / 3, F = w.fields;
    std::vector<double> fwd(groups.size() * nj * nz), inv(groups.size() * nz * nj), weights(modes.size() * F * nj);
    std::uint64_t familyGroups = 0;
    char id[128] = {};
    ok(skb_vertical_family(&w, SKB_FAMILY_K2_ROTATION, 0, fwd.data(), inv.data(), fwd.size(), &familyGroups, id));
    ok(skb_modal_weights(&w, weights.data()));
    std::vector<std::uint64_t> groupOf(modes.size());
    for (std::uint64_t g = 0; g < groups.size(); ++g)
        for (std::uint64_t m = 0; m < groups[g].mode_count; ++m) groupOf[groups[g].first_mode + m] = g;
    const auto spec = direct_r2c(w, real.data());
    const auto ret = gather(w, modes, spec.data());
    std::vector<cplx> back(ret.size());
    for (std::size_t m = 0; m < modes.size(); ++m)
        for (std::uint64_t f = 0; f < F; ++f) {
            std::vector<lcplx> modal(nj);
            for (std::uint64_t j = 0; j < nj; ++j) {
                lcplx acc = 0;
                for (std::uint64_t z = 0; z < nz; ++z) {
                    const cplx v = ret[(m * F + f) * nz + z];
                    acc += static_cast<long double>(fwd[(groupOf[m] * nj + j) * nz + z]) * lcplx(v.real(), v.imag());
                }
                modal[j] = lcplx(static_cast<double>(acc.real()), static_cast<double>(acc.imag())) *
                           static_cast<long double>(weights[(m * F + f) * nj + j]);
            }
            for (std::uint64_t z = 0; z < nz; ++z) {
                lcplx acc = 0;
                for (std::uint64_t j = 0; j < nj; ++j)
                    acc += static_cast<long double>(inv[(groupOf[m] * nz + z) * nj + j]) * modal[j];
                back[(m * F + f) * nz + z] = cplx(double(acc.real()), double(acc.imag()));
            }
        }
    const auto full = embed(w, modes, back.data());
    return direct_c2r(w, full.data());
}

ProviderRecord run_pipeline(const Options& o, const skb_workload& w, Report& report) {
    const int prec = precision_code(o);
    const bool f32 = prec == SKB_PRECISION_FP32;
    const std::uint64_t s = f32 ? 4 : 8, planes = w.nz * w.fields, realN = planes * w.nx * w.ny;
    std::vector<double> input(realN);
    ok(skb_make_fixture(&w, 2, o.seed, input.data()));
    skb_pipeline* h = nullptr;
    ok(skb_pipeline_create(&w, prec, &h));
    std::unique_ptr<skb_pipeline, int (*)(skb_pipeline*)> guard(h, skb_pipeline_destroy);
    void* stream = skb_pipeline_stream(h);
    skb_provider_info info{};
    ok(skb_pipeline_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    rec.algorithmId = f32 ? "pruned FP32 transforms + split-TF32x3 tcgen05 K2 GEMMs + modal work"
                          : "pruned FP64 transforms + FP64 K2 GEMMs + modal work";
    rec.nativeRepresentationId = "retained [mode][field][z] / modal [mode][field][j] interleaved";
    rec.modeOrderId = "radial-two-thirds-sorted(radius,k,l); K^2 groups contiguous";
    rec.planningConfiguration = "streaming-pruned-compact (device-resident); K^2 pair-rotation family";
    rec.gemmCallsPerExecution = 2;
    rec.forward.nativePlacement = "out-of-place device arrays";
    rec.forward.adapterPlacement = "out-of-place host arrays";
    rec.inverse = rec.forward;
    DeviceBuffer dIn(realN * s), dOut(realN * s);
    if (f32) dIn.upload(narrow<float>(input), stream);
    else dIn.upload(input, stream);
    const auto modes = retained_modes(w);
    const std::uint64_t nj = w.nz < 2 ? 0 : 2 * (w.nz - 1) / 3;
    const std::uint64_t bytes = 2 * realN * s;
    rec.timings.push_back(series("primitive", "spectral-pipeline round trip", "shared", bytes,
                                 measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_pipeline_execute_device(h, dIn.p, dOut.p, stream));
                                 })));
    std::vector<double> hostOut(realN);
    rec.timings.push_back(series("adapter-total", "spectral-pipeline round trip (host arrays)", "shared", bytes,
                                 measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_pipeline_execute(h, input.data(), hostOut.data()));
                                 })));
    std::vector<skb_stage_time> stages(16);
    std::uint64_t count = 0;
    ok(skb_pipeline_profile(h, dIn.p, dOut.p, stages.data(), stages.size(), &count));
    for (std::uint64_t i = 0; i < count; ++i)
        rec.timings.push_back(series("primitive-component", stages[i].name, "shared",
                                     std::uint64_t(stages[i].algorithmic_bytes), {stages[i].ms * 1e-3}));
    rec.ledger = {{"horizontal forward + retention", StageState::executed, "pruned rows, active-kx columns"},
                  {"vertical forward", StageState::executed, "one launch for all K^2 groups"},
                  {"synthetic modal work", StageState::executed, "one elementwise launch"},
                  {"vertical inverse", StageState::executed, "one launch for all K^2 groups"},
                  {"embedding + horizontal inverse", StageState::executed, "kx = 0 repair fused into the columns"}};
    // Correctness: the host composition with direct transforms where cheap,
    // else FP32 against the FP64 pipeline on the same input.
    const double tol = f32 ? 1e-5 : 1e-12;
    const auto got = hostOut;
    if (w.nx <= 64 && w.ny <= 64) {
        const auto used = as_used(input, f32);
        const auto want = host_pipeline(w, used);
        rec.correctness.push_back(metric("round trip vs direct host composition",
                                         max_relative_error(got.data(), want.data(), realN, 1.0),
                                         relative_l2_error(got.data(), want.data(), realN, 1.0), tol));
    } else if (f32) {
        skb_pipeline* h64 = nullptr;
        ok(skb_pipeline_create(&w, SKB_PRECISION_FP64, &h64));
        std::unique_ptr<skb_pipeline, int (*)(skb_pipeline*)> g64(h64, skb_pipeline_destroy);
        std::vector<double> want(realN);
        ok(skb_pipeline_execute(h64, input.data(), want.data()));
        rec.correctness.push_back(metric("FP32/TF32x3 vs FP64 pipeline",
                                         max_relative_error(got.data(), want.data(), realN, 1.0),
                                         relative_l2_error(got.data(), want.data(), realN, 1.0), tol));
    }
    (void)modes;
    (void)nj;
    report.verticalMatrixFamilyId = "k2-pair-rotation";
    return rec;
}

// ------------------------------------- constant-stratification vertical
// runConstantStratificationVerticalBenchmark (src/constant_stratification.cpp:
// 481-648): the type-I vertical call graph of the constant-stratification
// flux on the full half-spectrum rows and on the retained compact rows, with
// the same stage names, correctness checks and record layout.

namespace type1 {

// deterministicValue (constant_stratification.cpp:233-239).
cplx value(std::uint64_t row, std::uint64_t channel, std::uint64_t z) {
    const double a = 0.017 * double(1 + row % 97) + 0.113 * double(1 + channel) + 0.071 * double(1 + z);
    return cplx(std::sin(a), std::cos(1.7 * a));
}

std::vector<cplx> fill_full(std::uint64_t rows, std::uint64_t channels, std::uint64_t nz) {
    std::vector<cplx> a(rows * channels * nz);
    for (std::uint64_t r = 0; r < rows; ++r)
        for (std::uint64_t c = 0; c < channels; ++c)
            for (std::uint64_t z = 0; z < nz; ++z) a[(r * channels + c) * nz + z] = value(r, c, z);
    return a;
}

std::vector<cplx> fill_compact(const std::vector<skb_retained_mode>& modes, std::uint64_t nxHalf,
                               std::uint64_t channels, std::uint64_t nz) {
    std::vector<cplx> a(modes.size() * channels * nz);
    for (std::size_t m = 0; m < modes.size(); ++m) {
        const std::uint64_t row = modes[m].stored_kx + nxHalf * modes[m].stored_ky;
        for (std::uint64_t c = 0; c < channels; ++c)
            for (std::uint64_t z = 0; z < nz; ++z) {
                const cplx v = value(row, c, z);
                a[(m * channels + c) * nz + z] = modes[m].conjugates_stored_value ? std::conj(v) : v;
            }
    }
    return a;
}

// Normalised forward type-I transforms of one column in long double (the
// reference's directForwardDct / directForwardDst, 273-311).
std::vector<cplx> direct(const std::vector<cplx>& x, bool sine) {
    const std::uint64_t nz = x.size(), m = nz - 1;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<cplx> out(nz);
    for (std::uint64_t j = 0; j < nz; ++j) {
        if (sine && (j == 0 || j == m)) continue;
        lcplx acc = 0;
        if (!sine) {
            const long double sign = j % 2 == 0 ? 1.0L : -1.0L;
            acc = lcplx(x[0].real(), x[0].imag()) + sign * lcplx(x[m].real(), x[m].imag());
        }
        for (std::uint64_t z = 1; z < m; ++z) {
            const long double angle = pi * static_cast<long double>((j * z) % (2 * m)) / static_cast<long double>(m);
            const long double f = 2.0L * (sine ? std::sin(angle) : std::cos(angle));
            acc += f * lcplx(x[z].real(), x[z].imag());
        }
        acc /= static_cast<long double>(m);
        if (!sine && j == m) acc *= 0.5L;
        out[j] = cplx(double(acc.real()), double(acc.imag()));
    }
    return out;
}

// Compact rows against their full half-spectrum rows (conjugated where the
// mode stores its conjugate), as compactFullCorrectness (414-455).
std::pair<double, double> compact_vs_full(const std::vector<cplx>& compact, const std::vector<cplx>& full,
                                          const std::vector<skb_retained_mode>& modes, std::uint64_t nxHalf,
                                          std::uint64_t channels, std::uint64_t nz) {
    std::vector<cplx> ref(compact.size());
    for (std::size_t m = 0; m < modes.size(); ++m) {
        const std::uint64_t row = modes[m].stored_kx + nxHalf * modes[m].stored_ky;
        for (std::uint64_t i = 0; i < channels * nz; ++i) {
            const cplx v = full[row * channels * nz + i];
            ref[m * channels * nz + i] = modes[m].conjugates_stored_value ? std::conj(v) : v;
        }
    }
    return {max_relative_error(compact.data(), ref.data(), ref.size()),
            relative_l2_error(compact.data(), ref.data(), ref.size())};
}

}  // namespace type1

std::vector<ProviderRecord> run_constant_stratification(const Options& o, skb_workload& w, Report& report) {
    if (w.nx != w.ny || w.nx % 2 != 0 || w.nz < 3)
        throw std::invalid_argument(
            "constant-stratification vertical benchmark requires an even square horizontal grid and Nz >= 3.");
    w.fields = 4;
    report.fields = 4;
    const int prec = precision_code(o);
    const bool f32 = prec == SKB_PRECISION_FP32;
    const double tol = f32 ? 1e-5 : 1e-12;
    const std::uint64_t nz = w.nz, nxHalf = w.nx / 2 + 1, fullRows = w.ny * nxHalf;
    const auto modes = retained_modes(w);
    const std::uint64_t compactRows = modes.size(), es = f32 ? 8 : 16;
    report.verticalMatrixFamilyId = "wvm-constant-stratification-fftw-type1-v1";
    report.fullSpectrumBytes = fullRows * 4 * nz * es;
    report.retainedSpectrumBytes = compactRows * 4 * nz * es;
    report.modalSpectrumBytes = compactRows * report.nj * 4 * es;

    auto to_device = [&](const std::vector<cplx>& v, DeviceBuffer& d, void* stream) {
        std::vector<double> flat(2 * v.size());
        for (std::size_t i = 0; i < v.size(); ++i) {
            flat[2 * i] = v[i].real();
            flat[2 * i + 1] = v[i].imag();
        }
        if (f32) d.upload(narrow<float>(flat), stream);
        else d.upload(flat, stream);
    };
    auto from_device = [&](const DeviceBuffer& d, std::uint64_t count, void* stream) {
        return widen_complex(d, count, f32, stream);
    };
    auto as_used_c = [&](std::vector<cplx> v) {
        if (f32)
            for (auto& x : v) x = cplx(double(float(x.real())), double(float(x.imag())));
        return v;
    };

    // Handles and arenas for both row sets.
    struct Arena {
        std::uint64_t rows;
        skb_cs_vertical* h = nullptr;
        std::unique_ptr<DeviceBuffer> a3, a1;
    };
    Arena full{fullRows}, compact{compactRows};
    for (Arena* a : {&full, &compact}) {
        ok(skb_cs_vertical_create(a->rows, nz, prec, &a->h));
        a->a3 = std::make_unique<DeviceBuffer>(a->rows * 3 * nz * es);
        a->a1 = std::make_unique<DeviceBuffer>(a->rows * nz * es);
    }
    std::unique_ptr<skb_cs_vertical, int (*)(skb_cs_vertical*)> gFull(full.h, skb_cs_vertical_destroy),
        gCompact(compact.h, skb_cs_vertical_destroy);
    void* sFull = skb_cs_vertical_stream(full.h);
    void* sCompact = skb_cs_vertical_stream(compact.h);

    // Correctness probes on compact row 0, channel 0 (541-556).
    auto probe = [&](bool sine) {
        const auto input = as_used_c(type1::fill_compact(modes, nxHalf, 1, nz));
        to_device(input, *compact.a1, sCompact);
        ok(skb_cs_vertical_transform_device(compact.h, sine ? SKB_TYPE1_DST : SKB_TYPE1_DCT, 1, 0, 1, 1,
                                            compact.a1->p, sCompact));
        const auto got = from_device(*compact.a1, nz, sCompact);
        const std::vector<cplx> column(input.begin(), input.begin() + nz);
        const auto want = type1::direct(column, sine);
        return std::make_pair(max_relative_error(got.data(), want.data(), nz),
                              relative_l2_error(got.data(), want.data(), nz));
    };
    const auto dctErr = probe(false);
    const auto dstErr = probe(true);

    // The call schedule on both row sets, compact against full (558-568).
    to_device(as_used_c(type1::fill_full(fullRows, 3, nz)), *full.a3, sFull);
    to_device(as_used_c(type1::fill_full(fullRows, 1, nz)), *full.a1, sFull);
    to_device(as_used_c(type1::fill_compact(modes, nxHalf, 3, nz)), *compact.a3, sCompact);
    to_device(as_used_c(type1::fill_compact(modes, nxHalf, 1, nz)), *compact.a1, sCompact);
    ok(skb_cs_vertical_schedule_device(full.h, full.a3->p, full.a1->p, sFull));
    ok(skb_cs_vertical_schedule_device(compact.h, compact.a3->p, compact.a1->p, sCompact));
    const auto three = type1::compact_vs_full(from_device(*compact.a3, compactRows * 3 * nz, sCompact),
                                              from_device(*full.a3, fullRows * 3 * nz, sFull), modes, nxHalf, 3, nz);
    const auto oneErr = type1::compact_vs_full(from_device(*compact.a1, compactRows * nz, sCompact),
                                            from_device(*full.a1, fullRows * nz, sFull), modes, nxHalf, 1, nz);

    auto record = [&](bool isCompact) {
        Arena& a = isCompact ? compact : full;
        void* stream = isCompact ? sCompact : sFull;
        ProviderRecord rec;
        skb_provider_info info{};
        ok(skb_cs_vertical_info(a.h, &info));
        fill_info(rec, info);
        rec.id = isCompact ? "cuda-wvm-type1-retained-compact" : "cuda-wvm-type1-full-half";
        rec.algorithmId = isCompact ? "retained-rows-production-type1-call-graph"
                                    : "wvm-full-half-production-type1-call-graph";
        rec.nativeRepresentationId = isCompact ? "retained-radial-interleaved-complex-z-adjacent"
                                               : "wvm-full-half-interleaved-complex-z-adjacent";
        rec.modeOrderId = isCompact ? "logical-radial-retained-mode-order" : "wvm-half-spectrum-row-order";
        rec.planningConfiguration = std::string(info.library_identity) + "; one launch per call-graph step";
        rec.persistentBytes = info.persistent_bytes + a.a3->bytes + a.a1->bytes;
        rec.forward.nativePlacement = "in-place";
        rec.forward.adapterPlacement = "in-place";
        rec.forward.destroysNativeInput = true;
        rec.forward.adapterPreservesCallerInput = false;
        rec.forward.physicalExtents = "[rows,channels,Nz] with Nz adjacent";
        rec.forward.stridesElements = "complex: z=1, channel=Nz, row=Nz*channels; real/imag stride=1 scalar";
        rec.forward.aliasing = "exact in-place alias";
        rec.inverse = rec.forward;
        to_device(as_used_c(type1::fill_full(a.rows, 3, nz)), *a.a3, stream);
        to_device(as_used_c(type1::fill_full(a.rows, 1, nz)), *a.a1, stream);
        const std::uint64_t one = a.rows * nz * es;
        auto raw = [&](bool sine) {
            return measure_device(o.warmups, o.samples, stream, [&] {
                ok(skb_cs_vertical_transform_device(a.h, sine ? SKB_TYPE1_DST : SKB_TYPE1_DCT, 1, 0, 1, 0, a.a1->p,
                                                    stream));
            });
        };
        rec.timings.push_back(series("primitive", "raw DCT-I one complex channel", "inverse", 2 * one, raw(false)));
        rec.timings.push_back(
            series("primitive", "raw DST-I one complex interior channel", "inverse", 2 * one, raw(true)));
        rec.timings.push_back(series("primitive", "raw DCT-I one complex channel", "forward", 2 * one, raw(false)));
        rec.timings.push_back(
            series("primitive", "raw DST-I one complex interior channel", "forward", 2 * one, raw(true)));
        auto norm = [&](bool sine) {
            return measure_device(o.warmups, o.samples, stream, [&] {
                ok(skb_cs_vertical_normalize_device(a.h, sine ? SKB_TYPE1_DST : SKB_TYPE1_DCT, 1, 0, 1, a.a1->p,
                                                    stream));
            });
        };
        rec.timings.push_back(
            series("adapter-component", "WVM forward DCT-I normalization", "forward", 2 * one, norm(false)));
        rec.timings.push_back(series("adapter-component", "WVM forward DST-I normalization and endpoints", "forward",
                                     2 * one, norm(true)));
        rec.timings.push_back(series(
            "uninstrumented-total",
            "production nonlinear-flux vertical transform schedule (15 inverse + 4 forward complex channels)",
            "complete", 38 * one, measure_device(o.warmups, o.samples, stream, [&] {
                ok(skb_cs_vertical_schedule_device(a.h, a.a3->p, a.a1->p, stream));
            })));
        rec.ledger = {
            {"setup/planning", StageState::setupOnly, "twiddles of the 2(Nz-1)-point symmetric extension"},
            {"raw inverse vertical transforms", StageState::executed,
             "15 complex channels in 5 launches (DCT-I and DST-I channels of one arena share a launch)"},
            {"raw forward vertical transforms", StageState::executed, "four complex flux-target projections"},
            {"forward normalization", StageState::fused,
             "exact WVM type-I endpoint and 1/(Nz-1) scaling, in the forward transform's store"},
            {"horizontal retained transforms", StageState::unsupported,
             "isolated vertical call-graph benchmark; composed horizontal timing is deferred"},
            {"coefficient assembly and pointwise products", StageState::unsupported,
             "not part of this attributable vertical component benchmark"}};
        rec.correctness.push_back(
            metric("WVM normalized DCT-I versus direct oracle", dctErr.first, dctErr.second, tol));
        rec.correctness.push_back(
            metric("WVM normalized DST-I versus direct oracle", dstErr.first, dstErr.second, tol));
        if (isCompact) {
            rec.correctness.push_back(metric("retained three-channel vertical call schedule versus full-half control",
                                             three.first, three.second, tol));
            rec.correctness.push_back(metric("retained one-channel projection schedule versus full-half control",
                                             oneErr.first, oneErr.second, tol));
        }
        return rec;
    };
    return {record(false), record(true)};
}

int flux_mode(const std::string& m) {
    if (m == "fp64-plain") return SKB_FLUX_FP64_PLAIN;
    if (m == "fp32") return SKB_FLUX_FP32;
    if (m == "split-tf32x3") return SKB_FLUX_SPLIT_TF32X3;
    if (m == "split-bf16x3") return SKB_FLUX_SPLIT_BF16X3;
    throw std::invalid_argument("flux-mode must be 'fp64-plain', 'fp32', 'split-tf32x3' or 'split-bf16x3'.");
}

// runAuthoritativeProductionLifetimeFluxBenchmark (src/authoritative_spectral_flux.cpp:
// 1409-1571): the 15 -> 4 flux with the prepared fixture's wave-f / wave-g
// operators over its floating groups, checked against the fixture's expected
// modal targets (1e-12 FP64-plain, 1e-6 split).  Loading and reordering stay
// outside every timed region.
ProviderRecord run_flux_fixture(const Options& o, const skb_workload& w, Report& report) {
    const auto modes = retained_modes(w);
    const auto loadStart = std::chrono::steady_clock::now();
    const PreparedFixture fx = load_prepared_fixture(o.fluxFixture, modes);
    const double loadSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - loadStart).count();
    if (fx.nx != w.nx || fx.ny != w.ny || fx.nz != w.nz)
        throw std::invalid_argument("Prepared spectral-flux fixture dimensions do not match the selected profile.");
    const int mode = flux_mode(o.fluxMode);
    const bool f64 = mode == SKB_FLUX_FP64_PLAIN;
    skb_flux_options fo{w.nx, w.nz, 4, 1, mode, SKB_FAMILY_K2_ROTATION, 0};
    skb_flux_families fam{};
    fam.groups = fx.groupModes.size();
    fam.group_modes = fx.groupModes.data();
    for (int f = 0; f < 2; ++f) {
        fam.forward[f] = fx.forward[f].data();
        fam.inverse[f] = fx.inverse[f].data();
    }
    for (int i = 0; i < 15; ++i) fam.input_family[i] = fx.inputFamily[i];
    for (int i = 0; i < 4; ++i) fam.target_family[i] = fx.targetFamily[i];
    skb_flux* h = nullptr;
    ok(skb_flux_create_families(&fo, &fam, &h));
    std::unique_ptr<skb_flux, int (*)(skb_flux*)> guard(h, skb_flux_destroy);
    void* stream = skb_flux_stream(h);
    std::uint64_t nModes = 0, nj = 0, inN = 0, outN = 0;
    ok(skb_flux_sizes(h, &nModes, &nj, &inN, &outN));
    skb_provider_info info{};
    ok(skb_flux_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    rec.otherSetupSeconds += loadSeconds;
    rec.algorithmId = std::string(f64 ? "staged" : "split-TF32x3") +
                      " flux with wave-f / wave-g operators: one GEMM launch per family and direction";
    rec.nativeRepresentationId = "modal [mode][field][j] interleaved";
    rec.modeOrderId = "radial-two-thirds-sorted(radius,k,l); floating K^2 operator groups";
    rec.planningConfiguration = o.fluxMode + "; fixture " + fx.fixtureId + " (" + fx.fixtureHash + "); " +
                                std::to_string(fx.groupModes.size()) + " operator groups from " +
                                std::to_string(fx.sourceGroups) + " fixture groups";
    rec.gemmCallsPerExecution = 4;
    rec.forward.nativePlacement = "out-of-place device arrays";
    rec.forward.adapterPlacement = "out-of-place host arrays";
    rec.inverse.nativePlacement = rec.inverse.adapterPlacement = "unsupported";
    rec.inverse.physicalExtents = "the composition exposes one 15-to-4 forward flux boundary only";
    report.verticalMatrixFamilyId = "wvm-wave-f+wave-g-floating-k2-exact";
    report.verticalGroupCount = fx.groupModes.size();
    report.fields = 4;

    const std::uint64_t s = f64 ? 8 : 4;
    std::vector<double> x(2 * inN);
    for (std::uint64_t i = 0; i < inN; ++i) {
        x[2 * i] = fx.modalInputs[i].real();
        x[2 * i + 1] = fx.modalInputs[i].imag();
    }
    DeviceBuffer dIn(inN * 2 * s), dOut(outN * 2 * s);
    if (f64) dIn.upload(x, stream);
    else dIn.upload(narrow<float>(x), stream);
    const std::uint64_t bytes = (inN + outN) * 2 * s;
    rec.timings.push_back(series("primitive", "authoritative production-lifetime four-target spectral-flux composition",
                                 "forward", bytes, measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_flux_execute_device(h, dIn.p, dOut.p, stream));
                                 })));
    ok(skb_flux_capture_graph(h, dIn.p, dOut.p));
    rec.timings.push_back(series("uninstrumented-total",
                                 "authoritative production-lifetime four-target spectral-flux composition (CUDA graph)",
                                 "forward", bytes, measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_flux_replay_graph(h, stream));
                                 })));
    std::vector<double> got(2 * outN);
    rec.timings.push_back(series("adapter-total", "authoritative spectral-flux composition (host arrays)", "forward",
                                 bytes, measure_host(o.warmups, o.samples, [&] {
                                     ok(skb_flux_execute(h, reinterpret_cast<const skb_complex*>(x.data()),
                                                         reinterpret_cast<skb_complex*>(got.data())));
                                 })));
    ok(skb_flux_check_device(h));
    std::vector<cplx> actual(outN), expected(outN);
    for (std::uint64_t i = 0; i < outN; ++i) {
        actual[i] = cplx(got[2 * i], got[2 * i + 1]);
        expected[i] = fx.expectedTargets[i];
    }
    const double tol = f64 ? 1e-12 : 1e-6;
    rec.correctness.push_back(metric("four modal targets versus the fixture's expected outputs",
                                     max_relative_error(actual.data(), expected.data(), outN),
                                     relative_l2_error(actual.data(), expected.data(), outN), tol));
    rec.ledger = {{"fixture load and validation", StageState::setupOnly, "outside every timed region"},
                  {"vertical inverse", StageState::executed, "one launch per operator family"},
                  {"vertical forward", StageState::executed, "one launch per operator family"}};
    (void)nModes;
    (void)nj;
    return rec;
}

// Modal inputs as the reference's production-lifetime fixture draws them:
// uniform in [-1/8, 1/8], the DC mode's imaginary part zero.
std::vector<double> flux_inputs(const std::vector<skb_retained_mode>& modes, std::uint64_t fieldsIn, std::uint64_t nj,
                                std::uint64_t members, std::uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-0.125, 0.125);
    const std::uint64_t perMember = modes.size() * fieldsIn * nj;
    std::vector<double> x(2 * members * perMember);
    for (std::uint64_t mem = 0; mem < members; ++mem)
        for (std::uint64_t m = 0; m < modes.size(); ++m)
            for (std::uint64_t f = 0; f < fieldsIn * nj; ++f) {
                const std::uint64_t i = mem * perMember + m * fieldsIn * nj + f;
                x[2 * i] = u(rng);
                x[2 * i + 1] = (modes[m].k == 0 && modes[m].l == 0) ? 0.0 : u(rng);
            }
    return x;
}

std::vector<cplx> host_flux(std::uint64_t n, std::uint64_t nz, std::uint64_t targets,
                            const std::vector<skb_retained_mode>& modes, const std::vector<skb_mode_group>& groups,
                            const std::vector<double>& fwd, const std::vector<double>& inv, const std::vector<double>& x);

ProviderRecord run_flux(const Options& o, const skb_workload& w, Report& report) {
    if (w.nx != w.ny) throw std::invalid_argument("production-lifetime-flux needs Nx = Ny.");
    const int mode = flux_mode(o.fluxMode);
    const bool f64 = mode == SKB_FLUX_FP64_PLAIN;
    skb_flux_options fo{w.nx, w.nz, o.targets, o.members, mode, SKB_FAMILY_K2_ROTATION, o.seed};
    skb_flux* h = nullptr;
    ok(skb_flux_create(&fo, &h));
    std::unique_ptr<skb_flux, int (*)(skb_flux*)> guard(h, skb_flux_destroy);
    void* stream = skb_flux_stream(h);
    std::uint64_t nModes = 0, nj = 0, inN = 0, outN = 0;
    ok(skb_flux_sizes(h, &nModes, &nj, &inN, &outN));
    skb_provider_info info{};
    ok(skb_flux_info(h, &info));
    ProviderRecord rec;
    fill_info(rec, info);
    const bool split = mode == SKB_FLUX_SPLIT_TF32X3 || mode == SKB_FLUX_SPLIT_BF16X3;
    rec.algorithmId = split ? std::string("fused five-launch flux: tcgen05 ") +
                                  (mode == SKB_FLUX_SPLIT_TF32X3 ? "TF32x3" : "BF16x3") +
                                  " GEMMs, embed+columns, register-resident rows, columns+retention"
                          : "staged flux: grouped GEMM, pruned horizontal, pointwise, pruned horizontal, grouped GEMM";
    rec.nativeRepresentationId = "modal [member][mode][field][j] interleaved";
    rec.modeOrderId = "radial-two-thirds-sorted(radius,k,l); K^2 groups contiguous";
    rec.planningConfiguration = o.fluxMode + "; members " + std::to_string(o.members) + "; targets " +
                                std::to_string(o.targets) + "; K^2 pair-rotation family; scale 1/(Nx*Ny)^2";
    rec.gemmCallsPerExecution = 2;
    rec.forward.nativePlacement = "out-of-place device arrays";
    rec.forward.adapterPlacement = "out-of-place host arrays";
    rec.inverse.nativePlacement = rec.inverse.adapterPlacement = "unsupported";
    rec.inverse.physicalExtents = "the composition exposes one 15-to-4 forward flux boundary only";

    const auto modes = retained_modes(w);
    const auto x = flux_inputs(modes, 3 + 3 * o.targets, nj, o.members, o.seed);
    const std::uint64_t s = f64 ? 8 : 4;
    DeviceBuffer dIn(inN * 2 * s), dOut(outN * 2 * s);
    if (f64) dIn.upload(x, stream);
    else dIn.upload(narrow<float>(x), stream);
    const std::uint64_t bytes = (inN + outN) * 2 * s;
    if (o.autotune) {
        // Launch shapes from the project autotuner, measured on these buffers
        // before any timing; the tuning time counts as planning.
        std::vector<char> summary(8192);
        ok(skb_flux_autotune(h, dIn.p, dOut.p, summary.data(), summary.size()));
        ok(skb_flux_info(h, &info));
        rec.planningSeconds = info.planning_seconds;
        std::string choices;
        for (const char* line = summary.data(); *line;) {
            const char* end = std::strchr(line, '\n');
            std::string entry(line, end ? end : line + std::strlen(line));
            const auto bar = entry.find(" | ");
            const auto eq = entry.find(" = ");
            if (bar != std::string::npos && eq != std::string::npos)
                entry = entry.substr(0, bar) + entry.substr(eq);
            choices += (choices.empty() ? "" : "; ") + entry;
            if (!end) break;
            line = end + 1;
        }
        rec.planningConfiguration += "; autotuned: " + (choices.empty() ? std::string("no tuned shapes") : choices);
    }
    rec.timings.push_back(series("primitive", "production-lifetime streamed four-target spectral-flux composition",
                                 "forward", bytes, measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_flux_execute_device(h, dIn.p, dOut.p, stream));
                                 })));
    ok(skb_flux_capture_graph(h, dIn.p, dOut.p));
    rec.timings.push_back(series("uninstrumented-total",
                                 "production-lifetime streamed four-target spectral-flux composition (CUDA graph)",
                                 "forward", bytes, measure_device(o.warmups, o.samples, stream, [&] {
                                     ok(skb_flux_replay_graph(h, stream));
                                 })));
    std::vector<skb_stage_time> stages(32);
    std::uint64_t count = 0;
    ok(skb_flux_profile(h, dIn.p, dOut.p, stages.data(), stages.size(), &count));
    for (std::uint64_t i = 0; i < count; ++i)
        rec.timings.push_back(series("primitive-component", stages[i].name, "forward",
                                     std::uint64_t(stages[i].algorithmic_bytes), {stages[i].ms * 1e-3}));
    rec.ledger = {{"shared U,V,W reconstruction", StageState::executed, "once per composition"},
                  {"derivative reconstruction", StageState::executed, "per target"},
                  {"pointwise advection", split ? StageState::fused : StageState::executed,
                   split ? "inside the row kernel" : "separate kernel"},
                  {"forward horizontal and retention", StageState::executed, "per target"},
                  {"forward vertical GEMM", StageState::executed, "all targets in one launch"}};
    if (o.autotune)
        rec.ledger.push_back({"autotune", StageState::setupOnly, "launch shapes measured on the run's own buffers"});
    ok(skb_flux_check_device(h));

    // Correctness.  FP64-plain: member 0 against the direct host composition
    // where that is cheap (Nx <= 64), else against the independent split
    // path at its 1e-6 tolerance.  Reduced-precision modes: against
    // FP64-plain on the same inputs.
    if (f64 && w.nx <= 64) {
        ok(skb_flux_execute_device(h, dIn.p, dOut.p, stream));
        ok(skb_stream_synchronize(stream));
        const auto got = widen_complex(dOut, outN, false, stream);
        const skb_workload wf{w.nx, w.nx, w.nz, 1, 1.0, 1.0, 1};
        const auto groups = k2_groups(wf);
        const std::uint64_t perGroup = nj * w.nz;
        std::vector<double> fwd(groups.size() * perGroup), inv(groups.size() * perGroup);
        std::uint64_t familyGroups = 0;
        char id[128] = {};
        ok(skb_vertical_family(&wf, SKB_FAMILY_K2_ROTATION, o.seed, fwd.data(), inv.data(), fwd.size(), &familyGroups,
                               id));
        const std::vector<double> x0(x.begin(), x.begin() + 2 * (inN / o.members));
        const auto want = host_flux(w.nx, w.nz, o.targets, modes, groups, fwd, inv, x0);
        rec.correctness.push_back(metric("fp64-plain member 0 vs direct host composition",
                                         max_relative_error(got.data(), want.data(), want.size()),
                                         relative_l2_error(got.data(), want.data(), want.size()), 1e-12));
    } else if (f64) {
        skb_flux_options other = fo;
        other.mode = SKB_FLUX_SPLIT_TF32X3;
        skb_flux* hs = nullptr;
        ok(skb_flux_create(&other, &hs));
        std::unique_ptr<skb_flux, int (*)(skb_flux*)> guardS(hs, skb_flux_destroy);
        void* ss = skb_flux_stream(hs);
        DeviceBuffer dInS(inN * 8), dOutS(outN * 8);
        dInS.upload(narrow<float>(x), ss);
        ok(skb_flux_execute_device(hs, dInS.p, dOutS.p, ss));
        ok(skb_stream_synchronize(ss));
        ok(skb_flux_execute_device(h, dIn.p, dOut.p, stream));
        ok(skb_stream_synchronize(stream));
        const auto want = widen_complex(dOut, outN, false, stream);
        const auto got = widen_complex(dOutS, outN, true, ss);
        rec.correctness.push_back(metric("split-tf32x3 cross-check of fp64-plain", max_relative_error(got.data(), want.data(), outN),
                                         relative_l2_error(got.data(), want.data(), outN), 1e-6));
    } else {
        skb_flux_options ref = fo;
        ref.mode = SKB_FLUX_FP64_PLAIN;
        skb_flux* h64 = nullptr;
        ok(skb_flux_create(&ref, &h64));
        std::unique_ptr<skb_flux, int (*)(skb_flux*)> guard64(h64, skb_flux_destroy);
        void* s64 = skb_flux_stream(h64);
        DeviceBuffer dIn64(inN * 16), dOut64(outN * 16);
        dIn64.upload(x, s64);
        ok(skb_flux_execute_device(h64, dIn64.p, dOut64.p, s64));
        ok(skb_stream_synchronize(s64));
        ok(skb_flux_execute_device(h, dIn.p, dOut.p, stream));
        ok(skb_stream_synchronize(stream));
        const auto want = widen_complex(dOut64, outN, false, s64);
        const auto got = widen_complex(dOut, outN, true, stream);
        const double tol = split ? 1e-6 : 1e-4;
        rec.correctness.push_back(metric(o.fluxMode + " vs fp64-plain", max_relative_error(got.data(), want.data(), outN),
                                         relative_l2_error(got.data(), want.data(), outN), tol));
    }
    report.verticalMatrixFamilyId = "k2-pair-rotation";
    return rec;
}

// ------------------------------------------------------------ validate

// Host composition of the 15 -> 4 flux for one member with direct
// transforms: inverse vertical, embed, c2r, pointwise products, r2c, gather,
// forward vertical (the order of src/benchmark.cpp:4405-4424).
std::vector<cplx> host_flux(std::uint64_t n, std::uint64_t nz, std::uint64_t targets,
                            const std::vector<skb_retained_mode>& modes, const std::vector<skb_mode_group>& groups,
                            const std::vector<double>& fwd, const std::vector<double>& inv, const std::vector<double>& x) {
    const std::uint64_t fieldsIn = 3 + 3 * targets, nj = 2 * (nz - 1) / 3, H = modes.size();
    std::vector<std::uint64_t> groupOf(H);
    for (std::uint64_t g = 0; g < groups.size(); ++g)
        for (std::uint64_t m = 0; m < groups[g].mode_count; ++m) groupOf[groups[g].first_mode + m] = g;
    skb_workload wIn{n, n, nz, fieldsIn, 1.0, 1.0, 1};
    std::vector<cplx> retained(H * fieldsIn * nz);
    for (std::uint64_t m = 0; m < H; ++m)
        for (std::uint64_t f = 0; f < fieldsIn; ++f)
            for (std::uint64_t z = 0; z < nz; ++z) {
                long double re = 0, im = 0;
                for (std::uint64_t j = 0; j < nj; ++j) {
                    const long double a = inv[(groupOf[m] * nz + z) * nj + j];
                    const std::uint64_t i = (m * fieldsIn + f) * nj + j;
                    re += a * x[2 * i];
                    im += a * x[2 * i + 1];
                }
                retained[(m * fieldsIn + f) * nz + z] = cplx(double(re), double(im));
            }
    const auto spectrum = embed(wIn, modes, retained.data());
    const auto real = direct_c2r(wIn, spectrum.data());
    const std::uint64_t V = n * n * nz;
    const double scale = 1.0 / double(n * n) / double(n * n);
    skb_workload wOut{n, n, nz, targets, 1.0, 1.0, 1};
    std::vector<double> r(targets * V);
    for (std::uint64_t t = 0; t < targets; ++t)
        for (std::uint64_t i = 0; i < V; ++i) {
            long double acc = 0;
            for (int c = 0; c < 3; ++c)
                acc += static_cast<long double>(real[c * V + i]) * real[(3 + 3 * t + c) * V + i];
            r[t * V + i] = double(-scale * acc);
        }
    const auto outSpec = direct_r2c(wOut, r.data());
    const auto outRet = gather(wOut, modes, outSpec.data());
    std::vector<cplx> out(H * targets * nj);
    for (std::uint64_t m = 0; m < H; ++m)
        for (std::uint64_t t = 0; t < targets; ++t)
            for (std::uint64_t j = 0; j < nj; ++j) {
                long double re = 0, im = 0;
                for (std::uint64_t z = 0; z < nz; ++z) {
                    const long double a = fwd[(groupOf[m] * nj + j) * nz + z];
                    const cplx v = outRet[(m * targets + t) * nz + z];
                    re += a * v.real();
                    im += a * v.imag();
                }
                out[(m * targets + t) * nj + j] = cplx(double(re), double(im));
            }
    return out;
}

int validate(const std::string& profileName) {
    const auto requested = profile_named(profileName);
    const skb_workload w = requested.name == "smoke" ? requested.w : skb_workload{8, 8, 7, 2, 1.0, 1.0, 1};
    const double tol = 1e-12;
    const char* names[] = {"impulse", "sinusoid", "random", "dc", "nyquist"};
    const auto modes = retained_modes(w);
    const std::uint64_t planes = w.nz * w.fields, realN = planes * w.nx * w.ny, half = w.nx / 2 + 1;
    const std::uint64_t specN = planes * w.ny * half, retN = modes.size() * planes;
    bool passed = true;
    auto report = [&](const std::string& what, double err, double limit) {
        const bool good = std::isfinite(err) && err <= limit;
        passed = passed && good;
        std::cout << what << "=" << std::scientific << std::setprecision(6) << err << (good ? "" : " FAILED") << '\n';
    };
    skb_fft_provider* fft = nullptr;
    ok(skb_fft_create(&w, SKB_PRECISION_FP64, &fft));
    std::unique_ptr<skb_fft_provider, int (*)(skb_fft_provider*)> g1(fft, skb_fft_destroy);
    skb_pruned_provider* pruned = nullptr;
    ok(skb_pruned_create(&w, SKB_PRECISION_FP64, &pruned));
    std::unique_ptr<skb_pruned_provider, int (*)(skb_pruned_provider*)> g2(pruned, skb_pruned_destroy);
    for (int k = 0; k < 5; ++k) {
        std::vector<double> input(realN);
        ok(skb_make_fixture(&w, k, 129 + k, input.data()));
        const auto oracle = direct_r2c(w, input.data());
        std::vector<skb_complex> spec(specN);
        ok(skb_fft_forward(fft, input.data(), spec.data()));
        const auto* got = reinterpret_cast<const cplx*>(spec.data());
        report(std::string("cuda/") + names[k] + "/forward", max_relative_error(got, oracle.data(), specN), tol);
        std::vector<double> back(realN);
        ok(skb_fft_inverse(fft, reinterpret_cast<skb_complex*>(const_cast<cplx*>(oracle.data())), back.data()));
        report(std::string("cuda/") + names[k] + "/inverse",
               max_relative_error(back.data(), input.data(), realN, 1.0 / double(w.nx * w.ny)), tol);
        const auto retOracle = gather(w, modes, oracle.data());
        std::vector<skb_complex> ret(retN);
        ok(skb_pruned_forward(pruned, input.data(), ret.data()));
        report(std::string("cuda-pruned/") + names[k] + "/forward",
               max_relative_error(reinterpret_cast<const cplx*>(ret.data()), retOracle.data(), retN), tol);
        const auto embedded = embed(w, modes, retOracle.data());
        const auto invOracle = direct_c2r(w, embedded.data());
        ok(skb_pruned_inverse(pruned, reinterpret_cast<const skb_complex*>(retOracle.data()), back.data()));
        report(std::string("cuda-pruned/") + names[k] + "/inverse",
               max_relative_error(back.data(), invOracle.data(), realN, 1.0), tol);
    }
    // Vertical GEMM on the common DCT-II family against the direct product.
    {
        const std::uint64_t nz = w.nz, nj = 2 * (nz - 1) / 3, cols = modes.size() * w.fields;
        std::vector<double> fwd(nj * nz), inv(nz * nj);
        std::uint64_t groupsOut = 0;
        char id[128] = {};
        ok(skb_vertical_family(&w, SKB_FAMILY_COMMON_DCT2, 0, fwd.data(), inv.data(), fwd.size(), &groupsOut, id));
        skb_mode_group all{0, 0, modes.size()};
        skb_vertical_provider* v = nullptr;
        ok(skb_vertical_create(&w, &all, 1, fwd.data(), inv.data(), SKB_LAYOUT_INTERLEAVED, SKB_BUFFERS_BIDIRECTIONAL,
                               SKB_GEMM_FP64, &v));
        std::unique_ptr<skb_vertical_provider, int (*)(skb_vertical_provider*)> g3(v, skb_vertical_destroy);
        std::mt19937_64 rng(129);
        std::uniform_real_distribution<double> u(-1, 1);
        std::vector<cplx> phys(cols * nz), modal(cols * nj), want(cols * nj);
        for (auto& c : phys) c = cplx(u(rng), u(rng));
        for (std::uint64_t c = 0; c < cols; ++c)
            for (std::uint64_t j = 0; j < nj; ++j) {
                lcplx s = 0;
                for (std::uint64_t z = 0; z < nz; ++z)
                    s += static_cast<long double>(fwd[j * nz + z]) * lcplx(phys[c * nz + z].real(), phys[c * nz + z].imag());
                want[c * nj + j] = cplx(double(s.real()), double(s.imag()));
            }
        ok(skb_vertical_load_physical_input(v, reinterpret_cast<const skb_complex*>(phys.data())));
        ok(skb_vertical_execute_forward(v));
        ok(skb_vertical_copy_forward_output(v, reinterpret_cast<skb_complex*>(modal.data())));
        report("cuda-vertical/" + std::string(id) + "/forward", max_relative_error(modal.data(), want.data(), modal.size()),
               tol);
    }
    // The 15 -> 4 flux, FP64-plain and split-TF32x3, against the host composition.
    {
        const std::uint64_t n = 32, nz = 9, targets = 4;
        const skb_workload wf{n, n, nz, 1, 1.0, 1.0, 1};
        const auto fm = retained_modes(wf);
        const auto groups = k2_groups(wf);
        const std::uint64_t nj = 2 * (nz - 1) / 3;
        std::vector<double> fwd(groups.size() * nj * nz), inv(groups.size() * nz * nj);
        std::uint64_t familyGroups = 0;
        char id[128] = {};
        ok(skb_vertical_family(&wf, SKB_FAMILY_K2_ROTATION, 129, fwd.data(), inv.data(), fwd.size(), &familyGroups, id));
        const auto x = flux_inputs(fm, 3 + 3 * targets, nj, 1, 129);
        const auto want = host_flux(n, nz, targets, fm, groups, fwd, inv, x);
        for (const int mode : {SKB_FLUX_FP64_PLAIN, SKB_FLUX_SPLIT_TF32X3}) {
            skb_flux_options fo{n, nz, targets, 1, mode, SKB_FAMILY_K2_ROTATION, 129};
            skb_flux* h = nullptr;
            ok(skb_flux_create(&fo, &h));
            std::unique_ptr<skb_flux, int (*)(skb_flux*)> g4(h, skb_flux_destroy);
            std::vector<skb_complex> out(want.size());
            ok(skb_flux_execute(h, reinterpret_cast<const skb_complex*>(x.data()), out.data()));
            const auto* got = reinterpret_cast<const cplx*>(out.data());
            report(std::string("cuda-flux/") + (mode == SKB_FLUX_FP64_PLAIN ? "fp64-plain" : "split-tf32x3") + "/32x32x9",
                   max_relative_error(got, want.data(), want.size()), mode == SKB_FLUX_FP64_PLAIN ? tol : 1e-6);
        }
    }
    std::cout << (passed ? "validation passed" : "validation FAILED") << '\n';
    return passed ? 0 : 1;
}

// ----------------------------------------------------------------- CLI

void usage(std::ostream& out) {
    out << "Usage:\n"
        << "  skbench-cuda list\n"
        << "  skbench-cuda validate [--profile NAME]\n"
        << "  skbench-cuda run [--kernel fft|2d-rfft|pruned-horizontal|vertical-gemm|pointwise-advection|"
           "production-lifetime-flux|spectral-pipeline|constant-stratification-vertical] [--profile NAME]\n"
           "              [--providers cuda]\n"
        << "              [--precision fp64|fp32] [--vertical-gemm-family common|k2-grouped]\n"
        << "              [--vertical-gemm-precision fp64|fp32|tf32x3|bf16x3]\n"
        << "              [--flux-mode fp64-plain|fp32|split-tf32x3|split-bf16x3]\n"
        << "              [--members N] [--targets 3|4] [--autotune] [--nx N --ny N --nz N --fields N]\n"
        << "              [--spectral-flux-fixture PREPARED.bin]\n"
        << "              [--boundary-policy NAME] [--streaming-tile-width N] [--streaming-inverse-policy NAME]\n"
        << "              [--warmups N] [--samples N] [--seed N] [--output PATH]\n"
        << "  skbench-cuda compare --input SAMPLES.csv\n";
}

void list() {
    std::cout << "schema: spectral-kernel-benchmark-v1\nprofiles:\n";
    for (const auto& p : profiles())
        std::cout << "  " << p.name << ": " << p.w.nx << 'x' << p.w.ny << ", Nz=" << p.w.nz << ", fields=" << p.w.fields
                  << "\n    " << p.purpose << '\n';
    std::cout << "providers:\n  cuda: " << skb_version() << "\n"
              << "kernels:\n  fft (alias 2d-rfft)\n  pruned-horizontal\n  vertical-gemm\n  pointwise-advection\n"
              << "  production-lifetime-flux\n  spectral-pipeline\n  constant-stratification-vertical\n"
              << "precisions:\n  fp64\n  fp32\n"
              << "vertical GEMM precisions:\n  fp64\n  fp32\n  tf32x3\n  bf16x3\n"
              << "vertical GEMM matrix families:\n  common\n  k2-grouped\n"
              << "flux modes:\n  fp64-plain\n  fp32\n  split-tf32x3\n  split-bf16x3\n";
}

std::string value(int argc, char** argv, int& i) {
    if (i + 1 >= argc) throw std::invalid_argument("Missing value after " + std::string(argv[i]));
    return argv[++i];
}

int run(int argc, char** argv) {
    Options o;
    for (int i = 2; i < argc; ++i) {
        const std::string_view k = argv[i];
        if (k == "--kernel") o.kernel = value(argc, argv, i);
        else if (k == "--profile") o.profile = value(argc, argv, i);
        else if (k == "--providers") o.providers = value(argc, argv, i);
        else if (k == "--precision") o.precision = value(argc, argv, i);
        else if (k == "--vertical-gemm-family") o.family = value(argc, argv, i);
        else if (k == "--vertical-gemm-precision") o.gemm = value(argc, argv, i);
        else if (k == "--flux-mode") o.fluxMode = value(argc, argv, i);
        else if (k == "--members") o.members = std::stoull(value(argc, argv, i));
        else if (k == "--targets") o.targets = std::stoull(value(argc, argv, i));
        else if (k == "--nx") o.nx = std::stoull(value(argc, argv, i));
        else if (k == "--ny") o.ny = std::stoull(value(argc, argv, i));
        else if (k == "--nz") o.nz = std::stoull(value(argc, argv, i));
        else if (k == "--fields") o.fields = std::stoull(value(argc, argv, i));
        else if (k == "--warmups") {
            o.warmups = std::stoull(value(argc, argv, i));
            o.warmupsSet = true;
        } else if (k == "--samples") {
            o.samples = std::stoull(value(argc, argv, i));
            o.samplesSet = true;
        } else if (k == "--seed") o.seed = std::stoull(value(argc, argv, i));
        else if (k == "--output") o.output = value(argc, argv, i);
        else if (k == "--autotune") o.autotune = true;
        else if (k == "--spectral-flux-fixture") o.fluxFixture = value(argc, argv, i);
        else if (k == "--boundary-policy") o.boundaryPolicy = value(argc, argv, i);
        else if (k == "--streaming-tile-width") o.tileWidth = std::stoull(value(argc, argv, i));
        else if (k == "--streaming-inverse-policy") o.inversePolicy = value(argc, argv, i);
        else throw std::invalid_argument("Unknown run option: " + std::string(k));
    }
    if (o.kernel == "2d-rfft") o.kernel = "fft";
    check_streaming_options(o);
    if (!o.fluxFixture.empty() && o.kernel != "production-lifetime-flux")
        throw std::invalid_argument("--spectral-flux-fixture is valid only for production-lifetime-flux.");
    if (o.providers != "cuda" && o.providers != "both")
        throw std::invalid_argument("providers must be 'cuda' (this binary provides no other).");
    const auto prof = profile_named(o.profile);
    skb_workload w = prof.w;
    if (o.nx) w.nx = o.nx;
    if (o.ny) w.ny = o.ny;
    if (o.nz) w.nz = o.nz;
    if (o.fields) w.fields = o.fields;
    if (!o.warmupsSet) o.warmups = prof.warmups;
    if (!o.samplesSet) o.samples = prof.samples;
    if (o.samples == 0) throw std::invalid_argument("samples must be positive.");
    Report report = base_report(o, prof, w);
    std::vector<ProviderRecord> records;
    ProviderRecord rec;
    if (o.kernel == "constant-stratification-vertical") records = run_constant_stratification(o, w, report);
    else if (o.kernel == "fft") rec = run_fft(o, w, report);
    else if (o.kernel == "pruned-horizontal") rec = run_pruned(o, w, report);
    else if (o.kernel == "vertical-gemm") rec = run_vertical(o, w, report);
    else if (o.kernel == "pointwise-advection") rec = run_pointwise(o, w, report);
    else if (o.kernel == "production-lifetime-flux" && !o.fluxFixture.empty()) rec = run_flux_fixture(o, w, report);
    else if (o.kernel == "production-lifetime-flux") rec = run_flux(o, w, report);
    else if (o.kernel == "spectral-pipeline") rec = run_pipeline(o, w, report);
    else
        throw std::invalid_argument(
            "kernel must be 'fft', '2d-rfft', 'pruned-horizontal', 'vertical-gemm', 'pointwise-advection', "
            "'production-lifetime-flux', 'spectral-pipeline' or 'constant-stratification-vertical'.");
    if (records.empty()) records.push_back(rec);
    if (!o.boundaryPolicy.empty() || o.tileWidth != 1 || o.inversePolicy != "full-zero") {
        const std::string detail = "boundary policy '" + (o.boundaryPolicy.empty() ? "default" : o.boundaryPolicy) +
                                   "', tile width " + std::to_string(o.tileWidth) + ", inverse preparation '" +
                                   o.inversePolicy +
                                   "': recorded only; the GPU column embed rebuilds each column band from the "
                                   "retained values in one pass, so these CPU scratch strategies have no "
                                   "counterpart and do not change the result";
        for (auto& r : records) r.ledger.push_back({"streaming preparation options", StageState::elided, detail});
    }
    for (auto& r : records) {
        r.compilerFlags = "nvcc -gencode arch=compute_100a,code=sm_100a -O3";
        r.sourceIdentity = std::string("libskb_cuda ") + skb_version();
        for (const auto& m : r.correctness)
            if (!m.passed) report.status = "failed";
        report.providers.push_back(r);
    }

    std::filesystem::path json = o.output.empty() ? std::filesystem::path("results/local") / (report.runId + ".json")
                                                  : std::filesystem::path(o.output);
    auto csv = json;
    csv.replace_extension(".csv");
    if (!json.parent_path().empty()) std::filesystem::create_directories(json.parent_path());
    {
        std::ofstream out(json);
        if (!out) throw std::runtime_error("Unable to open JSON result: " + json.string());
        write_json(report, out);
    }
    {
        std::ofstream out(csv);
        if (!out) throw std::runtime_error("Unable to open CSV result: " + csv.string());
        write_csv(report, out);
    }
    std::cout << "run " << report.runId << " status=" << report.status << " profile=" << report.profile
              << " workload=" << w.nx << 'x' << w.ny << " Nz=" << w.nz << " fields=" << w.fields
              << " Nkl=" << report.nkl << '\n';
    std::cout << "provider\tscope\tstage\tdirection\tmedian_ms\n";
    for (const auto& r : report.providers)
        for (const auto& t : r.timings) {
            if (t.seconds.empty()) continue;
            std::cout << r.id << '\t' << t.scope << '\t' << t.stage << '\t' << t.direction << '\t' << std::fixed
                      << std::setprecision(6) << 1000.0 * median(t.seconds) << '\n';
        }
    for (const auto& r : report.providers)
        for (const auto& m : r.correctness)
            std::cout << r.id << " correctness " << m.name << '=' << std::scientific << m.maximumRelativeError
                      << " passed=" << (m.passed ? "true" : "false") << '\n';
    std::cout << "json=" << std::filesystem::absolute(json).string() << '\n';
    std::cout << "csv=" << std::filesystem::absolute(csv).string() << '\n';
    return report.status == "passed" ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc < 2) {
            usage(std::cerr);
            return 2;
        }
        const std::string_view command = argv[1];
        if (command == "list") {
            if (argc != 2) throw std::invalid_argument("list accepts no arguments.");
            list();
            return 0;
        }
        if (command == "validate") {
            std::string profile = "smoke";
            for (int i = 2; i < argc; ++i) {
                const std::string_view k = argv[i];
                if (k == "--profile") profile = value(argc, argv, i);
                else throw std::invalid_argument("Unknown validate option: " + std::string(k));
            }
            return validate(profile);
        }
        if (command == "run") return run(argc, argv);
        if (command == "compare") {
            std::string input;
            for (int i = 2; i < argc; ++i) {
                const std::string_view k = argv[i];
                if (k == "--input") input = value(argc, argv, i);
                else if (input.empty() && k.substr(0, 2) != "--") input = std::string(k);
                else throw std::invalid_argument("Unknown compare option: " + std::string(k));
            }
            if (input.empty()) throw std::invalid_argument("compare requires --input SAMPLES.csv.");
            std::ifstream in(input);
            if (!in) throw std::runtime_error("Unable to open CSV result: " + input);
            return compare_csv(in, std::cout);
        }
        usage(std::cerr);
        throw std::invalid_argument("Unknown command: " + std::string(command));
    } catch (const std::exception& e) {
        std::cerr << "skbench-cuda: " << e.what() << '\n';
        return 2;
    }
}
