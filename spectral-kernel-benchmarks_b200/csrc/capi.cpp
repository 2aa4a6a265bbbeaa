// extern "C" entry points of include/skb_cuda.h.

#include "skb_cuda.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "autotune.hpp"
#include "flux.hpp"
#include "noalloc.hpp"
#include "peaks.hpp"
#include "pipeline.hpp"
#include "server.hpp"
#include "pointwise.hpp"
#include "runtime.hpp"
#include "type1.hpp"
#include "util.hpp"

using namespace skb;

namespace {

thread_local std::string g_lastError;

template <typename F>
int guard(F&& body) {
    try {
        body();
        return SKB_OK;
    } catch (const Error& e) {
        g_lastError = e.what();
        return e.code();
    } catch (const std::invalid_argument& e) {
        g_lastError = e.what();
        return SKB_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc& e) {
        g_lastError = e.what();
        return SKB_ERR_OUT_OF_MEMORY;
    } catch (const std::logic_error& e) {
        g_lastError = e.what();
        return SKB_ERR_LOGIC;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return SKB_ERR_RUNTIME;
    }
}

void require(bool ok, const char* what) {
    if (!ok) throw Error(SKB_ERR_INVALID_ARGUMENT, what);
}

Workload to_workload(const skb_workload* w) {
    require(w != nullptr, "workload must be non-null");
    Workload out{w->nx, w->ny, w->nz, w->fields, w->lx, w->ly, w->antialias != 0};
    validate_workload(out);
    return out;
}

Precision to_precision(int p) {
    if (p == SKB_PRECISION_FP64) return Precision::f64;
    if (p == SKB_PRECISION_FP32) return Precision::f32;
    throw Error(SKB_ERR_INVALID_ARGUMENT, "precision must be SKB_PRECISION_FP64 or SKB_PRECISION_FP32");
}

cudaStream_t make_stream() {
    cudaStream_t s = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    return s;
}

void copy_in(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
}

void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync D2H");
}

void sync(cudaStream_t s) { check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize"); }

ViewSet to_views(const skb_field_view* views, uint64_t count, uint64_t nz) {
    require(views != nullptr || count == 0, "field views must be non-null");
    require(count <= static_cast<uint64_t>(kMaxViews), "too many field views");
    ViewSet v{};
    v.count = static_cast<int>(count);
    for (uint64_t i = 0; i < count; ++i) {
        require(views[i].real != nullptr, "field view pointers must be non-null");
        require(views[i].mode_stride >= nz, "field view mode stride must be at least Nz");
        v.v[i] = {views[i].real, views[i].imag, static_cast<long long>(views[i].mode_stride)};
    }
    return v;
}

// Default retained layout [mode][field][z] as one interleaved view per field.
ViewSet retained_views(void* base, const Workload& w, size_t complexBytes) {
    ViewSet v{};
    v.count = static_cast<int>(w.fields);
    for (uint64_t f = 0; f < w.fields; ++f)
        v.v[f] = {static_cast<unsigned char*>(base) + complexBytes * f * w.nz, nullptr,
                  static_cast<long long>(w.planes())};
    return v;
}

ViewSet retained_split_views(void* re, void* im, const Workload& w, size_t realBytes) {
    ViewSet v{};
    v.count = static_cast<int>(w.fields);
    for (uint64_t f = 0; f < w.fields; ++f)
        v.v[f] = {static_cast<unsigned char*>(re) + realBytes * f * w.nz,
                  static_cast<unsigned char*>(im) + realBytes * f * w.nz, static_cast<long long>(w.planes())};
    return v;
}

void fill_identity(skb_provider_info* info, const char* identity) {
    std::strncpy(info->library_identity, identity, sizeof(info->library_identity) - 1);
    std::strncpy(info->version, skb_version(), sizeof(info->version) - 1);
}

// Host doubles <-> device values of precision p through a staging buffer.
struct HostAdapter {
    Precision p;
    DeviceBuffer staging;  // doubles, used only for f32 handles
    void ensure(size_t doubles) {
        if (p == Precision::f32 && staging.bytes() < doubles * sizeof(double)) staging.allocate(doubles * sizeof(double));
    }
    void upload(void* dst, const double* src, size_t n, cudaStream_t s) {
        if (p == Precision::f64) {
            copy_in(dst, src, n * sizeof(double), s);
            return;
        }
        ensure(n);
        copy_in(staging.get(), src, n * sizeof(double), s);
        check_cuda(launch_convert_f64_to_f32(staging.get<double>(), static_cast<float*>(dst), (long long)n, s),
                   "convert kernel");
    }
    void download(double* dst, const void* src, size_t n, cudaStream_t s) {
        if (p == Precision::f64) {
            copy_out(dst, src, n * sizeof(double), s);
            return;
        }
        ensure(n);
        check_cuda(launch_convert_f32_to_f64(static_cast<const float*>(src), staging.get<double>(), (long long)n, s),
                   "convert kernel");
        copy_out(dst, staging.get(), n * sizeof(double), s);
    }
};

}  // namespace

// ------------------------------------------------------------------ handles

struct skb_fft_provider {
    Workload w;
    Precision p;
    cudaStream_t stream = nullptr;
    std::unique_ptr<HorizontalPlan> plan;
    DeviceBuffer real, spectrum, retained, splitRe, splitIm;
    HostAdapter host{Precision::f64, {}};
    double otherSetup = 0.0, allocation = 0.0;
    ~skb_fft_provider() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_pruned_provider {
    Workload w;
    Precision p;
    cudaStream_t stream = nullptr;
    std::unique_ptr<HorizontalPlan> plan;
    DeviceBuffer real, retained, retainedIm;
    HostAdapter host{Precision::f64, {}};
    double otherSetup = 0.0, allocation = 0.0;
    ~skb_pruned_provider() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_vertical_provider {
    Workload w;
    int layout = SKB_LAYOUT_INTERLEAVED;
    int policy = SKB_BUFFERS_BIDIRECTIONAL;
    GemmPrecision gp = GemmPrecision::f64;
    Precision p = Precision::f64;
    cudaStream_t stream = nullptr;
    std::unique_ptr<VerticalPlan> forward, inverse;
    uint64_t columns = 0, groups = 0;
    DeviceBuffer physIn, physInIm, modalOut, modalOutIm, modalIn, modalInIm, physOut, physOutIm;
    HostAdapter host{Precision::f64, {}};
    double allocation = 0.0, preparation = 0.0;
    ~skb_vertical_provider() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_vertical_wvm_provider {
    Workload w;
    GemmPrecision gp = GemmPrecision::f64;
    Precision p = Precision::f64;
    cudaStream_t stream = nullptr;
    std::unique_ptr<VerticalPlan> forward, inverse;
    // Per retained mode: element offsets of its stored cell in the WVM
    // spectrum and in the WVM modal spectrum, and of the kx = 0 partner cell.
    DeviceBuffer cellSpec, partnerSpec, cellModal, partnerModal;
    DeviceBuffer spectrum, modal;  // device staging of the host forms
    HostAdapter host{Precision::f64, {}};
    uint64_t spectrumElements = 0, modalElements = 0;
    double allocation = 0.0, preparation = 0.0;
    ~skb_vertical_wvm_provider() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_pipeline {
    std::unique_ptr<SpectralPipeline> pipe;
    cudaStream_t stream = nullptr;
    DeviceBuffer in, out;  // device staging of the host form
    HostAdapter host{Precision::f64, {}};
    ~skb_pipeline() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_pointwise_executor {
    uint64_t volume = 0;
    double scale = 0.0;
    Precision p = Precision::f64;
    cudaStream_t stream = nullptr;
    DeviceBuffer shared, derivative, target;
    HostAdapter host{Precision::f64, {}};
    ~skb_pointwise_executor() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_flux {
    std::unique_ptr<FluxPipeline> pipeline;
    cudaStream_t stream = nullptr;
    DeviceBuffer in, out;
    HostAdapter host{Precision::f64, {}};
    // Host-array path: copy streams, FP64 staging of the FP32 forms, and one
    // pair of events per member (input landed / result ready).
    cudaStream_t copyIn = nullptr, copyOut = nullptr;
    DeviceBuffer stageIn, stageOut;
    std::vector<cudaEvent_t> landed, ready;
    ~skb_flux() {
        pipeline.reset();
        for (auto e : landed) cudaEventDestroy(e);
        for (auto e : ready) cudaEventDestroy(e);
        if (copyIn) cudaStreamDestroy(copyIn);
        if (copyOut) cudaStreamDestroy(copyOut);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_cs_vertical {
    uint64_t rows = 0, nz = 0;
    Precision p = Precision::f64;
    cudaStream_t stream = nullptr;
    DeviceBuffer tw;        // 2(nz-1) twiddles exp(-2 pi i m / (2(nz-1)))
    DeviceBuffer arena, arena1;  // device staging of host arrays
    HostAdapter host{Precision::f64, {}};
    double allocation = 0.0, planning = 0.0;
    ~skb_cs_vertical() {
        if (stream) cudaStreamDestroy(stream);
    }
};

struct skb_timer {
    cudaEvent_t start = nullptr, stop = nullptr;
    ~skb_timer() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
    }
};

extern "C" {

const char* skb_last_error(void) { return g_lastError.c_str(); }

const char* skb_version(void) { return "skb-cuda 0.1.0 (sm_100a)"; }

int skb_device_count(int* count) {
    return guard([&] {
        require(count != nullptr, "count must be non-null");
        check_cuda(cudaGetDeviceCount(count), "cudaGetDeviceCount");
    });
}

int skb_set_device(int device) {
    return guard([&] { check_cuda(cudaSetDevice(device), "cudaSetDevice"); });
}

int skb_device_synchronize(void) {
    return guard([&] { check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); });
}

int skb_measure_simt_peaks(double* fp32_tflops, double* fp64_tflops) {
    return guard([&] {
        require(fp32_tflops != nullptr && fp64_tflops != nullptr, "outputs must be non-null");
        check_cuda(measure_simt_peaks(fp32_tflops, fp64_tflops), "SIMT peak measurement");
    });
}

// ------------------------------------------------------------------- model

int skb_retained_modes(const skb_workload* w, skb_retained_mode* out, uint64_t capacity, uint64_t* count) {
    return guard([&] {
        const auto modes = retained_modes(to_workload(w));
        require(count != nullptr, "count must be non-null");
        *count = modes.size();
        if (out == nullptr) return;
        require(capacity >= modes.size(), "retained mode capacity too small");
        for (size_t i = 0; i < modes.size(); ++i)
            out[i] = {modes[i].k, modes[i].l, modes[i].kx, modes[i].ky, modes[i].conj ? 1 : 0, modes[i].radial};
    });
}

int skb_squared_wavenumber_groups(const skb_workload* w, skb_mode_group* out, uint64_t capacity, uint64_t* count) {
    return guard([&] {
        const auto groups = squared_wavenumber_groups(retained_modes(to_workload(w)));
        require(count != nullptr, "count must be non-null");
        *count = groups.size();
        if (out == nullptr) return;
        require(capacity >= groups.size(), "group capacity too small");
        for (size_t i = 0; i < groups.size(); ++i) out[i] = {groups[i].key, groups[i].first, groups[i].count};
    });
}

int skb_order_hashes(const skb_workload* w, char* mode_hash, char* group_hash, char* wvm_hash) {
    return guard([&] {
        const auto wl = to_workload(w);
        const auto modes = retained_modes(wl);
        auto put = [](char* dst, const std::string& s) {
            if (dst) std::snprintf(dst, 32, "%s", s.c_str());
        };
        put(mode_hash, mode_order_hash(modes));
        put(group_hash, group_order_hash(squared_wavenumber_groups(modes)));
        if (wvm_hash) put(wvm_hash, wvm_order_hash(wl));
    });
}

int skb_make_fixture(const skb_workload* w, int kind, uint64_t seed, double* out) {
    return guard([&] {
        require(out != nullptr, "output must be non-null");
        require(kind >= 0 && kind <= 4, "fixture kind must be 0..4");
        const auto values = make_fixture(to_workload(w), kind, seed);
        std::memcpy(out, values.data(), values.size() * sizeof(double));
    });
}

int skb_vertical_family(const skb_workload* w, int family, uint64_t seed, double* forward, double* inverse,
                        uint64_t capacity, uint64_t* groups, char* id) {
    return guard([&] {
        const auto wl = to_workload(w);
        VerticalFamily fam;
        if (family == SKB_FAMILY_COMMON_DCT2) {
            fam = orthonormal_family(wl.nz, wl.nj());
        } else {
            const auto g = squared_wavenumber_groups(retained_modes(wl));
            if (family == SKB_FAMILY_K2_ROTATION)
                fam = k2_rotation_family(wl, g);
            else if (family == SKB_FAMILY_STURM_LIOUVILLE)
                fam = sturm_liouville_family(wl, g, seed);
            else
                throw Error(SKB_ERR_INVALID_ARGUMENT, "unknown vertical family");
        }
        if (groups) *groups = fam.groups;
        if (id) std::snprintf(id, 96, "%s", fam.id.c_str());
        if (forward == nullptr && inverse == nullptr) return;
        require(capacity >= fam.forward.size(), "vertical family capacity too small");
        if (forward) std::memcpy(forward, fam.forward.data(), fam.forward.size() * sizeof(double));
        if (inverse) std::memcpy(inverse, fam.inverse.data(), fam.inverse.size() * sizeof(double));
    });
}

// --------------------------------------------------------------------- FFT

int skb_fft_create(const skb_workload* w, int precision, skb_fft_provider** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        auto p = std::make_unique<skb_fft_provider>();
        const auto t0 = Clock::now();
        p->w = to_workload(w);
        p->p = to_precision(precision);
        p->stream = make_stream();
        p->otherSetup = seconds_since(t0);
        p->plan = std::make_unique<HorizontalPlan>(p->w, p->p, false, p->w.planes());
        const auto t1 = Clock::now();
        const size_t es = element_bytes(p->p);
        p->real.allocate(es * p->w.realElements());
        p->spectrum.allocate(2 * es * p->w.spectrumElements());
        p->retained.allocate(2 * es * std::max<uint64_t>(1, p->plan->modes() * p->w.planes()));
        p->host.p = p->p;
        p->allocation = seconds_since(t1) + p->plan->allocationSeconds;
        *out = p.release();
    });
}

int skb_fft_destroy(skb_fft_provider* p) {
    return guard([&] { delete p; });
}

int skb_fft_info(const skb_fft_provider* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->allocation_seconds = p->allocation;
        info->planning_seconds = p->plan->planningSeconds;
        info->other_setup_seconds = p->otherSetup;
        info->persistent_bytes = p->plan->persistentBytes;
        info->scratch_bytes = p->plan->scratchBytes;
        info->planning_bytes = 0;
        info->active_kx = p->w.nxHalf();
        info->full_kx = p->w.nxHalf();
        info->row_transforms_per_direction = p->w.ny * p->w.planes();
        info->column_transforms_per_direction = p->w.nxHalf() * p->w.planes();
        info->launches_per_execution = 2;
        info->precision = p->p == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        info->destroys_native_input = 0;
        fill_identity(info, "skb-cuda hand-written sm_100a row/column shared-memory FFT");
    });
}

void* skb_fft_stream(skb_fft_provider* p) { return p ? p->stream : nullptr; }

int skb_fft_forward_device(skb_fft_provider* p, const void* real, void* wvm, void* stream) {
    return guard([&] {
        require(p && real && wvm, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->forward_dense(real, wvm, p->w.planes(), s);
    });
}

int skb_fft_inverse_device(skb_fft_provider* p, const void* wvm, void* real, void* stream) {
    return guard([&] {
        require(p && real && wvm, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->inverse_dense(wvm, real, p->w.planes(), s);
    });
}

int skb_fft_inverse_device_noalloc(const skb_workload* w, int precision, const void* wvm, void* real, void* stream) {
    return guard([&] {
        require(wvm && real, "buffers must be non-null");
        inverse_dense_static(to_workload(w), to_precision(precision), wvm, real, static_cast<cudaStream_t>(stream));
    });
}

int skb_fft_gather_retained_device(skb_fft_provider* p, const void* wvm, const skb_field_view* views,
                                   uint64_t count, double scale, void* stream) {
    return guard([&] {
        require(p && wvm, "handle and buffers must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->gather_dense(wvm, p->w.planes(), to_views(views, count, p->w.nz), scale, s);
    });
}

int skb_fft_embed_retained_device(skb_fft_provider* p, const skb_field_view* views, uint64_t count, void* wvm,
                                  void* stream) {
    return guard([&] {
        require(p && wvm, "handle and buffers must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->embed_dense(to_views(views, count, p->w.nz), wvm, p->w.planes(), s);
    });
}

int skb_fft_forward(skb_fft_provider* p, const double* input, skb_complex* wvm) {
    return guard([&] {
        require(p && input && wvm, "handle and buffers must be non-null");
        p->host.upload(p->real.get(), input, p->w.realElements(), p->stream);
        p->plan->forward_dense(p->real.get(), p->spectrum.get(), p->w.planes(), p->stream);
        p->host.download(reinterpret_cast<double*>(wvm), p->spectrum.get(), 2 * p->w.spectrumElements(), p->stream);
        sync(p->stream);
    });
}

int skb_fft_inverse(skb_fft_provider* p, skb_complex* wvm, double* output) {
    return guard([&] {
        require(p && wvm && output, "handle and buffers must be non-null");
        p->host.upload(p->spectrum.get(), reinterpret_cast<const double*>(wvm), 2 * p->w.spectrumElements(),
                       p->stream);
        p->plan->inverse_dense(p->spectrum.get(), p->real.get(), p->w.planes(), p->stream);
        p->host.download(output, p->real.get(), p->w.realElements(), p->stream);
        sync(p->stream);
    });
}

int skb_fft_forward_split(skb_fft_provider* p, const double* input, double* re, double* im) {
    return guard([&] {
        require(p && input && re && im, "handle and buffers must be non-null");
        const auto n = p->w.spectrumElements();
        const size_t es = element_bytes(p->p);
        if (p->splitRe.bytes() < n * es) {
            p->splitRe.allocate(n * es);
            p->splitIm.allocate(n * es);
        }
        p->host.upload(p->real.get(), input, p->w.realElements(), p->stream);
        p->plan->forward_dense(p->real.get(), p->spectrum.get(), p->w.planes(), p->stream);
        check_cuda(launch_split(p->p == Precision::f64, p->spectrum.get(), p->splitRe.get(), p->splitIm.get(),
                                (long long)n, p->stream),
                   "split kernel");
        p->host.download(re, p->splitRe.get(), n, p->stream);
        p->host.download(im, p->splitIm.get(), n, p->stream);
        sync(p->stream);
    });
}

int skb_fft_inverse_split(skb_fft_provider* p, double* re, double* im, double* output) {
    return guard([&] {
        require(p && re && im && output, "handle and buffers must be non-null");
        const auto n = p->w.spectrumElements();
        const size_t es = element_bytes(p->p);
        if (p->splitRe.bytes() < n * es) {
            p->splitRe.allocate(n * es);
            p->splitIm.allocate(n * es);
        }
        p->host.upload(p->splitRe.get(), re, n, p->stream);
        p->host.upload(p->splitIm.get(), im, n, p->stream);
        check_cuda(launch_interleave(p->p == Precision::f64, p->splitRe.get(), p->splitIm.get(), p->spectrum.get(),
                                     (long long)n, p->stream),
                   "interleave kernel");
        p->plan->inverse_dense(p->spectrum.get(), p->real.get(), p->w.planes(), p->stream);
        p->host.download(output, p->real.get(), p->w.realElements(), p->stream);
        sync(p->stream);
    });
}

int skb_fft_gather_retained(skb_fft_provider* p, const skb_complex* wvm, skb_complex* retained) {
    return guard([&] {
        require(p && wvm && retained, "handle and buffers must be non-null");
        const size_t ces = 2 * element_bytes(p->p);
        p->host.upload(p->spectrum.get(), reinterpret_cast<const double*>(wvm), 2 * p->w.spectrumElements(),
                       p->stream);
        p->plan->gather_dense(p->spectrum.get(), p->w.planes(), retained_views(p->retained.get(), p->w, ces), 1.0,
                              p->stream);
        p->host.download(reinterpret_cast<double*>(retained), p->retained.get(),
                         2 * p->plan->modes() * p->w.planes(), p->stream);
        sync(p->stream);
    });
}

int skb_fft_embed_retained(skb_fft_provider* p, const skb_complex* retained, skb_complex* wvm) {
    return guard([&] {
        require(p && wvm && retained, "handle and buffers must be non-null");
        const size_t ces = 2 * element_bytes(p->p);
        p->host.upload(p->retained.get(), reinterpret_cast<const double*>(retained),
                       2 * p->plan->modes() * p->w.planes(), p->stream);
        p->plan->embed_dense(retained_views(p->retained.get(), p->w, ces), p->spectrum.get(), p->w.planes(),
                             p->stream);
        p->host.download(reinterpret_cast<double*>(wvm), p->spectrum.get(), 2 * p->w.spectrumElements(), p->stream);
        sync(p->stream);
    });
}

int skb_fft_gather_retained_to_split(skb_fft_provider* p, const skb_complex* wvm, double* re, double* im,
                                     double scale) {
    return guard([&] {
        require(p && wvm && re && im, "handle and buffers must be non-null");
        const auto n = p->plan->modes() * p->w.planes();
        const size_t es = element_bytes(p->p);
        if (p->splitRe.bytes() < std::max<uint64_t>(n, p->w.spectrumElements()) * es) {
            p->splitRe.allocate(std::max<uint64_t>(n, p->w.spectrumElements()) * es);
            p->splitIm.allocate(std::max<uint64_t>(n, p->w.spectrumElements()) * es);
        }
        p->host.upload(p->spectrum.get(), reinterpret_cast<const double*>(wvm), 2 * p->w.spectrumElements(),
                       p->stream);
        p->plan->gather_dense(p->spectrum.get(), p->w.planes(),
                              retained_split_views(p->splitRe.get(), p->splitIm.get(), p->w, es), scale, p->stream);
        p->host.download(re, p->splitRe.get(), n, p->stream);
        p->host.download(im, p->splitIm.get(), n, p->stream);
        sync(p->stream);
    });
}

int skb_fft_embed_retained_from_split(skb_fft_provider* p, const double* re, const double* im, skb_complex* wvm) {
    return guard([&] {
        require(p && wvm && re && im, "handle and buffers must be non-null");
        const auto n = p->plan->modes() * p->w.planes();
        const size_t es = element_bytes(p->p);
        if (p->splitRe.bytes() < std::max<uint64_t>(n, p->w.spectrumElements()) * es) {
            p->splitRe.allocate(std::max<uint64_t>(n, p->w.spectrumElements()) * es);
            p->splitIm.allocate(std::max<uint64_t>(n, p->w.spectrumElements()) * es);
        }
        p->host.upload(p->splitRe.get(), re, n, p->stream);
        p->host.upload(p->splitIm.get(), im, n, p->stream);
        p->plan->embed_dense(retained_split_views(p->splitRe.get(), p->splitIm.get(), p->w, es), p->spectrum.get(),
                             p->w.planes(), p->stream);
        p->host.download(reinterpret_cast<double*>(wvm), p->spectrum.get(), 2 * p->w.spectrumElements(), p->stream);
        sync(p->stream);
    });
}

// ------------------------------------------------------------------ pruned

int skb_pruned_create(const skb_workload* w, int precision, skb_pruned_provider** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        auto p = std::make_unique<skb_pruned_provider>();
        const auto t0 = Clock::now();
        p->w = to_workload(w);
        p->p = to_precision(precision);
        p->stream = make_stream();
        p->otherSetup = seconds_since(t0);
        p->plan = std::make_unique<HorizontalPlan>(p->w, p->p, true, p->w.planes());
        const auto t1 = Clock::now();
        const size_t es = element_bytes(p->p);
        p->real.allocate(es * p->w.realElements());
        p->retained.allocate(2 * es * p->plan->modes() * p->w.planes());
        p->retainedIm.allocate(es * p->plan->modes() * p->w.planes());
        p->host.p = p->p;
        p->allocation = seconds_since(t1) + p->plan->allocationSeconds;
        *out = p.release();
    });
}

int skb_pruned_destroy(skb_pruned_provider* p) {
    return guard([&] { delete p; });
}

int skb_pruned_info(const skb_pruned_provider* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->allocation_seconds = p->allocation;
        info->planning_seconds = p->plan->planningSeconds;
        info->other_setup_seconds = p->otherSetup;
        info->persistent_bytes = p->plan->persistentBytes;
        info->scratch_bytes = p->plan->scratchBytes;
        info->active_kx = static_cast<uint64_t>(p->plan->keep());
        info->full_kx = p->w.nxHalf();
        info->row_transforms_per_direction = p->w.ny * p->w.planes();
        info->column_transforms_per_direction = info->active_kx * p->w.planes();
        info->omitted_column_transforms_per_direction = (info->full_kx - info->active_kx) * p->w.planes();
        info->launches_per_execution = 2;
        info->precision = p->p == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        fill_identity(info, "skb-cuda hand-written sm_100a pruned row/active-column FFT with fused retention");
    });
}

void* skb_pruned_stream(skb_pruned_provider* p) { return p ? p->stream : nullptr; }

int skb_pruned_forward_device(skb_pruned_provider* p, const void* real, const skb_field_view* fields, uint64_t count,
                              double scale, void* stream) {
    return guard([&] {
        require(p && real, "handle and buffers must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->forward(real, p->w.planes(), to_views(fields, count, p->w.nz), scale, s);
    });
}

int skb_pruned_inverse_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t count, void* real,
                              void* stream) {
    return guard([&] {
        require(p && real, "handle and buffers must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->inverse(to_views(fields, count, p->w.nz), real, s);
    });
}

int skb_pruned_forward_rows_device(skb_pruned_provider* p, const void* real, void* stream) {
    return guard([&] {
        require(p && real, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->forward_rows(real, p->w.planes(), s);
    });
}

int skb_pruned_forward_columns_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t count,
                                      double scale, void* stream) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->forward_columns(to_views(fields, count, p->w.nz), scale, s);
    });
}

int skb_pruned_inverse_columns_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t count,
                                      void* stream) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        require(count == p->w.fields, "one field view per workload field");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->inverse_columns(to_views(fields, count, p->w.nz), s);
    });
}

int skb_pruned_inverse_rows_device(skb_pruned_provider* p, void* real, void* stream) {
    return guard([&] {
        require(p && real, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->plan->inverse_rows(real, p->w.planes(), s);
    });
}

int skb_pruned_forward(skb_pruned_provider* p, const double* input, skb_complex* retained) {
    return guard([&] {
        require(p && input && retained, "handle and buffers must be non-null");
        const size_t ces = 2 * element_bytes(p->p);
        p->host.upload(p->real.get(), input, p->w.realElements(), p->stream);
        p->plan->forward(p->real.get(), p->w.planes(), retained_views(p->retained.get(), p->w, ces), 1.0, p->stream);
        p->host.download(reinterpret_cast<double*>(retained), p->retained.get(), 2 * p->plan->modes() * p->w.planes(),
                         p->stream);
        sync(p->stream);
    });
}

int skb_pruned_forward_split(skb_pruned_provider* p, const double* input, double* re, double* im, double scale) {
    return guard([&] {
        require(p && input && re && im, "handle and buffers must be non-null");
        const size_t es = element_bytes(p->p);
        const auto n = p->plan->modes() * p->w.planes();
        p->host.upload(p->real.get(), input, p->w.realElements(), p->stream);
        p->plan->forward(p->real.get(), p->w.planes(),
                         retained_split_views(p->retained.get(), p->retainedIm.get(), p->w, es), scale, p->stream);
        p->host.download(re, p->retained.get(), n, p->stream);
        p->host.download(im, p->retainedIm.get(), n, p->stream);
        sync(p->stream);
    });
}

int skb_pruned_inverse(skb_pruned_provider* p, const skb_complex* retained, double* output) {
    return guard([&] {
        require(p && output && retained, "handle and buffers must be non-null");
        const size_t ces = 2 * element_bytes(p->p);
        p->host.upload(p->retained.get(), reinterpret_cast<const double*>(retained),
                       2 * p->plan->modes() * p->w.planes(), p->stream);
        p->plan->inverse(retained_views(p->retained.get(), p->w, ces), p->real.get(), p->stream);
        p->host.download(output, p->real.get(), p->w.realElements(), p->stream);
        sync(p->stream);
    });
}

int skb_pruned_inverse_split(skb_pruned_provider* p, const double* re, const double* im, double* output) {
    return guard([&] {
        require(p && output && re && im, "handle and buffers must be non-null");
        const size_t es = element_bytes(p->p);
        const auto n = p->plan->modes() * p->w.planes();
        p->host.upload(p->retained.get(), re, n, p->stream);
        p->host.upload(p->retainedIm.get(), im, n, p->stream);
        p->plan->inverse(retained_split_views(p->retained.get(), p->retainedIm.get(), p->w, es), p->real.get(),
                         p->stream);
        p->host.download(output, p->real.get(), p->w.realElements(), p->stream);
        sync(p->stream);
    });
}

int skb_pruned_forward_split_fields(skb_pruned_provider* p, const double* input, const skb_field_view* fields,
                                    uint64_t count, double scale) {
    return guard([&] {
        require(p && input && fields, "handle and buffers must be non-null");
        require(count == p->w.fields, "Streaming pruned output field views must match the workload field count.");
        for (uint64_t f = 0; f < count; ++f)
            require(fields[f].real && fields[f].imag && fields[f].mode_stride >= p->w.nz,
                    "Streaming pruned output field view is invalid.");
        const size_t es = element_bytes(p->p);
        const auto H = p->plan->modes(), nz = p->w.nz;
        p->host.upload(p->real.get(), input, p->w.realElements(), p->stream);
        // Device-side compact split fields [field][mode][z], then strided copies out.
        ViewSet v{};
        v.count = static_cast<int>(count);
        for (uint64_t f = 0; f < count; ++f)
            v.v[f] = {p->retained.get<unsigned char>() + es * f * H * nz,
                      p->retainedIm.get<unsigned char>() + es * f * H * nz, static_cast<long long>(nz)};
        p->plan->forward(p->real.get(), p->w.planes(), v, scale, p->stream);
        if (p->p == Precision::f64) {
            for (uint64_t f = 0; f < count; ++f) {
                check_cuda(cudaMemcpy2DAsync(fields[f].real, fields[f].mode_stride * sizeof(double),
                                             p->retained.get<unsigned char>() + es * f * H * nz, nz * es, nz * es, H,
                                             cudaMemcpyDeviceToHost, p->stream),
                           "cudaMemcpy2DAsync");
                check_cuda(cudaMemcpy2DAsync(fields[f].imag, fields[f].mode_stride * sizeof(double),
                                             p->retainedIm.get<unsigned char>() + es * f * H * nz, nz * es, nz * es,
                                             H, cudaMemcpyDeviceToHost, p->stream),
                           "cudaMemcpy2DAsync");
            }
            sync(p->stream);
        } else {
            std::vector<double> re(H * nz), im(H * nz);
            for (uint64_t f = 0; f < count; ++f) {
                p->host.download(re.data(), p->retained.get<unsigned char>() + es * f * H * nz, H * nz, p->stream);
                p->host.download(im.data(), p->retainedIm.get<unsigned char>() + es * f * H * nz, H * nz, p->stream);
                sync(p->stream);
                auto* dr = static_cast<double*>(fields[f].real);
                auto* di = static_cast<double*>(fields[f].imag);
                for (uint64_t m = 0; m < H; ++m)
                    for (uint64_t z = 0; z < nz; ++z) {
                        dr[z + fields[f].mode_stride * m] = re[z + nz * m];
                        di[z + fields[f].mode_stride * m] = im[z + nz * m];
                    }
            }
        }
    });
}

int skb_pruned_inverse_split_fields(skb_pruned_provider* p, const skb_field_view* fields, uint64_t count,
                                    double* output) {
    return guard([&] {
        require(p && output && fields, "handle and buffers must be non-null");
        require(count == p->w.fields, "Streaming pruned input field views must match the workload field count.");
        for (uint64_t f = 0; f < count; ++f)
            require(fields[f].real && fields[f].imag && fields[f].mode_stride >= p->w.nz,
                    "Streaming pruned input field view is invalid.");
        const size_t es = element_bytes(p->p);
        const auto H = p->plan->modes(), nz = p->w.nz;
        std::vector<double> re(H * nz), im(H * nz);
        for (uint64_t f = 0; f < count; ++f) {
            const auto* sr = static_cast<const double*>(fields[f].real);
            const auto* si = static_cast<const double*>(fields[f].imag);
            for (uint64_t m = 0; m < H; ++m)
                for (uint64_t z = 0; z < nz; ++z) {
                    re[z + nz * m] = sr[z + fields[f].mode_stride * m];
                    im[z + nz * m] = si[z + fields[f].mode_stride * m];
                }
            p->host.upload(p->retained.get<unsigned char>() + es * f * H * nz, re.data(), H * nz, p->stream);
            p->host.upload(p->retainedIm.get<unsigned char>() + es * f * H * nz, im.data(), H * nz, p->stream);
            sync(p->stream);
        }
        ViewSet v{};
        v.count = static_cast<int>(count);
        for (uint64_t f = 0; f < count; ++f)
            v.v[f] = {p->retained.get<unsigned char>() + es * f * H * nz,
                      p->retainedIm.get<unsigned char>() + es * f * H * nz, static_cast<long long>(nz)};
        p->plan->inverse(v, p->real.get(), p->stream);
        p->host.download(output, p->real.get(), p->w.realElements(), p->stream);
        sync(p->stream);
    });
}

// ---------------------------------------------------------------- vertical

int skb_vertical_create(const skb_workload* w, const skb_mode_group* groups, uint64_t group_count,
                        const double* forward, const double* inverse, int layout, int policy, int gemm_precision,
                        skb_vertical_provider** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        require(groups != nullptr && group_count > 0, "Vertical GEMM requires at least one horizontal mode and field.");
        require(layout == SKB_LAYOUT_INTERLEAVED || layout == SKB_LAYOUT_SPLIT, "unknown layout");
        require(policy >= SKB_BUFFERS_BIDIRECTIONAL && policy <= SKB_BUFFERS_INVERSE_ONLY, "unknown buffer policy");
        auto p = std::make_unique<skb_vertical_provider>();
        p->w = to_workload(w);
        p->layout = layout;
        p->policy = policy;
        if (gemm_precision == SKB_GEMM_FP64) {
            p->gp = GemmPrecision::f64;
            p->p = Precision::f64;
        } else if (gemm_precision == SKB_GEMM_FP32) {
            p->gp = GemmPrecision::f32;
            p->p = Precision::f32;
        } else if (gemm_precision == SKB_GEMM_TF32X3 || gemm_precision == SKB_GEMM_BF16X3) {
            require(layout == SKB_LAYOUT_INTERLEAVED, "the split tensor-core forms take the interleaved layout");
            p->gp = gemm_precision == SKB_GEMM_TF32X3 ? GemmPrecision::tf32x3 : GemmPrecision::bf16x3;
            p->p = Precision::f32;
        } else {
            throw Error(SKB_ERR_INVALID_ARGUMENT, "unknown vertical GEMM precision");
        }
        p->host.p = p->p;
        const auto prepStart = Clock::now();
        std::vector<ModeGroup> g(group_count);
        uint64_t modes = 0;
        for (uint64_t i = 0; i < group_count; ++i) {
            g[i] = {groups[i].squared_mode_key, groups[i].first_mode, groups[i].mode_count};
            modes += groups[i].mode_count;
        }
        VerticalFamily fam;
        fam.nz = p->w.nz;
        fam.nj = p->w.nj();
        require(fam.nj > 0, "Vertical GEMM requires Nz >= 2.");
        const bool fwd = policy != SKB_BUFFERS_INVERSE_ONLY, inv = policy != SKB_BUFFERS_FORWARD_ONLY;
        require(!fwd || forward != nullptr, "forward matrices must be non-null");
        require(!inv || inverse != nullptr, "inverse matrices must be non-null");
        fam.groups = group_count;
        const auto elems = fam.nz * fam.nj * group_count;
        fam.forward.assign(elems, 0.0);
        fam.inverse.assign(elems, 0.0);
        if (fwd) std::memcpy(fam.forward.data(), forward, elems * sizeof(double));
        if (inv) std::memcpy(fam.inverse.data(), inverse, elems * sizeof(double));
        p->stream = make_stream();
        if (fwd)
            p->forward = std::make_unique<VerticalPlan>(p->gp, static_cast<int>(fam.nj), static_cast<int>(fam.nz), g,
                                                        p->w.fields, 1, fam.forward);
        if (inv)
            p->inverse = std::make_unique<VerticalPlan>(p->gp, static_cast<int>(fam.nz), static_cast<int>(fam.nj), g,
                                                        p->w.fields, 1, fam.inverse);
        p->preparation = seconds_since(prepStart);
        p->groups = group_count;
        p->columns = modes * p->w.fields;
        const auto allocStart = Clock::now();
        const size_t es = element_bytes(p->p);
        const size_t mult = layout == SKB_LAYOUT_SPLIT ? 1 : 2;
        if (fwd) {
            p->physIn.allocate(mult * es * p->columns * fam.nz);
            p->modalOut.allocate(mult * es * p->columns * fam.nj);
            if (layout == SKB_LAYOUT_SPLIT) {
                p->physInIm.allocate(es * p->columns * fam.nz);
                p->modalOutIm.allocate(es * p->columns * fam.nj);
            }
        }
        if (inv) {
            p->modalIn.allocate(mult * es * p->columns * fam.nj);
            p->physOut.allocate(mult * es * p->columns * fam.nz);
            if (layout == SKB_LAYOUT_SPLIT) {
                p->modalInIm.allocate(es * p->columns * fam.nj);
                p->physOutIm.allocate(es * p->columns * fam.nz);
            }
        }
        p->allocation = seconds_since(allocStart);
        *out = p.release();
    });
}

int skb_vertical_destroy(skb_vertical_provider* p) {
    return guard([&] { delete p; });
}

// ------------------------------------------------- WVM-direct vertical GEMM

int skb_vertical_wvm_create(const skb_workload* w, const skb_mode_group* groups, uint64_t group_count,
                            const double* forward, const double* inverse, int policy, int gemm_precision,
                            skb_vertical_wvm_provider** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        require(groups != nullptr && group_count > 0, "Direct WVM vertical GEMM requires modes, groups, and fields.");
        require(policy >= SKB_BUFFERS_BIDIRECTIONAL && policy <= SKB_BUFFERS_INVERSE_ONLY, "unknown buffer policy");
        auto p = std::make_unique<skb_vertical_wvm_provider>();
        p->w = to_workload(w);
        if (gemm_precision == SKB_GEMM_FP64) {
            p->gp = GemmPrecision::f64;
            p->p = Precision::f64;
        } else if (gemm_precision == SKB_GEMM_FP32) {
            p->gp = GemmPrecision::f32;
            p->p = Precision::f32;
        } else if (gemm_precision == SKB_GEMM_TF32X3 || gemm_precision == SKB_GEMM_BF16X3) {
            p->gp = gemm_precision == SKB_GEMM_TF32X3 ? GemmPrecision::tf32x3 : GemmPrecision::bf16x3;
            p->p = Precision::f32;
        } else {
            throw Error(SKB_ERR_INVALID_ARGUMENT, "unknown vertical GEMM precision");
        }
        p->host.p = p->p;
        const auto prepStart = Clock::now();
        const auto modes = retained_modes(p->w);
        std::vector<ModeGroup> g(group_count);
        uint64_t covered = 0;
        for (uint64_t i = 0; i < group_count; ++i) {
            g[i] = {groups[i].squared_mode_key, groups[i].first_mode, groups[i].mode_count};
            require(groups[i].mode_count > 0 && groups[i].first_mode == covered,
                    "Direct WVM vertical GEMM groups must be nonempty, contiguous, and cover the modes.");
            covered += groups[i].mode_count;
        }
        require(covered == modes.size(), "Direct WVM vertical GEMM groups do not cover every retained mode.");
        const uint64_t nz = p->w.nz, nj = p->w.nj(), fields = p->w.fields, half = p->w.nxHalf();
        require(nj > 0, "Vertical GEMM requires Nz >= 2.");
        const bool fwd = policy != SKB_BUFFERS_INVERSE_ONLY, inv = policy != SKB_BUFFERS_FORWARD_ONLY;
        require(!fwd || forward != nullptr, "forward matrices must be non-null");
        require(!inv || inverse != nullptr, "inverse matrices must be non-null");
        const auto elems = nz * nj * group_count;
        std::vector<double> F(fwd ? elems : 0), I(inv ? elems : 0);
        if (fwd) std::memcpy(F.data(), forward, elems * sizeof(double));
        if (inv) std::memcpy(I.data(), inverse, elems * sizeof(double));
        std::vector<long long> cs(modes.size()), ps(modes.size()), cm(modes.size()), pm(modes.size());
        for (size_t m = 0; m < modes.size(); ++m) {
            const auto& md = modes[m];
            const long long cell = static_cast<long long>(md.kx + half * md.ky);
            cs[m] = cell * static_cast<long long>(nz * fields);
            cm[m] = cell * static_cast<long long>(nj * fields);
            const bool partner = md.kx == 0 && md.ky != 0 && 2 * md.ky != p->w.ny;
            const long long pcell = static_cast<long long>(half * ((p->w.ny - md.ky) % p->w.ny));
            ps[m] = partner ? pcell * static_cast<long long>(nz * fields) : -1;
            pm[m] = partner ? pcell * static_cast<long long>(nj * fields) : -1;
        }
        p->preparation = seconds_since(prepStart);
        const auto allocStart = Clock::now();
        p->stream = make_stream();
        if (fwd)
            p->forward = std::make_unique<VerticalPlan>(p->gp, static_cast<int>(nj), static_cast<int>(nz), g, fields, 1, F);
        if (inv)
            p->inverse = std::make_unique<VerticalPlan>(p->gp, static_cast<int>(nz), static_cast<int>(nj), g, fields, 1, I);
        p->cellSpec = upload_vector(cs);
        p->partnerSpec = upload_vector(ps);
        p->cellModal = upload_vector(cm);
        p->partnerModal = upload_vector(pm);
        p->spectrumElements = p->w.spectrumElements();
        p->modalElements = half * p->w.ny * nj * fields;
        const size_t es = element_bytes(p->p);
        p->spectrum.allocate(2 * es * p->spectrumElements);
        p->modal.allocate(2 * es * p->modalElements);
        p->allocation = seconds_since(allocStart);
        *out = p.release();
    });
}

int skb_vertical_wvm_destroy(skb_vertical_wvm_provider* p) {
    return guard([&] { delete p; });
}

int skb_vertical_wvm_info(const skb_vertical_wvm_provider* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->allocation_seconds = p->allocation;
        info->planning_seconds = p->preparation;
        info->persistent_bytes = (p->forward ? p->forward->persistentBytes() : 0) +
                                 (p->inverse ? p->inverse->persistentBytes() : 0) + p->cellSpec.bytes() +
                                 p->partnerSpec.bytes() + p->cellModal.bytes() + p->partnerModal.bytes();
        info->scratch_bytes = p->spectrum.bytes() + p->modal.bytes();
        info->launches_per_execution = 1;
        info->precision = p->p == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        fill_identity(info, "skb-cuda hand-written sm_100a direct WVM-order per-mode grouped GEMM");
    });
}

int skb_vertical_wvm_sizes(const skb_vertical_wvm_provider* p, uint64_t* spectrum_elements, uint64_t* modal_elements) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        if (spectrum_elements) *spectrum_elements = p->spectrumElements;
        if (modal_elements) *modal_elements = p->modalElements;
    });
}

namespace {
BinBoundary wvm_boundary(const DeviceBuffer& cell, const DeviceBuffer& partner, uint64_t fields, uint64_t stride,
                         bool withPartner) {
    return {cell.get<long long>(), withPartner ? partner.get<long long>() : nullptr, nullptr, static_cast<int>(fields),
            static_cast<int>(stride)};
}

void wvm_forward(skb_vertical_wvm_provider* p, const void* spectrum, void* modal, cudaStream_t s) {
    const BinBoundary in = wvm_boundary(p->cellSpec, p->partnerSpec, p->w.fields, p->w.nz, false);
    const BinBoundary out = wvm_boundary(p->cellModal, p->partnerModal, p->w.fields, p->w.nj(), true);
    if (!p->forward) throw std::logic_error("Forward GEMM requested from an inverse-only direct WVM provider.");
    p->forward->execute({const_cast<void*>(spectrum), nullptr}, {modal, nullptr}, s, 1, &in, &out);
}

void wvm_inverse(skb_vertical_wvm_provider* p, const void* modal, void* spectrum, cudaStream_t s) {
    const BinBoundary in = wvm_boundary(p->cellModal, p->partnerModal, p->w.fields, p->w.nj(), false);
    const BinBoundary out = wvm_boundary(p->cellSpec, p->partnerSpec, p->w.fields, p->w.nz, true);
    if (!p->inverse) throw std::logic_error("Inverse GEMM requested from a forward-only direct WVM provider.");
    p->inverse->execute({const_cast<void*>(modal), nullptr}, {spectrum, nullptr}, s, 1, &in, &out);
}
}  // namespace

int skb_vertical_wvm_forward_device(skb_vertical_wvm_provider* p, const void* spectrum, void* modal, void* stream) {
    return guard([&] {
        require(p && spectrum && modal, "handle and buffers must be non-null");
        wvm_forward(p, spectrum, modal, stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

int skb_vertical_wvm_inverse_device(skb_vertical_wvm_provider* p, const void* modal, void* spectrum, void* stream) {
    return guard([&] {
        require(p && spectrum && modal, "handle and buffers must be non-null");
        wvm_inverse(p, modal, spectrum, stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

int skb_vertical_wvm_forward(skb_vertical_wvm_provider* p, const skb_complex* spectrum, skb_complex* modal) {
    return guard([&] {
        require(p && spectrum && modal, "handle and buffers must be non-null");
        // The output's cells without a retained mode keep the caller's values.
        p->host.upload(p->spectrum.get(), reinterpret_cast<const double*>(spectrum), 2 * p->spectrumElements, p->stream);
        p->host.upload(p->modal.get(), reinterpret_cast<const double*>(modal), 2 * p->modalElements, p->stream);
        wvm_forward(p, p->spectrum.get(), p->modal.get(), p->stream);
        p->host.download(reinterpret_cast<double*>(modal), p->modal.get(), 2 * p->modalElements, p->stream);
        sync(p->stream);
        p->forward->check_device_error();
    });
}

int skb_vertical_wvm_inverse(skb_vertical_wvm_provider* p, const skb_complex* modal, skb_complex* spectrum) {
    return guard([&] {
        require(p && spectrum && modal, "handle and buffers must be non-null");
        p->host.upload(p->modal.get(), reinterpret_cast<const double*>(modal), 2 * p->modalElements, p->stream);
        p->host.upload(p->spectrum.get(), reinterpret_cast<const double*>(spectrum), 2 * p->spectrumElements,
                       p->stream);
        wvm_inverse(p, p->modal.get(), p->spectrum.get(), p->stream);
        p->host.download(reinterpret_cast<double*>(spectrum), p->spectrum.get(), 2 * p->spectrumElements, p->stream);
        sync(p->stream);
        p->inverse->check_device_error();
    });
}

int skb_vertical_wvm_initialize_modal_output(const skb_vertical_wvm_provider* p, skb_complex* modal) {
    return guard([&] {
        require(p && modal, "handle and output must be non-null");
        std::memset(modal, 0, sizeof(skb_complex) * p->modalElements);
    });
}

int skb_vertical_wvm_initialize_spectrum_output(const skb_vertical_wvm_provider* p, skb_complex* spectrum) {
    return guard([&] {
        require(p && spectrum, "handle and output must be non-null");
        std::memset(spectrum, 0, sizeof(skb_complex) * p->spectrumElements);
    });
}

void* skb_vertical_wvm_stream(skb_vertical_wvm_provider* p) { return p ? p->stream : nullptr; }

// ------------------------------------------------------- spectral pipeline

int skb_modal_weights(const skb_workload* w, double* out) {
    return guard([&] {
        require(out != nullptr, "output must be non-null");
        const Workload wl = to_workload(w);
        const auto weights = synthetic_modal_weights(wl, retained_modes(wl));
        std::memcpy(out, weights.data(), weights.size() * sizeof(double));
    });
}

int skb_pipeline_create(const skb_workload* w, int precision, skb_pipeline** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        auto p = std::make_unique<skb_pipeline>();
        const Workload wl = to_workload(w);
        const Precision pr = to_precision(precision);
        p->pipe = std::make_unique<SpectralPipeline>(wl, pr);
        p->stream = make_stream();
        p->host.p = pr;
        const size_t es = element_bytes(pr);
        p->in.allocate(es * wl.realElements());
        p->out.allocate(es * wl.realElements());
        *out = p.release();
    });
}

int skb_pipeline_destroy(skb_pipeline* p) {
    return guard([&] { delete p; });
}

int skb_pipeline_info(const skb_pipeline* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->allocation_seconds = p->pipe->allocationSeconds;
        info->planning_seconds = p->pipe->planningSeconds;
        info->persistent_bytes = p->pipe->persistentBytes;
        info->scratch_bytes = p->pipe->scratchBytes + p->in.bytes() + p->out.bytes();
        info->launches_per_execution = 7;
        info->precision = p->pipe->precision() == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        fill_identity(info, p->pipe->precision() == Precision::f64
                                ? "skb-cuda spectral pipeline: FP64 pruned transforms, FP64 K2-grouped GEMMs"
                                : "skb-cuda spectral pipeline: FP32 pruned transforms, split-TF32x3 tcgen05 GEMMs");
    });
}

int skb_pipeline_execute_device(skb_pipeline* p, const void* real_in, void* real_out, void* stream) {
    return guard([&] {
        require(p && real_in && real_out, "handle and buffers must be non-null");
        p->pipe->execute(real_in, real_out, stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

int skb_pipeline_execute(skb_pipeline* p, const double* real_in, double* real_out) {
    return guard([&] {
        require(p && real_in && real_out, "handle and buffers must be non-null");
        const size_t n = p->pipe->workload().realElements();
        p->host.upload(p->in.get(), real_in, n, p->stream);
        p->pipe->execute(p->in.get(), p->out.get(), p->stream);
        p->host.download(real_out, p->out.get(), n, p->stream);
        sync(p->stream);
        p->pipe->check_device_error();
    });
}

int skb_pipeline_profile(skb_pipeline* p, const void* real_in, void* real_out, skb_stage_time* stages,
                         uint64_t capacity, uint64_t* count) {
    return guard([&] {
        require(p && real_in && real_out && count, "handle, buffers and count must be non-null");
        const auto st = p->pipe->profile(real_in, real_out, p->stream);
        *count = st.size();
        for (size_t i = 0; i < st.size() && i < capacity; ++i) {
            std::memset(&stages[i], 0, sizeof(skb_stage_time));
            std::strncpy(stages[i].name, st[i].name.c_str(), sizeof(stages[i].name) - 1);
            stages[i].ms = st[i].ms;
            stages[i].launches = st[i].launches;
            stages[i].algorithmic_bytes = st[i].bytes;
        }
    });
}

void* skb_pipeline_stream(skb_pipeline* p) { return p ? p->stream : nullptr; }

// ------------------------------------------ constant-stratification type-I

namespace {

unsigned type1_mask(int kind, uint64_t channels) {
    if (kind == SKB_TYPE1_DCT) return 0u;
    if (kind == SKB_TYPE1_DST) return channels >= 32 ? 0xFFFFFFFFu : ((1u << channels) - 1u);
    throw Error(SKB_ERR_INVALID_ARGUMENT, "kind must be SKB_TYPE1_DCT or SKB_TYPE1_DST");
}

void type1_check(const skb_cs_vertical* p, uint64_t storage, uint64_t first, uint64_t channels) {
    require(p != nullptr, "handle must be non-null");
    require(storage >= 1 && storage <= 32, "storage channels must be in [1, 32]");
    require(channels >= 1 && first + channels <= storage,
            "Invalid constant-stratification R2R plan shape: channels outside the storage channels.");
}

void type1_run(skb_cs_vertical* p, unsigned mask, uint64_t storage, uint64_t first, uint64_t channels,
               bool normalize, void* data, cudaStream_t s) {
    check_cuda(launch_type1(p->p == Precision::f64, data, static_cast<long long>(p->rows), static_cast<int>(p->nz),
                            static_cast<int>(storage), static_cast<int>(first), static_cast<int>(channels), mask,
                            normalize, p->tw.get(), s),
               "type-I vertical transform kernel");
}

}  // namespace

int skb_cs_vertical_create(uint64_t rows, uint64_t nz, int precision, skb_cs_vertical** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        require(rows > 0, "constant-stratification rows must be positive");
        require(nz >= 3 && nz <= 16385, "constant-stratification Nz must be in [3, 16385]");
        require(rows * 32 * nz < (uint64_t(1) << 62), "constant-stratification arrays too large");
        auto p = std::make_unique<skb_cs_vertical>();
        p->rows = rows;
        p->nz = nz;
        p->p = to_precision(precision);
        p->host.p = p->p;
        p->stream = make_stream();
        const auto t0 = std::chrono::steady_clock::now();
        const auto tw = twiddle_table(2 * (nz - 1));
        if (p->p == Precision::f64) {
            p->tw = upload_vector(tw);
        } else {
            p->tw = upload_vector(std::vector<float>(tw.begin(), tw.end()));
        }
        p->planning = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *out = p.release();
    });
}

int skb_cs_vertical_destroy(skb_cs_vertical* p) {
    return guard([&] { delete p; });
}

void* skb_cs_vertical_stream(skb_cs_vertical* p) { return p ? p->stream : nullptr; }

int skb_cs_vertical_info(const skb_cs_vertical* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->planning_seconds = p->planning;
        info->allocation_seconds = p->allocation;
        info->persistent_bytes = p->tw.bytes();
        info->scratch_bytes = p->arena.bytes() + p->arena1.bytes();
        info->launches_per_execution = 1;
        info->precision = p->p == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        fill_identity(info, type1_uses_fft(static_cast<int>(p->nz))
                                ? "skb-cuda type-I vertical: warp FFT of the 2(Nz-1)-point symmetric extension"
                                : "skb-cuda type-I vertical: direct sums");
    });
}

int skb_cs_vertical_transform_device(skb_cs_vertical* p, int kind, uint64_t storage, uint64_t first,
                                     uint64_t channels, int normalize, void* data, void* stream) {
    return guard([&] {
        type1_check(p, storage, first, channels);
        require(data != nullptr, "data must be non-null");
        type1_run(p, type1_mask(kind, channels), storage, first, channels, normalize != 0, data,
                  stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

int skb_cs_vertical_normalize_device(skb_cs_vertical* p, int kind, uint64_t storage, uint64_t first,
                                     uint64_t channels, void* data, void* stream) {
    return guard([&] {
        type1_check(p, storage, first, channels);
        require(data != nullptr, "data must be non-null");
        check_cuda(launch_type1_normalize(p->p == Precision::f64, data, static_cast<long long>(p->rows),
                                          static_cast<int>(p->nz), static_cast<int>(storage),
                                          static_cast<int>(first), static_cast<int>(channels),
                                          type1_mask(kind, channels),
                                          stream ? static_cast<cudaStream_t>(stream) : p->stream),
                   "type-I normalisation kernel");
    });
}

int skb_cs_vertical_transform(skb_cs_vertical* p, int kind, uint64_t storage, uint64_t first, uint64_t channels,
                              int normalize, double* data) {
    return guard([&] {
        type1_check(p, storage, first, channels);
        require(data != nullptr, "data must be non-null");
        const unsigned mask = type1_mask(kind, channels);
        const size_t values = 2 * p->rows * storage * p->nz;
        if (p->arena.bytes() < values * element_bytes(p->p)) p->arena.allocate(values * element_bytes(p->p));
        p->host.upload(p->arena.get(), data, values, p->stream);
        type1_run(p, mask, storage, first, channels, normalize != 0, p->arena.get(), p->stream);
        p->host.download(data, p->arena.get(), values, p->stream);
        sync(p->stream);
    });
}

namespace {
// executeCompleteVerticalGraph (src/constant_stratification.cpp:359-379).
// The reference's per-plan calls on disjoint channels of one arena (DCT-I on
// channels 0-1 then DST-I on channel 2, and the converse) are one launch
// each here, with the kind chosen per channel.
void type1_schedule(skb_cs_vertical* p, void* arena3, void* arena1, cudaStream_t s) {
    for (int g = 0; g < 3; ++g) type1_run(p, 0x4u, 3, 0, 3, false, arena3, s);  // velocity + cosine derivatives
    for (int g = 0; g < 2; ++g) type1_run(p, 0x3u, 3, 0, 3, false, arena3, s);  // sine-family derivatives
    for (int g = 0; g < 2; ++g) type1_run(p, 0x0u, 1, 0, 1, true, arena1, s);   // cosine flux targets
    for (int g = 0; g < 2; ++g) type1_run(p, 0x1u, 1, 0, 1, true, arena1, s);   // sine flux targets
}
}  // namespace

int skb_cs_vertical_schedule_device(skb_cs_vertical* p, void* arena3, void* arena1, void* stream) {
    return guard([&] {
        require(p != nullptr && arena3 != nullptr && arena1 != nullptr, "handle and arenas must be non-null");
        type1_schedule(p, arena3, arena1, stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

int skb_cs_vertical_schedule(skb_cs_vertical* p, double* arena3, double* arena1) {
    return guard([&] {
        require(p != nullptr && arena3 != nullptr && arena1 != nullptr, "handle and arenas must be non-null");
        const size_t v3 = 2 * p->rows * 3 * p->nz, v1 = 2 * p->rows * p->nz;
        const size_t es = element_bytes(p->p);
        if (p->arena.bytes() < v3 * es) p->arena.allocate(v3 * es);
        if (p->arena1.bytes() < v1 * es) p->arena1.allocate(v1 * es);
        p->host.upload(p->arena.get(), arena3, v3, p->stream);
        p->host.upload(p->arena1.get(), arena1, v1, p->stream);
        type1_schedule(p, p->arena.get(), p->arena1.get(), p->stream);
        p->host.download(arena3, p->arena.get(), v3, p->stream);
        p->host.download(arena1, p->arena1.get(), v1, p->stream);
        sync(p->stream);
    });
}

int skb_vertical_info(const skb_vertical_provider* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        info->allocation_seconds = p->allocation;
        info->planning_seconds = p->preparation;
        info->persistent_bytes = (p->forward ? p->forward->persistentBytes() : 0) +
                                 (p->inverse ? p->inverse->persistentBytes() : 0) + p->physIn.bytes() +
                                 p->physInIm.bytes() + p->modalOut.bytes() + p->modalOutIm.bytes() +
                                 p->modalIn.bytes() + p->modalInIm.bytes() + p->physOut.bytes() + p->physOutIm.bytes();
        info->launches_per_execution = 1;
        info->precision = p->p == Precision::f64 ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        info->column_transforms_per_direction = p->columns;
        fill_identity(info, "skb-cuda hand-written sm_100a K2-grouped GEMM (one launch for all groups)");
    });
}

void* skb_vertical_stream(skb_vertical_provider* p) { return p ? p->stream : nullptr; }

namespace {
const VerticalPlan& need(const std::unique_ptr<VerticalPlan>& plan, const char* what) {
    if (!plan) throw Error(SKB_ERR_LOGIC, what);
    return *plan;
}
}  // namespace

int skb_vertical_forward_device(skb_vertical_provider* p, const void* in_re, const void* in_im, void* out_re,
                                void* out_im, void* stream) {
    return guard([&] {
        require(p && in_re && out_re, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.")
            .execute({const_cast<void*>(in_re), const_cast<void*>(in_im)}, {out_re, out_im}, s);
    });
}

int skb_vertical_inverse_device(skb_vertical_provider* p, const void* in_re, const void* in_im, void* out_re,
                                void* out_im, void* stream) {
    return guard([&] {
        require(p && in_re && out_re, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.")
            .execute({const_cast<void*>(in_re), const_cast<void*>(in_im)}, {out_re, out_im}, s);
    });
}

namespace {
void require_layout(const skb_vertical_provider* p, int layout) {
    if (p->layout != layout)
        throw Error(SKB_ERR_LOGIC, layout == SKB_LAYOUT_SPLIT
                                       ? "Split GEMM component requested from the complex GEMM provider."
                                       : "Interleaved GEMM component requested from the split GEMM provider.");
}
}  // namespace

int skb_vertical_load_physical_input(skb_vertical_provider* p, const skb_complex* input) {
    return guard([&] {
        require(p && input, "handle and input must be non-null");
        require_layout(p, SKB_LAYOUT_INTERLEAVED);
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.");
        p->host.upload(p->physIn.get(), reinterpret_cast<const double*>(input), 2 * p->columns * p->w.nz, p->stream);
        sync(p->stream);
    });
}

int skb_vertical_load_modal_input(skb_vertical_provider* p, const skb_complex* input) {
    return guard([&] {
        require(p && input, "handle and input must be non-null");
        require_layout(p, SKB_LAYOUT_INTERLEAVED);
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.");
        p->host.upload(p->modalIn.get(), reinterpret_cast<const double*>(input), 2 * p->columns * p->w.nj(),
                       p->stream);
        sync(p->stream);
    });
}

int skb_vertical_load_physical_input_split(skb_vertical_provider* p, const double* re, const double* im) {
    return guard([&] {
        require(p && re && im, "handle and inputs must be non-null");
        require_layout(p, SKB_LAYOUT_SPLIT);
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.");
        p->host.upload(p->physIn.get(), re, p->columns * p->w.nz, p->stream);
        p->host.upload(p->physInIm.get(), im, p->columns * p->w.nz, p->stream);
        sync(p->stream);
    });
}

int skb_vertical_load_modal_input_split(skb_vertical_provider* p, const double* re, const double* im) {
    return guard([&] {
        require(p && re && im, "handle and inputs must be non-null");
        require_layout(p, SKB_LAYOUT_SPLIT);
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.");
        p->host.upload(p->modalIn.get(), re, p->columns * p->w.nj(), p->stream);
        p->host.upload(p->modalInIm.get(), im, p->columns * p->w.nj(), p->stream);
        sync(p->stream);
    });
}

int skb_vertical_expire_wait_for_test(skb_vertical_provider* p, int enable) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        require(p->gp == GemmPrecision::tf32x3 || p->gp == GemmPrecision::bf16x3,
                "the expired-wait test applies to the tensor-core GEMM forms");
        for (auto* plan : {p->forward.get(), p->inverse.get()})
            if (plan) plan->set_expire_wait_for_test(enable != 0);
    });
}

int skb_vertical_execute_forward(skb_vertical_provider* p) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.")
            .execute({p->physIn.get(), p->physInIm.get()}, {p->modalOut.get(), p->modalOutIm.get()}, p->stream);
        sync(p->stream);
        p->forward->check_device_error();
    });
}

int skb_vertical_execute_inverse(skb_vertical_provider* p) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.")
            .execute({p->modalIn.get(), p->modalInIm.get()}, {p->physOut.get(), p->physOutIm.get()}, p->stream);
        sync(p->stream);
        p->inverse->check_device_error();
    });
}

int skb_vertical_copy_forward_output(skb_vertical_provider* p, skb_complex* output) {
    return guard([&] {
        require(p && output, "handle and output must be non-null");
        require_layout(p, SKB_LAYOUT_INTERLEAVED);
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.");
        p->host.download(reinterpret_cast<double*>(output), p->modalOut.get(), 2 * p->columns * p->w.nj(), p->stream);
        sync(p->stream);
    });
}

int skb_vertical_copy_inverse_output(skb_vertical_provider* p, skb_complex* output) {
    return guard([&] {
        require(p && output, "handle and output must be non-null");
        require_layout(p, SKB_LAYOUT_INTERLEAVED);
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.");
        p->host.download(reinterpret_cast<double*>(output), p->physOut.get(), 2 * p->columns * p->w.nz, p->stream);
        sync(p->stream);
    });
}

int skb_vertical_copy_forward_output_split(skb_vertical_provider* p, double* re, double* im) {
    return guard([&] {
        require(p && re && im, "handle and outputs must be non-null");
        require_layout(p, SKB_LAYOUT_SPLIT);
        need(p->forward, "Forward GEMM component requested from an inverse-only provider.");
        p->host.download(re, p->modalOut.get(), p->columns * p->w.nj(), p->stream);
        p->host.download(im, p->modalOutIm.get(), p->columns * p->w.nj(), p->stream);
        sync(p->stream);
    });
}

int skb_vertical_copy_inverse_output_split(skb_vertical_provider* p, double* re, double* im) {
    return guard([&] {
        require(p && re && im, "handle and outputs must be non-null");
        require_layout(p, SKB_LAYOUT_SPLIT);
        need(p->inverse, "Inverse GEMM component requested from a forward-only provider.");
        p->host.download(re, p->physOut.get(), p->columns * p->w.nz, p->stream);
        p->host.download(im, p->physOutIm.get(), p->columns * p->w.nz, p->stream);
        sync(p->stream);
    });
}

// --------------------------------------------------------------- pointwise

int skb_pointwise_create(uint64_t volume, double scale, int precision, skb_pointwise_executor** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        require(volume > 0, "Pointwise advection volume must be positive.");
        auto p = std::make_unique<skb_pointwise_executor>();
        p->volume = volume;
        p->scale = scale;
        p->p = to_precision(precision);
        p->host.p = p->p;
        p->stream = make_stream();
        *out = p.release();
    });
}

int skb_pointwise_destroy(skb_pointwise_executor* p) {
    return guard([&] { delete p; });
}

void* skb_pointwise_stream(skb_pointwise_executor* p) { return p ? p->stream : nullptr; }

int skb_pointwise_execute_device(skb_pointwise_executor* p, const void* shared, const void* derivative, void* target,
                                 void* stream) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        require(shared && derivative && target, "Pointwise advection buffers must be non-null.");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        check_cuda(launch_pointwise(p->p == Precision::f64, static_cast<long long>(p->volume), p->scale, shared,
                                    derivative, target, sm_count(), s),
                   "pointwise advection kernel");
    });
}

int skb_pointwise_execute(skb_pointwise_executor* p, const double* shared, const double* derivative,
                          double* target) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        require(shared && derivative && target, "Pointwise advection buffers must be non-null.");
        const size_t es = element_bytes(p->p);
        if (p->shared.bytes() == 0) {
            p->shared.allocate(3 * es * p->volume);
            p->derivative.allocate(3 * es * p->volume);
            p->target.allocate(es * p->volume);
        }
        p->host.upload(p->shared.get(), shared, 3 * p->volume, p->stream);
        p->host.upload(p->derivative.get(), derivative, 3 * p->volume, p->stream);
        check_cuda(launch_pointwise(p->p == Precision::f64, static_cast<long long>(p->volume), p->scale,
                                    p->shared.get(), p->derivative.get(), p->target.get(), sm_count(), p->stream),
                   "pointwise advection kernel");
        p->host.download(target, p->target.get(), p->volume, p->stream);
        sync(p->stream);
    });
}

// -------------------------------------------------------------------- flux

int skb_flux_create(const skb_flux_options* o, skb_flux** out) {
    return guard([&] {
        require(o != nullptr && out != nullptr, "options and output handle must be non-null");
        require(o->mode >= SKB_FLUX_FP64_PLAIN && o->mode <= SKB_FLUX_SPLIT_BF16X3, "unknown flux mode");
        FluxConfig cfg;
        cfg.n = o->n;
        cfg.nz = o->nz;
        cfg.targets = o->targets;
        cfg.members = o->members;
        cfg.mode = static_cast<FluxMode>(o->mode);
        cfg.family = o->family;
        cfg.familySeed = o->family_seed;
        require(cfg.family == SKB_FAMILY_K2_ROTATION || cfg.family == SKB_FAMILY_STURM_LIOUVILLE,
                "flux family must be K2 rotation or Sturm-Liouville");
        auto p = std::make_unique<skb_flux>();
        p->pipeline = std::make_unique<FluxPipeline>(cfg);
        p->stream = make_stream();
        *out = p.release();
    });
}

int skb_flux_create_families(const skb_flux_options* o, const skb_flux_families* fam, skb_flux** out) {
    return guard([&] {
        require(o != nullptr && fam != nullptr && out != nullptr, "options, families and handle must be non-null");
        require(o->mode >= SKB_FLUX_FP64_PLAIN && o->mode <= SKB_FLUX_SPLIT_BF16X3, "unknown flux mode");
        require(o->targets == 4, "operator families are defined for the 15 -> 4 flux");
        require(fam->groups > 0 && fam->group_modes != nullptr, "families need their operator groups");
        const uint64_t nj = o->nz < 2 ? 0 : 2 * (o->nz - 1) / 3;
        auto F = std::make_shared<FluxFamilies>();
        std::uint64_t first = 0;
        for (uint64_t g = 0; g < fam->groups; ++g) {
            require(fam->group_modes[g] > 0, "operator groups must be nonempty");
            F->groups.push_back({0, first, fam->group_modes[g]});
            first += fam->group_modes[g];
        }
        const size_t matrix = static_cast<size_t>(fam->groups * nj * o->nz);
        for (int f = 0; f < 2; ++f) {
            require(fam->forward[f] != nullptr && fam->inverse[f] != nullptr, "both families need both directions");
            F->forward[f].assign(fam->forward[f], fam->forward[f] + matrix);
            F->inverse[f].assign(fam->inverse[f], fam->inverse[f] + matrix);
        }
        F->inputFamily.assign(fam->input_family, fam->input_family + 15);
        F->targetFamily.assign(fam->target_family, fam->target_family + 4);
        FluxConfig cfg;
        cfg.n = o->n;
        cfg.nz = o->nz;
        cfg.targets = o->targets;
        cfg.members = o->members;
        cfg.mode = static_cast<FluxMode>(o->mode);
        cfg.families = std::move(F);
        auto p = std::make_unique<skb_flux>();
        p->pipeline = std::make_unique<FluxPipeline>(cfg);
        p->stream = make_stream();
        *out = p.release();
    });
}

int skb_flux_destroy(skb_flux* p) {
    return guard([&] { delete p; });
}

int skb_flux_info(const skb_flux* p, skb_provider_info* info) {
    return guard([&] {
        require(p != nullptr && info != nullptr, "handle and info must be non-null");
        std::memset(info, 0, sizeof(*info));
        const auto& f = *p->pipeline;
        info->allocation_seconds = f.allocationSeconds;
        info->planning_seconds = f.planningSeconds;
        info->persistent_bytes = f.persistentBytes;
        info->scratch_bytes = f.scratchBytes;
        info->launches_per_execution = f.launchesPerExecution();
        info->precision = f.f64() ? SKB_PRECISION_FP64 : SKB_PRECISION_FP32;
        fill_identity(info, f.familyId.c_str());
    });
}

void* skb_flux_stream(skb_flux* p) { return p ? p->stream : nullptr; }

int skb_flux_sizes(const skb_flux* p, uint64_t* modes, uint64_t* nj, uint64_t* in, uint64_t* out) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        if (modes) *modes = p->pipeline->modes();
        if (nj) *nj = p->pipeline->nj();
        if (in) *in = p->pipeline->inputElements();
        if (out) *out = p->pipeline->outputElements();
    });
}

int skb_flux_execute_device(skb_flux* p, const void* in, void* out, void* stream) {
    return guard([&] {
        require(p && in && out, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->pipeline->execute(in, out, s);
    });
}

int skb_flux_execute_device_members(skb_flux* p, const void* in, void* out, uint64_t members, void* stream) {
    return guard([&] {
        require(p && in && out, "handle and buffers must be non-null");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
        p->pipeline->execute(in, out, s, members);
    });
}

// Host arrays: the members are pipelined so the link never waits on the
// device.  Member m's input is uploaded on copyIn while member m-1 is computed
// on the handle's stream and member m-2's result is downloaded on copyOut
// (PCIe moves both directions at once); each member runs as a one-member flux
// on its slice of the device buffers, with the FP64 <-> FP32 conversions of
// reduced-precision handles on the compute stream.
int skb_flux_execute(skb_flux* p, const skb_complex* in, skb_complex* out) {
    return guard([&] {
        require(p && in && out, "handle and buffers must be non-null");
        auto& f = *p->pipeline;
        const bool f64 = f.f64();
        const size_t es = f64 ? sizeof(double) : sizeof(float);
        const std::uint64_t members = f.config().members;
        const std::uint64_t inPer = 2 * f.inputElements() / members, outPer = 2 * f.outputElements() / members;
        if (p->in.bytes() == 0) {
            p->in.allocate(es * inPer * members);
            p->out.allocate(es * outPer * members);
        }
        if (p->copyIn == nullptr) {
            p->copyIn = make_stream();
            p->copyOut = make_stream();
            for (std::uint64_t m = 0; m < members; ++m) {
                cudaEvent_t a = nullptr, b = nullptr;
                check_cuda(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "cudaEventCreate");
                p->landed.push_back(a);
                check_cuda(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "cudaEventCreate");
                p->ready.push_back(b);
            }
            if (!f64) {
                p->stageIn.allocate(sizeof(double) * inPer * members);
                p->stageOut.allocate(sizeof(double) * outPer * members);
            }
        }
        const auto* src = reinterpret_cast<const double*>(in);
        auto* dst = reinterpret_cast<double*>(out);
        // The previous call's downloads have finished (it synchronised), so
        // the staging buffers are free; the compute stream orders after them.
        for (std::uint64_t m = 0; m < members; ++m) {
            void* upTarget = f64 ? static_cast<void*>(p->in.get<double>() + m * inPer)
                                 : static_cast<void*>(p->stageIn.get<double>() + m * inPer);
            copy_in(upTarget, src + m * inPer, sizeof(double) * inPer, p->copyIn);
            check_cuda(cudaEventRecord(p->landed[m], p->copyIn), "cudaEventRecord");
        }
        for (std::uint64_t m = 0; m < members; ++m) {
            check_cuda(cudaStreamWaitEvent(p->stream, p->landed[m], 0), "cudaStreamWaitEvent");
            unsigned char* dIn = p->in.get<unsigned char>() + es * m * inPer;
            unsigned char* dOut = p->out.get<unsigned char>() + es * m * outPer;
            if (!f64)
                check_cuda(launch_convert_f64_to_f32(p->stageIn.get<double>() + m * inPer, reinterpret_cast<float*>(dIn),
                                                     static_cast<long long>(inPer), p->stream),
                           "convert kernel");
            f.execute(dIn, dOut, p->stream, 1);
            if (!f64)
                check_cuda(launch_convert_f32_to_f64(reinterpret_cast<const float*>(dOut),
                                                     p->stageOut.get<double>() + m * outPer,
                                                     static_cast<long long>(outPer), p->stream),
                           "convert kernel");
            check_cuda(cudaEventRecord(p->ready[m], p->stream), "cudaEventRecord");
        }
        for (std::uint64_t m = 0; m < members; ++m) {
            check_cuda(cudaStreamWaitEvent(p->copyOut, p->ready[m], 0), "cudaStreamWaitEvent");
            const void* downSource = f64 ? static_cast<const void*>(p->out.get<double>() + m * outPer)
                                         : static_cast<const void*>(p->stageOut.get<double>() + m * outPer);
            copy_out(dst + m * outPer, downSource, sizeof(double) * outPer, p->copyOut);
        }
        sync(p->copyOut);
        sync(p->stream);
        f.check_device_errors();
    });
}

int skb_flux_profile(skb_flux* p, const void* in, void* out, skb_stage_time* stages, uint64_t capacity,
                     uint64_t* count) {
    return guard([&] {
        require(p && in && out && count, "handle, buffers and count must be non-null");
        const auto result = p->pipeline->profile(in, out, p->stream);
        *count = result.size();
        if (stages == nullptr) return;
        require(capacity >= result.size(), "stage capacity too small");
        for (size_t i = 0; i < result.size(); ++i) {
            std::memset(&stages[i], 0, sizeof(stages[i]));
            std::snprintf(stages[i].name, sizeof(stages[i].name), "%s", result[i].name.c_str());
            stages[i].ms = result[i].ms;
            stages[i].launches = result[i].launches;
            stages[i].algorithmic_bytes = result[i].bytes;
            stages[i].flops = result[i].flops;
        }
    });
}

int skb_flux_check_device(skb_flux* p) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        sync(p->stream);
        p->pipeline->check_device_errors();
    });
}

int skb_flux_rows_expire_wait_for_test(skb_flux* p, int enable) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        p->pipeline->set_rows_expire_wait_for_test(enable != 0);
    });
}

int skb_flux_capture_graph(skb_flux* p, const void* in, void* out) {
    return guard([&] {
        require(p && in && out, "handle and buffers must be non-null");
        p->pipeline->capture(in, out, p->stream);
    });
}

int skb_flux_replay_graph(skb_flux* p, void* stream) {
    return guard([&] {
        require(p != nullptr, "handle must be non-null");
        p->pipeline->replay(stream ? static_cast<cudaStream_t>(stream) : p->stream);
    });
}

// --------------------------------------------------------------- autotuner

namespace {
void copy_string(const std::string& text, char* out, uint64_t capacity) {
    if (out == nullptr || capacity == 0) return;
    const size_t n = std::min<size_t>(text.size(), static_cast<size_t>(capacity - 1));
    std::memcpy(out, text.data(), n);
    out[n] = '\0';
}
}  // namespace

int skb_flux_autotune(skb_flux* p, const void* in, void* out, char* summary, uint64_t capacity) {
    return guard([&] {
        require(p && in && out, "handle and buffers must be non-null");
        const auto chosen = p->pipeline->autotune(in, out, p->stream);
        std::string text;
        for (const auto& c : chosen) {
            char ms[32];
            std::snprintf(ms, sizeof ms, "%.4f", c.ms);
            text += c.key + " = " + std::to_string(c.value) + " (" + ms + " ms)\n";
        }
        copy_string(text, summary, capacity);
    });
}

int skb_tune_cache_size(uint64_t* count) {
    return guard([&] {
        require(count != nullptr, "count must be non-null");
        *count = tune_entries().size();
    });
}

int skb_tune_cache_entry(uint64_t index, char* key, uint64_t key_capacity, int* value, double* ms) {
    return guard([&] {
        const auto entries = tune_entries();
        require(index < entries.size(), "tuning cache index out of range");
        copy_string(entries[index].key, key, key_capacity);
        if (value != nullptr) *value = entries[index].value;
        if (ms != nullptr) *ms = entries[index].ms;
    });
}

int skb_tune_cache_store(const char* key, int value, double ms) {
    return guard([&] {
        require(key != nullptr && *key != '\0', "key must be non-empty");
        const std::string k(key);
        require(k.find('\n') == std::string::npos, "key must be one line");
        tune_store(k, value, ms);
    });
}

int skb_tune_cache_lookup(const char* key, int* value, int* found) {
    return guard([&] {
        require(key != nullptr && found != nullptr, "key and found must be non-null");
        int v = 0;
        *found = tune_lookup(key, v) ? 1 : 0;
        if (value != nullptr && *found) *value = v;
    });
}

int skb_tune_cache_clear(void) {
    return guard([&] { tune_clear(); });
}

int skb_tune_cache_load(const char* path, uint64_t* count) {
    return guard([&] {
        require(path != nullptr, "path must be non-null");
        const int n = tune_load(path);
        if (count != nullptr) *count = static_cast<uint64_t>(n);
    });
}

int skb_tune_cache_save(const char* path, uint64_t* count) {
    return guard([&] {
        require(path != nullptr, "path must be non-null");
        const int n = tune_save(path);
        if (count != nullptr) *count = static_cast<uint64_t>(n);
    });
}

// ----------------------------------------------------------------- server

int skb_server_create(const skb_server_class* classes, uint64_t count, uint64_t budget, int maxSlots,
                      skb_server** out) {
    return guard([&] {
        require(classes != nullptr && count > 0 && out != nullptr, "classes and output handle must be non-null");
        std::vector<ServerClass> cs;
        for (uint64_t i = 0; i < count; ++i) {
            require(classes[i].mode >= SKB_FLUX_FP64_PLAIN && classes[i].mode <= SKB_FLUX_SPLIT_BF16X3,
                    "unknown flux mode");
            cs.push_back({classes[i].n, classes[i].nz, classes[i].targets, classes[i].max_batch,
                          static_cast<FluxMode>(classes[i].mode)});
        }
        *out = reinterpret_cast<skb_server*>(new Server(cs, budget, maxSlots));
    });
}

int skb_server_destroy(skb_server* s) {
    return guard([&] { delete reinterpret_cast<Server*>(s); });
}

int skb_server_sizes(skb_server* s, int cls, uint64_t* in, uint64_t* out) {
    return guard([&] {
        require(s != nullptr, "handle must be non-null");
        auto* srv = reinterpret_cast<Server*>(s);
        if (in) *in = srv->inputElements(cls);
        if (out) *out = srv->outputElements(cls);
    });
}

int skb_server_submit(skb_server* s, int cls, const skb_complex* in, skb_complex* out, uint64_t* ticket) {
    return guard([&] {
        require(s != nullptr && ticket != nullptr, "handle and ticket must be non-null");
        *ticket = reinterpret_cast<Server*>(s)->submit(cls, reinterpret_cast<const double*>(in),
                                                       reinterpret_cast<double*>(out));
    });
}

int skb_server_load_state(skb_server* s, int cls, const skb_complex* in, int64_t* state) {
    return guard([&] {
        require(s != nullptr && state != nullptr, "handle and state must be non-null");
        *state = reinterpret_cast<Server*>(s)->loadState(cls, reinterpret_cast<const double*>(in));
    });
}

int skb_server_release_state(skb_server* s, int64_t state) {
    return guard([&] {
        require(s != nullptr, "handle must be non-null");
        reinterpret_cast<Server*>(s)->releaseState(state);
    });
}

int skb_server_submit_state(skb_server* s, int64_t state, skb_complex* out, uint64_t* ticket) {
    return guard([&] {
        require(s != nullptr && ticket != nullptr, "handle and ticket must be non-null");
        *ticket = reinterpret_cast<Server*>(s)->submitState(state, reinterpret_cast<double*>(out));
    });
}

int skb_server_wait(skb_server* s, uint64_t ticket, double timeout, int* done, double* latency) {
    return guard([&] {
        require(s != nullptr && done != nullptr, "handle and done flag must be non-null");
        *done = reinterpret_cast<Server*>(s)->wait(ticket, timeout, latency) ? 1 : 0;
    });
}

int skb_server_get_stats(skb_server* s, skb_server_stats* st) {
    return guard([&] {
        require(s != nullptr && st != nullptr, "handle and stats must be non-null");
        const auto x = reinterpret_cast<Server*>(s)->stats();
        *st = {x.submitted, x.completed, x.batches, x.slots, x.residentStates, x.slotBytes, x.stateBytes,
               x.budgetBytes};
    });
}

int skb_server_hold(skb_server* s, int held) {
    return guard([&] {
        require(s != nullptr, "handle must be non-null");
        reinterpret_cast<Server*>(s)->hold(held != 0);
    });
}

// ------------------------------------------------------------------ timing

int skb_timer_create(skb_timer** out) {
    return guard([&] {
        require(out != nullptr, "output handle must be non-null");
        auto t = std::make_unique<skb_timer>();
        check_cuda(cudaEventCreate(&t->start), "cudaEventCreate");
        check_cuda(cudaEventCreate(&t->stop), "cudaEventCreate");
        *out = t.release();
    });
}

int skb_timer_destroy(skb_timer* t) {
    return guard([&] { delete t; });
}

int skb_timer_start(skb_timer* t, void* stream) {
    return guard([&] { check_cuda(cudaEventRecord(t->start, static_cast<cudaStream_t>(stream)), "cudaEventRecord"); });
}

int skb_timer_stop(skb_timer* t, void* stream) {
    return guard([&] { check_cuda(cudaEventRecord(t->stop, static_cast<cudaStream_t>(stream)), "cudaEventRecord"); });
}

int skb_timer_elapsed_ms(skb_timer* t, double* ms) {
    return guard([&] {
        require(t && ms, "timer and output must be non-null");
        check_cuda(cudaEventSynchronize(t->stop), "cudaEventSynchronize");
        float f = 0.0f;
        check_cuda(cudaEventElapsedTime(&f, t->start, t->stop), "cudaEventElapsedTime");
        *ms = f;
    });
}

// ----------------------------------------------------------------- buffers

int skb_device_alloc(uint64_t bytes, void** ptr) {
    return guard([&] {
        require(ptr != nullptr, "output pointer must be non-null");
        check_cuda(cudaMalloc(ptr, bytes), "cudaMalloc");
    });
}

int skb_device_free(void* ptr) {
    return guard([&] { check_cuda(cudaFree(ptr), "cudaFree"); });
}

int skb_host_alloc_pinned(uint64_t bytes, void** ptr) {
    return guard([&] {
        require(ptr != nullptr, "output pointer must be non-null");
        check_cuda(cudaMallocHost(ptr, bytes), "cudaMallocHost");
    });
}

int skb_host_free_pinned(void* ptr) {
    return guard([&] { check_cuda(cudaFreeHost(ptr), "cudaFreeHost"); });
}

int skb_copy_to_device(void* dst, const void* src, uint64_t bytes, void* stream) {
    return guard([&] {
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)),
                   "cudaMemcpyAsync H2D");
    });
}

int skb_copy_to_host(void* dst, const void* src, uint64_t bytes, void* stream) {
    return guard([&] {
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)),
                   "cudaMemcpyAsync D2H");
    });
}

int skb_stream_synchronize(void* stream) {
    return guard([&] { check_cuda(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "cudaStreamSynchronize"); });
}

}  // extern "C"
