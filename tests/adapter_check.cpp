// The reference-side C++ adapter over the C ABI (include/skb_cuda.h): the
// binding a skbench maintainer adds so that `--providers cuda` constructs these
// classes where the `fftw` branch constructs FFTWProvider
// (src/benchmark.cpp:5375-5447).  It is compiled by tests/test_adapter_cpu.py
// with -fsyntax-only against the reference's own headers
// (include/skbench/skbench.hpp, src/pointwise_advection.hpp), and the
// static_asserts at the end check that every adapter method has exactly the
// parameter and return types of the reference method it replaces, so a drift
// of either side (a changed RetainedMode vector parameter, a FieldView type, a
// const) fails the build of this file.
//
// Errors rethrow the reference's exception types, so main.cpp's exit codes
// (main.cpp:242-245) stay the same.

#include <skb_cuda.h>

#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "pointwise_advection.hpp"
#include "skbench/skbench.hpp"

namespace skbench {

inline void skbCheck(int rc) {
    if (rc == SKB_OK) return;
    const std::string what = skb_last_error();
    if (rc == SKB_ERR_INVALID_ARGUMENT) throw std::invalid_argument(what);
    if (rc == SKB_ERR_LOGIC) throw std::logic_error(what);
    if (rc == SKB_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
    throw std::runtime_error(what);
}

inline skb_workload toSkb(const Workload& w) {
    return {w.nx, w.ny, w.nz, w.fields, w.lx, w.ly, w.antialias ? 1 : 0};
}

inline skb_complex* asSkb(Complex* p) { return reinterpret_cast<skb_complex*>(p); }
inline const skb_complex* asSkb(const Complex* p) { return reinterpret_cast<const skb_complex*>(p); }
static_assert(sizeof(Complex) == sizeof(skb_complex), "Complex and skb_complex must share their layout");

inline std::string infoIdentity(const skb_provider_info& i) { return i.library_identity; }

// FFTWProvider (skbench.hpp:364-421).  The retained-mode vector is accepted for
// the reference's signature; the library uses its own identical mode table
// (retainedHorizontalModes order), built at handle creation.
class CudaFFTProvider {
public:
    explicit CudaFFTProvider(const Workload& w) {
        const auto s = toSkb(w);
        skbCheck(skb_fft_create(&s, SKB_PRECISION_FP64, &h_));
    }
    ~CudaFFTProvider() { skb_fft_destroy(h_); }
    CudaFFTProvider(const CudaFFTProvider&) = delete;
    CudaFFTProvider& operator=(const CudaFFTProvider&) = delete;

    void forward(const double* input, Complex* wvmSpectrum) { skbCheck(skb_fft_forward(h_, input, asSkb(wvmSpectrum))); }
    void inverse(Complex* wvmSpectrum, double* output) { skbCheck(skb_fft_inverse(h_, asSkb(wvmSpectrum), output)); }
    void gatherRetainedOuter(const std::vector<RetainedMode>&, const Complex* wvmSpectrum, Complex* retainedSpectrum) {
        skbCheck(skb_fft_gather_retained(h_, asSkb(wvmSpectrum), asSkb(retainedSpectrum)));
    }
    void embedRetainedOuter(const std::vector<RetainedMode>&, const Complex* retainedSpectrum, Complex* wvmSpectrum) {
        skbCheck(skb_fft_embed_retained(h_, asSkb(retainedSpectrum), asSkb(wvmSpectrum)));
    }
    void gatherRetainedToSplitOuter(const std::vector<RetainedMode>&, const Complex* spectrum, double* retainedReal,
                                    double* retainedImag, double scale = 1.0) {
        skbCheck(skb_fft_gather_retained_to_split(h_, asSkb(spectrum), retainedReal, retainedImag, scale));
    }
    void embedRetainedFromSplitOuter(const std::vector<RetainedMode>&, const double* retainedReal,
                                     const double* retainedImag, Complex* spectrum) {
        skbCheck(skb_fft_embed_retained_from_split(h_, retainedReal, retainedImag, asSkb(spectrum)));
    }
    void forwardSplit(const double* input, double* wvmSpectrumReal, double* wvmSpectrumImag) {
        skbCheck(skb_fft_forward_split(h_, input, wvmSpectrumReal, wvmSpectrumImag));
    }
    void inverseSplit(double* wvmSpectrumReal, double* wvmSpectrumImag, double* output) {
        skbCheck(skb_fft_inverse_split(h_, wvmSpectrumReal, wvmSpectrumImag, output));
    }
    double allocationSeconds() const noexcept { return infoOrZero().allocation_seconds; }
    double planningSeconds() const noexcept { return infoOrZero().planning_seconds; }
    double otherSetupSeconds() const noexcept { return infoOrZero().other_setup_seconds; }
    std::size_t planningBytes() const noexcept { return infoOrZero().planning_bytes; }
    std::string libraryIdentity() const { return infoIdentity(infoOrZero()); }

private:
    skb_provider_info infoOrZero() const noexcept {
        skb_provider_info i{};
        if (skb_fft_info(h_, &i) != SKB_OK) i = skb_provider_info{};
        return i;
    }
    skb_fft_provider* h_ = nullptr;
};

// FFTWStreamingPrunedSplitProvider (skbench.hpp:534-624): split retained
// spectra and {real, imaginary, modeStride} field views.
class CudaStreamingPrunedSplitProvider {
public:
    using ConstFieldView = FFTWStreamingPrunedSplitProvider::ConstFieldView;
    using FieldView = FFTWStreamingPrunedSplitProvider::FieldView;

    explicit CudaStreamingPrunedSplitProvider(const Workload& w) {
        const auto s = toSkb(w);
        skbCheck(skb_pruned_create(&s, SKB_PRECISION_FP64, &h_));
    }
    ~CudaStreamingPrunedSplitProvider() { skb_pruned_destroy(h_); }
    CudaStreamingPrunedSplitProvider(const CudaStreamingPrunedSplitProvider&) = delete;
    CudaStreamingPrunedSplitProvider& operator=(const CudaStreamingPrunedSplitProvider&) = delete;

    void forwardSplit(const double* input, double* retainedReal, double* retainedImag, double scale = 1.0) {
        skbCheck(skb_pruned_forward_split(h_, input, retainedReal, retainedImag, scale));
    }
    void inverseSplit(const double* retainedReal, const double* retainedImag, double* output) {
        skbCheck(skb_pruned_inverse_split(h_, retainedReal, retainedImag, output));
    }
    void forwardSplitFields(const double* input, const FieldView* fields, std::size_t fieldCount, double scale = 1.0) {
        std::vector<skb_field_view> v(fieldCount);
        for (std::size_t i = 0; i < fieldCount; ++i) v[i] = {fields[i].real, fields[i].imaginary, fields[i].modeStride};
        skbCheck(skb_pruned_forward_split_fields(h_, input, v.data(), fieldCount, scale));
    }
    void inverseSplitFields(const ConstFieldView* fields, std::size_t fieldCount, double* output) {
        std::vector<skb_field_view> v(fieldCount);
        for (std::size_t i = 0; i < fieldCount; ++i)
            v[i] = {const_cast<double*>(fields[i].real), const_cast<double*>(fields[i].imaginary), fields[i].modeStride};
        skbCheck(skb_pruned_inverse_split_fields(h_, v.data(), fieldCount, output));
    }

private:
    skb_pruned_provider* h_ = nullptr;
};

// VerticalGemmProvider (skbench.hpp:152-218) over a GroupedVerticalOperators
// family, interleaved layout.
class CudaVerticalGemmProvider {
public:
    CudaVerticalGemmProvider(const Workload& w, const GroupedVerticalOperators& ops, VerticalGemmBufferPolicy policy) {
        const auto s = toSkb(w);
        std::vector<skb_mode_group> groups;
        for (const auto& g : ops.groups) groups.push_back({g.squaredModeKey, g.firstMode, g.modeCount});
        const int buffers = policy == VerticalGemmBufferPolicy::forwardOnly   ? SKB_BUFFERS_FORWARD_ONLY
                            : policy == VerticalGemmBufferPolicy::inverseOnly ? SKB_BUFFERS_INVERSE_ONLY
                                                                              : SKB_BUFFERS_BIDIRECTIONAL;
        skbCheck(skb_vertical_create(&s, groups.data(), groups.size(), ops.forward.data(), ops.inverse.data(),
                                     SKB_LAYOUT_INTERLEAVED, buffers, SKB_GEMM_FP64, &h_));
    }
    ~CudaVerticalGemmProvider() { skb_vertical_destroy(h_); }
    CudaVerticalGemmProvider(const CudaVerticalGemmProvider&) = delete;
    CudaVerticalGemmProvider& operator=(const CudaVerticalGemmProvider&) = delete;

    void loadPhysicalInput(const Complex* input) { skbCheck(skb_vertical_load_physical_input(h_, asSkb(input))); }
    void loadModalInput(const Complex* input) { skbCheck(skb_vertical_load_modal_input(h_, asSkb(input))); }
    void executeForward() { skbCheck(skb_vertical_execute_forward(h_)); }
    void executeInverse() { skbCheck(skb_vertical_execute_inverse(h_)); }
    void copyForwardOutput(Complex* output) const { skbCheck(skb_vertical_copy_forward_output(h_, asSkb(output))); }
    void copyInverseOutput(Complex* output) const { skbCheck(skb_vertical_copy_inverse_output(h_, asSkb(output))); }

private:
    skb_vertical_provider* h_ = nullptr;
};

// PointwiseAdvectionExecutor (pointwise_advection.hpp:18-43).
class CudaPointwiseAdvectionExecutor {
public:
    CudaPointwiseAdvectionExecutor(std::size_t volumeElements, double scale) {
        skbCheck(skb_pointwise_create(volumeElements, scale, SKB_PRECISION_FP64, &h_));
    }
    ~CudaPointwiseAdvectionExecutor() { skb_pointwise_destroy(h_); }
    CudaPointwiseAdvectionExecutor(const CudaPointwiseAdvectionExecutor&) = delete;
    CudaPointwiseAdvectionExecutor& operator=(const CudaPointwiseAdvectionExecutor&) = delete;

    void execute(const double* shared, const double* derivative, double* target) {
        skbCheck(skb_pointwise_execute(h_, shared, derivative, target));
    }

private:
    skb_pointwise_executor* h_ = nullptr;
};

// Constant-stratification R2RPlan set (constant_stratification.cpp:95-186): one
// handle per (rows, Nz); a plan's execute() transforms a channel range of one
// arena in place.
class CudaType1Plans {
public:
    CudaType1Plans(std::size_t rows, std::size_t nz) {
        skbCheck(skb_cs_vertical_create(rows, nz, SKB_PRECISION_FP64, &h_));
    }
    ~CudaType1Plans() { skb_cs_vertical_destroy(h_); }
    CudaType1Plans(const CudaType1Plans&) = delete;
    CudaType1Plans& operator=(const CudaType1Plans&) = delete;

    void execute(Complex* storage, std::size_t storageChannels, std::size_t first, std::size_t channels, bool sine) {
        skbCheck(skb_cs_vertical_transform(h_, sine ? SKB_TYPE1_DST : SKB_TYPE1_DCT, storageChannels, first, channels,
                                           0, reinterpret_cast<double*>(storage)));
    }
    void completeGraph(Complex* arena3, Complex* arena1) {
        skbCheck(skb_cs_vertical_schedule(h_, reinterpret_cast<double*>(arena3), reinterpret_cast<double*>(arena1)));
    }

private:
    skb_cs_vertical* h_ = nullptr;
};

// ------------------------------------------------- signature checks

// The plain function type of a member function pointer, const and noexcept
// recorded separately so they are compared too.
template <typename T>
struct Method;
template <typename C, typename R, typename... A>
struct Method<R (C::*)(A...)> {
    using type = R(A...);
    static constexpr bool isConst = false;
};
template <typename C, typename R, typename... A>
struct Method<R (C::*)(A...) const> {
    using type = R(A...);
    static constexpr bool isConst = true;
};
template <typename C, typename R, typename... A>
struct Method<R (C::*)(A...) noexcept> {
    using type = R(A...);
    static constexpr bool isConst = false;
};
template <typename C, typename R, typename... A>
struct Method<R (C::*)(A...) const noexcept> {
    using type = R(A...);
    static constexpr bool isConst = true;
};

template <typename Ours, typename Theirs>
constexpr bool sameMethod() {
    return std::is_same_v<typename Method<Ours>::type, typename Method<Theirs>::type> &&
           Method<Ours>::isConst == Method<Theirs>::isConst;
}

#define SKB_SAME_METHOD(ours, theirs, name)                                                   \
    static_assert(sameMethod<decltype(&ours::name), decltype(&theirs::name)>(),              \
                  #ours "::" #name " differs from the reference's " #theirs "::" #name)

SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, forward);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, inverse);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, gatherRetainedOuter);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, embedRetainedOuter);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, gatherRetainedToSplitOuter);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, embedRetainedFromSplitOuter);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, forwardSplit);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, inverseSplit);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, allocationSeconds);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, planningSeconds);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, otherSetupSeconds);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, planningBytes);
SKB_SAME_METHOD(CudaFFTProvider, FFTWProvider, libraryIdentity);
SKB_SAME_METHOD(CudaStreamingPrunedSplitProvider, FFTWStreamingPrunedSplitProvider, forwardSplit);
SKB_SAME_METHOD(CudaStreamingPrunedSplitProvider, FFTWStreamingPrunedSplitProvider, inverseSplit);
SKB_SAME_METHOD(CudaStreamingPrunedSplitProvider, FFTWStreamingPrunedSplitProvider, forwardSplitFields);
SKB_SAME_METHOD(CudaStreamingPrunedSplitProvider, FFTWStreamingPrunedSplitProvider, inverseSplitFields);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, loadPhysicalInput);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, loadModalInput);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, executeForward);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, executeInverse);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, copyForwardOutput);
SKB_SAME_METHOD(CudaVerticalGemmProvider, VerticalGemmProvider, copyInverseOutput);
SKB_SAME_METHOD(CudaPointwiseAdvectionExecutor, PointwiseAdvectionExecutor, execute);

// The C ABI's plain structs against the reference types they stand for.
static_assert(sizeof(skb_complex) == 2 * sizeof(double), "skb_complex is two doubles");
static_assert(std::is_same_v<decltype(FFTWStreamingPrunedSplitProvider::FieldView::modeStride), std::size_t> &&
                  sizeof(std::size_t) == sizeof(uint64_t),
              "a field view's mode stride fits skb_field_view::mode_stride");
static_assert(std::is_same_v<decltype(RetainedMode::k), std::int64_t> && std::is_same_v<decltype(Workload::nx), std::size_t>,
              "mode keys and workload sizes keep the types skb_retained_mode and skb_workload mirror");

}  // namespace skbench
