/*
 * skb_cuda.h — C ABI of the B200 `cuda` provider for the skbench spectral path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * an int status (SKB_OK = 0).  On failure skb_last_error() returns the message
 * of the calling thread's most recent error.  The status classes mirror the
 * exception types the reference's providers throw, so a C++ wrapper can
 * rethrow the same type and keep the CLI's exit codes
 * (include/skbench/skbench.hpp, src/main.cpp:242-245):
 *   SKB_ERR_INVALID_ARGUMENT  std::invalid_argument (bad shape, null pointer)
 *   SKB_ERR_RUNTIME           std::runtime_error    (CUDA failure, unsupported)
 *   SKB_ERR_LOGIC             std::logic_error      (wrong layout / direction)
 *   SKB_ERR_OUT_OF_MEMORY     std::bad_alloc
 *
 * Pointer families.  Functions without a suffix take HOST arrays and block
 * until the result is back in host memory (the reference's providers are
 * host-array APIs).  `_device` functions take DEVICE pointers, enqueue on the
 * given CUDA stream (NULL = the handle's own stream) and return without
 * synchronising.  Device arrays use the handle's precision: double for
 * SKB_PRECISION_FP64 handles, float for SKB_PRECISION_FP32; complex values are
 * interleaved (re, im) pairs unless a split view is given.
 *
 * Layouts are the reference's (src/model.cpp:219-244):
 *   real      [field][z][y][x]            x fastest
 *   wvm       [ky][kx][field][z]          WVM frequency-major half spectrum,
 *                                         index z + Nz*field + planes*(kx + (Nx/2+1)*ky)
 *   retained  [mode][field][z]            index z + Nz*field + planes*mode
 *   modal     [mode][field][j]            index j + Nj*field + Nj*fields*mode
 * Transforms are unnormalised in both directions like FFTW's.
 *
 * Handles own their device scratch; steady-state calls allocate nothing.
 * A handle is single-owner: calls on one handle must not overlap.
 */
#ifndef SKB_CUDA_H
#define SKB_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SKB_API __attribute__((visibility("default")))
#else
#define SKB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SKB_OK 0
#define SKB_ERR_INVALID_ARGUMENT (-1)
#define SKB_ERR_RUNTIME (-2)
#define SKB_ERR_LOGIC (-3)
#define SKB_ERR_OUT_OF_MEMORY (-4)

#define SKB_PRECISION_FP64 0
#define SKB_PRECISION_FP32 1

#define SKB_GEMM_FP64 0
#define SKB_GEMM_FP32 1
#define SKB_GEMM_TF32X3 2
#define SKB_GEMM_BF16X3 3

#define SKB_LAYOUT_INTERLEAVED 0
#define SKB_LAYOUT_SPLIT 1

/* VerticalGemmBufferPolicy (skbench.hpp:132-136). */
#define SKB_BUFFERS_BIDIRECTIONAL 0
#define SKB_BUFFERS_FORWARD_ONLY 1
#define SKB_BUFFERS_INVERSE_ONLY 2

/* Vertical operator families (src/model.cpp:489-565, plus the build's seeded
 * Sturm-Liouville family). */
#define SKB_FAMILY_COMMON_DCT2 0
#define SKB_FAMILY_K2_ROTATION 1
#define SKB_FAMILY_STURM_LIOUVILLE 2

/* Workload (skbench.hpp:23-39). */
typedef struct skb_workload {
    uint64_t nx, ny, nz, fields;
    double lx, ly;
    int32_t antialias;
} skb_workload;

/* Complex (skbench.hpp:15-18). */
typedef struct skb_complex {
    double real, imag;
} skb_complex;

/* RetainedMode (skbench.hpp:41-48). */
typedef struct skb_retained_mode {
    int64_t k, l;
    uint64_t stored_kx, stored_ky;
    int32_t conjugates_stored_value;
    double radial_mode;
} skb_retained_mode;

/* VerticalModeGroup (skbench.hpp:50-56). */
typedef struct skb_mode_group {
    uint64_t squared_mode_key, first_mode, mode_count;
} skb_mode_group;

/* FieldView / ConstFieldView of FFTWStreamingPrunedSplitProvider
 * (skbench.hpp:536-546): element (mode, z) at z + mode_stride*mode.  A split
 * view has both pointers; an interleaved view sets imag = NULL and real points
 * at complex (re, im) pairs. */
typedef struct skb_field_view {
    void* real;
    void* imag;
    uint64_t mode_stride;
} skb_field_view;

/* Accounting getters shared by every handle (skbench.hpp:401-416, 495-515,
 * 169-187).  planning_seconds = table and launch-configuration set-up. */
typedef struct skb_provider_info {
    double allocation_seconds;
    double planning_seconds;
    double other_setup_seconds;
    uint64_t persistent_bytes;
    uint64_t scratch_bytes;
    uint64_t planning_bytes;
    uint64_t active_kx;
    uint64_t full_kx;
    uint64_t row_transforms_per_direction;
    uint64_t column_transforms_per_direction;
    uint64_t omitted_column_transforms_per_direction;
    uint64_t launches_per_execution;
    int32_t precision;
    int32_t destroys_native_input;
    char library_identity[128];
    char version[64];
} skb_provider_info;

/* ---------------------------------------------------------------- library */
SKB_API const char* skb_last_error(void);
SKB_API const char* skb_version(void);
SKB_API int skb_device_count(int* count);
/* Select the device this library's calls on the calling thread use. */
SKB_API int skb_set_device(int device);
/* Synchronise the current device (host-side barrier for timing). */
SKB_API int skb_device_synchronize(void);
/* Measured FP32 and FP64 SIMT FMA throughput of the current device in
 * TFLOP/s (2 flops per FMA; independent FMA chains at full occupancy, best
 * of three runs of a few ms each).  No counterpart in the reference: it gives
 * the FFT, pointwise and FP64-plain kernels' rooflines a measured compute
 * peak.  Allocates a small device buffer for the kernels' results. */
SKB_API int skb_measure_simt_peaks(double* fp32_tflops, double* fp64_tflops);

/* ------------------------------------------------- model (host, no GPU)  */
/* retainedHorizontalModes, src/model.cpp:129-167. */
SKB_API int skb_retained_modes(const skb_workload* w, skb_retained_mode* out, uint64_t capacity, uint64_t* count);
/* squaredWavenumberGroups, src/model.cpp:169-207. */
SKB_API int skb_squared_wavenumber_groups(const skb_workload* w, skb_mode_group* out, uint64_t capacity, uint64_t* count);
/* modeOrderHash / verticalModeGroupHash / wvmSpectrumOrderHash,
 * src/model.cpp:209-217, 462-487; each buffer holds at least 32 chars. */
SKB_API int skb_order_hashes(const skb_workload* w, char* mode_hash, char* group_hash, char* wvm_hash);
/* makeFixture, src/model.cpp:618-661; kind 0 impulse, 1 sinusoid, 2 random,
 * 3 dc, 4 nyquist; out holds nx*ny*nz*fields doubles. */
SKB_API int skb_make_fixture(const skb_workload* w, int kind, uint64_t seed, double* out);
/* Vertical operator family: forward[g][j][z], inverse[g][z][j] for
 * groups*nj*nz doubles each (groups = 1 for SKB_FAMILY_COMMON_DCT2);
 * orthonormalVerticalFixture / squaredWavenumberVerticalFixture,
 * src/model.cpp:489-565.  id holds at least 96 chars. */
SKB_API int skb_vertical_family(const skb_workload* w, int family, uint64_t seed, double* forward, double* inverse,
                        uint64_t capacity, uint64_t* groups, char* id);

/* ---------------------------------------------- full 2-D r2c/c2r provider */
/* Replaces FFTWProvider (skbench.hpp:364-421; src/fftw_provider.cpp:206-917). */
typedef struct skb_fft_provider skb_fft_provider;
SKB_API int skb_fft_create(const skb_workload* w, int precision, skb_fft_provider** out);
SKB_API int skb_fft_destroy(skb_fft_provider* p);
SKB_API int skb_fft_info(const skb_fft_provider* p, skb_provider_info* info);
/* forward(const double*, Complex*), fftw_provider.cpp:304-309. */
SKB_API int skb_fft_forward(skb_fft_provider* p, const double* input, skb_complex* wvm_spectrum);
/* inverse(Complex*, double*), fftw_provider.cpp:311-316; the input is preserved. */
SKB_API int skb_fft_inverse(skb_fft_provider* p, skb_complex* wvm_spectrum, double* output);
/* forwardSplit / inverseSplit, skbench.hpp:390-391. */
SKB_API int skb_fft_forward_split(skb_fft_provider* p, const double* input, double* spectrum_real, double* spectrum_imag);
SKB_API int skb_fft_inverse_split(skb_fft_provider* p, double* spectrum_real, double* spectrum_imag, double* output);
/* gatherRetainedOuter / embedRetainedOuter and the split/scale variants,
 * fftw_provider.cpp:318-395. */
SKB_API int skb_fft_gather_retained(skb_fft_provider* p, const skb_complex* wvm_spectrum, skb_complex* retained);
SKB_API int skb_fft_embed_retained(skb_fft_provider* p, const skb_complex* retained, skb_complex* wvm_spectrum);
SKB_API int skb_fft_gather_retained_to_split(skb_fft_provider* p, const skb_complex* wvm_spectrum, double* retained_real,
                                     double* retained_imag, double scale);
SKB_API int skb_fft_embed_retained_from_split(skb_fft_provider* p, const double* retained_real, const double* retained_imag,
                                      skb_complex* wvm_spectrum);
/* Device forms. */
SKB_API int skb_fft_forward_device(skb_fft_provider* p, const void* real, void* wvm_spectrum, void* stream);
SKB_API int skb_fft_inverse_device(skb_fft_provider* p, const void* wvm_spectrum, void* real, void* stream);
SKB_API int skb_fft_gather_retained_device(skb_fft_provider* p, const void* wvm_spectrum, const skb_field_view* views,
                                   uint64_t view_count, double scale, void* stream);
SKB_API int skb_fft_embed_retained_device(skb_fft_provider* p, const skb_field_view* views, uint64_t view_count,
                                  void* wvm_spectrum, void* stream);
/* Handle-free dense inverse that allocates nothing.  It has no counterpart in
 * the reference.  It is for callers that may not allocate device memory while
 * they run: a host that enforces its own device-memory budget through its own
 * allocator, or a plugin whose host forbids cudaMalloc / cudaFree inside its
 * compute callbacks (an allocation can fail once the budget is reserved, and
 * cudaFree stalls every stream on the device).  The result equals that of
 * skb_fft_inverse_device for the same workload and precision to within
 * rounding, not bit for bit: the twiddle tables here are computed on the
 * device with sincospi, the handle's are built on the host (both are tested
 * against the CPU oracle at 1e-12 relative for FP64 and 1e-5 for FP32).  The
 * spectrum is preserved.  The scratch (twiddle tables and the column-transformed
 * spectrum) is a fixed 64 MiB device array inside this library, which every
 * GPU that loads the library holds until the process exits; a workload that
 * needs more is refused with SKB_ERR_INVALID_ARGUMENT.  The first call on each
 * device looks the array's address up and may make the driver load the
 * library's device code, so make that call before any stream capture begins;
 * the address kept belongs to the device's current context, so after a
 * cudaDeviceReset of that device the entry point must not be called on it again
 * in the same process.
 * Each call writes everything it later reads, so nothing has to start at zero,
 * but all calls share the one array: calls whose GPU work overlaps (other
 * streams, other threads) race and corrupt each other; serialise them.
 * stream NULL is the legacy default stream. */
SKB_API int skb_fft_inverse_device_noalloc(const skb_workload* w, int precision, const void* wvm_spectrum, void* real,
                                           void* stream);

/* ------------------------------------------- pruned horizontal provider */
/* Replaces FFTWPrunedProvider (skbench.hpp:467-520) and
 * FFTWStreamingPrunedSplitProvider (skbench.hpp:534-624): row r2c/c2r on all
 * rows, column c2c only on the active kx band, retention / embedding with the
 * kx = 0 Hermitian repair fused into the column kernels. */
typedef struct skb_pruned_provider skb_pruned_provider;
SKB_API int skb_pruned_create(const skb_workload* w, int precision, skb_pruned_provider** out);
SKB_API int skb_pruned_destroy(skb_pruned_provider* p);
SKB_API int skb_pruned_info(const skb_pruned_provider* p, skb_provider_info* info);
/* forward / forwardSplit / inverse / inverseSplit, pruned_fftw_provider.cpp:230-269. */
SKB_API int skb_pruned_forward(skb_pruned_provider* p, const double* input, skb_complex* retained);
SKB_API int skb_pruned_forward_split(skb_pruned_provider* p, const double* input, double* retained_real,
                             double* retained_imag, double scale);
SKB_API int skb_pruned_inverse(skb_pruned_provider* p, const skb_complex* retained, double* output);
SKB_API int skb_pruned_inverse_split(skb_pruned_provider* p, const double* retained_real, const double* retained_imag,
                             double* output);
/* forwardSplitFields / inverseSplitFields, pruned_fftw_provider.cpp:787-805;
 * one host view per field, split layout. */
SKB_API int skb_pruned_forward_split_fields(skb_pruned_provider* p, const double* input, const skb_field_view* fields,
                                    uint64_t field_count, double scale);
SKB_API int skb_pruned_inverse_split_fields(skb_pruned_provider* p, const skb_field_view* fields, uint64_t field_count,
                                    double* output);
/* Device forms over field views (views may be split or interleaved). */
SKB_API int skb_pruned_forward_device(skb_pruned_provider* p, const void* real, const skb_field_view* fields,
                              uint64_t field_count, double scale, void* stream);
SKB_API int skb_pruned_inverse_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t field_count,
                              void* real, void* stream);
/* Component stages for diagnostic timings (executeForwardRows /
 * executeForwardColumns+gather / embed+executeInverseColumns /
 * executeInverseRows, skbench.hpp:478-492); they use the handle's scratch. */
SKB_API int skb_pruned_forward_rows_device(skb_pruned_provider* p, const void* real, void* stream);
SKB_API int skb_pruned_forward_columns_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t field_count,
                                      double scale, void* stream);
SKB_API int skb_pruned_inverse_columns_device(skb_pruned_provider* p, const skb_field_view* fields, uint64_t field_count,
                                      void* stream);
SKB_API int skb_pruned_inverse_rows_device(skb_pruned_provider* p, void* real, void* stream);

/* ----------------------------------------------- vertical GEMM provider */
/* Replaces VerticalGemmProvider (skbench.hpp:152-218,
 * src/vertical_gemm.cpp:270-634).  forward/inverse matrices are the family in
 * reference layout (forward[g][j][z], inverse[g][z][j]); groups are the K^2
 * groups (one group covering every mode for the common family). */
typedef struct skb_vertical_provider skb_vertical_provider;
SKB_API int skb_vertical_create(const skb_workload* w, const skb_mode_group* groups, uint64_t group_count,
                        const double* forward, const double* inverse, int layout, int buffer_policy,
                        int gemm_precision, skb_vertical_provider** out);
SKB_API int skb_vertical_destroy(skb_vertical_provider* p);
SKB_API int skb_vertical_info(const skb_vertical_provider* p, skb_provider_info* info);
/* loadPhysicalInput / loadModalInput / executeForward / executeInverse /
 * copyForwardOutput / copyInverseOutput, vertical_gemm.cpp:731-770 (host
 * arrays; interleaved layout). */
SKB_API int skb_vertical_load_physical_input(skb_vertical_provider* p, const skb_complex* input);
SKB_API int skb_vertical_load_modal_input(skb_vertical_provider* p, const skb_complex* input);
SKB_API int skb_vertical_execute_forward(skb_vertical_provider* p);
SKB_API int skb_vertical_execute_inverse(skb_vertical_provider* p);
SKB_API int skb_vertical_copy_forward_output(skb_vertical_provider* p, skb_complex* output);
SKB_API int skb_vertical_copy_inverse_output(skb_vertical_provider* p, skb_complex* output);
/* Split-layout host loads and copies (split*Data accessors, skbench.hpp:203-210). */
SKB_API int skb_vertical_load_physical_input_split(skb_vertical_provider* p, const double* real, const double* imag);
SKB_API int skb_vertical_load_modal_input_split(skb_vertical_provider* p, const double* real, const double* imag);
SKB_API int skb_vertical_copy_forward_output_split(skb_vertical_provider* p, double* real, double* imag);
SKB_API int skb_vertical_copy_inverse_output_split(skb_vertical_provider* p, double* real, double* imag);
/* Device forms: imag = NULL means interleaved complex in `real`. */
SKB_API int skb_vertical_forward_device(skb_vertical_provider* p, const void* in_real, const void* in_imag, void* out_real,
                                void* out_imag, void* stream);
SKB_API int skb_vertical_inverse_device(skb_vertical_provider* p, const void* in_real, const void* in_imag, void* out_real,
                                void* out_imag, void* stream);

/* Test of the failure path (no counterpart in the reference; the reference's
 * CPU GEMMs cannot wait on a device).  With enable != 0, every later launch of
 * this tensor-core (SKB_GEMM_TF32X3) provider makes its MMA lane wait first on
 * a device barrier that nothing signals.  That wait is bounded like every wait
 * of the kernel, so it runs out: the kernel records the expiry, every role of
 * every CTA stops, outstanding copies are drained and TMEM is freed, and the
 * next host-array call reports SKB_ERR_RUNTIME ("a bounded device wait
 * expired").  The handle stays in that state; the CUDA context stays usable. */
SKB_API int skb_vertical_expire_wait_for_test(skb_vertical_provider* p, int enable);

/* ------------------------------------ WVM-direct vertical GEMM provider */
/* Replaces WvmDirectVerticalGemmProvider (skbench.hpp:220-257,
 * src/vertical_gemm.cpp:935-1169): per retained mode, the group matrix times
 * the mode's stored cell of a full WVM spectrum [ky][kx][field][z] (fields are
 * the columns; the stored values are used as they are, no conjugation),
 * written to the same cell of a full WVM modal spectrum [ky][kx][field][j];
 * then the kx = 0 boundary copy (copyModalBoundary / copySpectrumBoundary):
 * the partner cell (0, Ny - ky) receives the conjugate.  Output cells that
 * hold no retained mode are not written; initialize_*_output zero a host
 * output once (initializeModalOutput / initializeSpectrumOutput).  Groups and
 * matrices as for skb_vertical_create.  One launch per direction. */
typedef struct skb_vertical_wvm_provider skb_vertical_wvm_provider;
SKB_API int skb_vertical_wvm_create(const skb_workload* w, const skb_mode_group* groups, uint64_t group_count,
                                    const double* forward, const double* inverse, int buffer_policy,
                                    int gemm_precision, skb_vertical_wvm_provider** out);
SKB_API int skb_vertical_wvm_destroy(skb_vertical_wvm_provider* p);
SKB_API int skb_vertical_wvm_info(const skb_vertical_wvm_provider* p, skb_provider_info* info);
/* Complex element counts of the full WVM spectrum and modal spectrum. */
SKB_API int skb_vertical_wvm_sizes(const skb_vertical_wvm_provider* p, uint64_t* spectrum_elements,
                                   uint64_t* modal_elements);
/* executeForward / executeInverse on host FP64 arrays. */
SKB_API int skb_vertical_wvm_forward(skb_vertical_wvm_provider* p, const skb_complex* spectrum, skb_complex* modal);
SKB_API int skb_vertical_wvm_inverse(skb_vertical_wvm_provider* p, const skb_complex* modal, skb_complex* spectrum);
SKB_API int skb_vertical_wvm_initialize_modal_output(const skb_vertical_wvm_provider* p, skb_complex* modal);
SKB_API int skb_vertical_wvm_initialize_spectrum_output(const skb_vertical_wvm_provider* p, skb_complex* spectrum);
/* Device forms: FP64 complex for SKB_GEMM_FP64, FP32 complex otherwise. */
SKB_API int skb_vertical_wvm_forward_device(skb_vertical_wvm_provider* p, const void* spectrum, void* modal,
                                            void* stream);
SKB_API int skb_vertical_wvm_inverse_device(skb_vertical_wvm_provider* p, const void* modal, void* spectrum,
                                            void* stream);

/* ------------------------------------------------- pointwise advection */
/* Replaces PointwiseAdvectionExecutor (src/pointwise_advection.hpp:18-43). */
typedef struct skb_pointwise_executor skb_pointwise_executor;
SKB_API int skb_pointwise_create(uint64_t volume_elements, double scale, int precision, skb_pointwise_executor** out);
SKB_API int skb_pointwise_destroy(skb_pointwise_executor* p);
/* execute(shared, derivative, target), pointwise_advection.cpp:178-195. */
SKB_API int skb_pointwise_execute(skb_pointwise_executor* p, const double* shared, const double* derivative, double* target);
SKB_API int skb_pointwise_execute_device(skb_pointwise_executor* p, const void* shared, const void* derivative, void* target,
                                 void* stream);

/* ------------------------------------------------- 15 -> 4 flux pipeline */
/* The composed streamed flux of runProductionLifetimeFluxBenchmark's
 * executeAll (src/benchmark.cpp:4405-4424): inverse vertical GEMM of the
 * 3+3T modal inputs, inverse pruned horizontal of [U,V,W], then per target the
 * inverse of its derivative triple, pointwise advection with scale
 * 1/(Nx*Ny)^2, forward pruned horizontal + retention, and the forward vertical
 * GEMM of the T targets.  T = 4 is the reference's 15 -> 4 boundary; T = 3 is
 * the 12 -> 3 serving variant.  `members` independent ensemble members are
 * evaluated per call, member-major: input [member][mode][field][j]. */
#define SKB_FLUX_FP64_PLAIN 0
#define SKB_FLUX_FP32 1
#define SKB_FLUX_SPLIT_TF32X3 2
#define SKB_FLUX_SPLIT_BF16X3 3

typedef struct skb_flux_options {
    uint64_t n;        /* Nx = Ny */
    uint64_t nz;
    uint64_t targets;  /* 4 (15 -> 4) or 3 (12 -> 3) */
    uint64_t members;  /* ensemble members per call */
    int32_t mode;      /* SKB_FLUX_* */
    int32_t family;    /* SKB_FAMILY_K2_ROTATION or SKB_FAMILY_STURM_LIOUVILLE */
    uint64_t family_seed;
} skb_flux_options;

typedef struct skb_flux skb_flux;
SKB_API int skb_flux_create(const skb_flux_options* options, skb_flux** out);
/* The authoritative WVM form (runAuthoritativeProductionLifetimeFluxBenchmark,
 * src/authoritative_spectral_flux.cpp:1409-1571; loadPreparedSpectralFluxFixture,
 * src/spectral_flux_fixture.cpp:150-411): the same 15 -> 4 composition with
 * the vertical operators of two families (wave-f = 0, wave-g = 1) given by the
 * caller over explicit operator groups (contiguous runs of the retained modes
 * in retainedHorizontalModes order; one matrix per group and family, groups
 * may share a K^2 key), each input slot and target using its family's
 * matrices.  options->family is ignored; targets must be 4. */
typedef struct skb_flux_families {
    uint64_t groups;              /* operator groups */
    const uint64_t* group_modes;  /* modes in each group, in order; sum = retained modes */
    const double* forward[2];     /* family f: [group][j][z], groups*Nj*Nz doubles */
    const double* inverse[2];     /* family f: [group][z][j] */
    uint32_t input_family[15];    /* family of each input slot */
    uint32_t target_family[4];    /* family of each target */
} skb_flux_families;
SKB_API int skb_flux_create_families(const skb_flux_options* options, const skb_flux_families* families,
                                     skb_flux** out);
SKB_API int skb_flux_destroy(skb_flux* p);
SKB_API int skb_flux_info(const skb_flux* p, skb_provider_info* info);
/* Sizes in complex elements for all members. */
SKB_API int skb_flux_sizes(const skb_flux* p, uint64_t* modes, uint64_t* nj, uint64_t* input_elements,
                   uint64_t* output_elements);
/* Host arrays (double complex), blocking. */
SKB_API int skb_flux_execute(skb_flux* p, const skb_complex* modal_input, skb_complex* modal_output);
/* Device arrays, the first `members` (1..capacity) ensemble members only. */
SKB_API int skb_flux_execute_device_members(skb_flux* p, const void* modal_input, void* modal_output,
                                            uint64_t members, void* stream);
/* Device arrays: FP64 complex for SKB_FLUX_FP64_PLAIN, FP32 complex otherwise. */
SKB_API int skb_flux_execute_device(skb_flux* p, const void* modal_input, void* modal_output, void* stream);
/* One execute_device with CUDA events between stages: per stage the device
 * milliseconds, kernel launches and algorithmic bytes / flops (for roofline
 * reporting).  `count` receives the number of stages. */
typedef struct skb_stage_time {
    char name[48];
    double ms;
    uint64_t launches;
    double algorithmic_bytes;
    double flops;
} skb_stage_time;
SKB_API int skb_flux_profile(skb_flux* p, const void* modal_input, void* modal_output, skb_stage_time* stages,
                             uint64_t capacity, uint64_t* count);
/* Raises SKB_ERR_RUNTIME if a bounded wait inside a tensor-core kernel of
 * this handle expired since creation (the kernel then skipped its work and
 * released its tensor memory instead of hanging). */
SKB_API int skb_flux_check_device(skb_flux* p);
/* Test of the fused row kernel's failure path (no counterpart in the
 * reference).  With enable != 0, later launches of the row kernel's TMA forms
 * (the autotuner's flux.rows.tma = 1 or 2) make thread 0 of every CTA wait,
 * once its first stage copy has landed, on a barrier nothing signals.  The
 * wait is bounded (a short limit), so it runs out: every thread of the CTA
 * leaves, the kernel's error word is set, and skb_flux_check_device reports
 * SKB_ERR_RUNTIME.  Other row-kernel forms ignore the flag.  Executions that
 * are not already captured in a graph pick it up. */
SKB_API int skb_flux_rows_expire_wait_for_test(skb_flux* p, int enable);
/* Capture execute_device on these buffers into a CUDA graph and replay it. */
SKB_API int skb_flux_capture_graph(skb_flux* p, const void* modal_input, void* modal_output);
SKB_API int skb_flux_replay_graph(skb_flux* p, void* stream);

/* ---------------------------------------------------------- autotuner */
/* The project autotuner picks the fused flux path's launch shapes (work-unit
 * size of each tensor-core GEMM: 4, 8, 16 or 32 M-tiles; z-planes per CTA of
 * the fused row kernel: 4, 8 or 16; kernel form of each 512-point band column
 * stage: direct, warp-per-plane, persistent direct, or direct at four CTAs
 * per SM) by timing every candidate with CUDA events on the caller's device
 * buffers.  Choices are
 * cached per (stage shape, device) for the process and, when the environment
 * variable SKB_TUNE_CACHE names a file, in that file (one "<value> <ms> <key>"
 * line per choice); every flux handle created afterwards with the same shape
 * starts with them.  skb_flux_autotune measures what is not cached yet,
 * applies the choices, leaves the flux of modal_input in modal_output, drops
 * any captured graph (capture again afterwards), adds the time to the
 * handle's planning seconds, and writes "key = value (ms)" lines to summary
 * (NUL-terminated, truncated to capacity; may be NULL).  The staged FP64 and
 * FP32 modes have no tuned shapes (an empty summary). */
SKB_API int skb_flux_autotune(skb_flux* p, const void* modal_input, void* modal_output, char* summary,
                              uint64_t capacity);
/* Host-side access to the cache (no GPU needed). */
SKB_API int skb_tune_cache_size(uint64_t* count);
SKB_API int skb_tune_cache_entry(uint64_t index, char* key, uint64_t key_capacity, int* value, double* ms);
SKB_API int skb_tune_cache_store(const char* key, int value, double ms);
SKB_API int skb_tune_cache_lookup(const char* key, int* value, int* found);
SKB_API int skb_tune_cache_clear(void);
SKB_API int skb_tune_cache_load(const char* path, uint64_t* count);
SKB_API int skb_tune_cache_save(const char* path, uint64_t* count);

/* ---------------------------------------------- spectral-pipeline round trip */
/* The spectral-pipeline kernel of skbench (runSpectralPipelineBenchmark,
 * src/benchmark.cpp:2978-3956; reference order 3072-3110): r2c with radial 2/3
 * retention, K^2-grouped vertical forward (pair-rotation family), synthetic
 * modal work (each modal value times syntheticModalWorkWeights,
 * src/model.cpp:246-274), vertical inverse, embedding with the kx = 0 repair,
 * and the unnormalised c2r.  SKB_PRECISION_FP64: FP64 transforms and FP64
 * GEMMs; SKB_PRECISION_FP32: FP32 transforms and split-TF32x3 tensor-core
 * GEMMs.  Real [field][z][y][x] in and out. */
typedef struct skb_pipeline skb_pipeline;
/* syntheticModalWorkWeights: modes*fields*nj doubles, [mode][field][j]. */
SKB_API int skb_modal_weights(const skb_workload* w, double* out);
SKB_API int skb_pipeline_create(const skb_workload* w, int precision, skb_pipeline** out);
SKB_API int skb_pipeline_destroy(skb_pipeline* p);
SKB_API int skb_pipeline_info(const skb_pipeline* p, skb_provider_info* info);
/* Host FP64 arrays, blocking. */
SKB_API int skb_pipeline_execute(skb_pipeline* p, const double* real_in, double* real_out);
/* Device arrays of the handle's precision, stream-ordered. */
SKB_API int skb_pipeline_execute_device(skb_pipeline* p, const void* real_in, void* real_out, void* stream);
/* One device execution with per-stage event times and algorithmic bytes. */
SKB_API int skb_pipeline_profile(skb_pipeline* p, const void* real_in, void* real_out, skb_stage_time* stages,
                                 uint64_t capacity, uint64_t* count);
SKB_API void* skb_pipeline_stream(skb_pipeline* p);

/* ------------------------------- constant-stratification type-I vertical */
/* Replaces the six FFTW guru64 REDFT00/RODFT00 plans of the constant-
 * stratification kernel (R2RPlan, src/constant_stratification.cpp:95-146),
 * the WVM forward normalisations (normalizeForwardDct / normalizeForwardDst,
 * 199-231) and the production call schedule (executeCompleteVerticalGraph,
 * 359-379).  Arrays are complex [row][storage_channels][nz] with z adjacent
 * (re/im interleaved; double for SKB_PRECISION_FP64 handles, float for FP32),
 * transformed in place; channels first_channel .. +channels-1 of each row.
 *   SKB_TYPE1_DCT: DCT-I over all nz points (unnormalised, FFTW REDFT00).
 *   SKB_TYPE1_DST: DST-I over the nz-2 interior points (RODFT00); the two
 *                  endpoints are left as they are.
 * normalize != 0 appends the WVM forward normalisation: DCT values times
 * 1/(nz-1) with the last point halved; DST interior times 1/(nz-1) with both
 * endpoints set to zero.  nz >= 3. */
#define SKB_TYPE1_DCT 0
#define SKB_TYPE1_DST 1
typedef struct skb_cs_vertical skb_cs_vertical;
SKB_API int skb_cs_vertical_create(uint64_t rows, uint64_t nz, int precision, skb_cs_vertical** out);
SKB_API int skb_cs_vertical_destroy(skb_cs_vertical* p);
SKB_API int skb_cs_vertical_info(const skb_cs_vertical* p, skb_provider_info* info);
/* R2RPlan::execute (+ normalisation) on a device array, stream-ordered. */
SKB_API int skb_cs_vertical_transform_device(skb_cs_vertical* p, int kind, uint64_t storage_channels,
                                             uint64_t first_channel, uint64_t channels, int normalize, void* data,
                                             void* stream);
/* The same on a host array (FP64 interleaved complex), blocking. */
SKB_API int skb_cs_vertical_transform(skb_cs_vertical* p, int kind, uint64_t storage_channels,
                                      uint64_t first_channel, uint64_t channels, int normalize, double* data);
/* normalizeForwardDct / normalizeForwardDst alone, on a device array. */
SKB_API int skb_cs_vertical_normalize_device(skb_cs_vertical* p, int kind, uint64_t storage_channels,
                                             uint64_t first_channel, uint64_t channels, void* data, void* stream);
/* executeCompleteVerticalGraph: 15 inverse channel transforms on arena3
 * ([rows][3][nz]) and 4 normalised forward transforms on arena1
 * ([rows][1][nz]).  Device arrays, stream-ordered. */
SKB_API int skb_cs_vertical_schedule_device(skb_cs_vertical* p, void* arena3, void* arena1, void* stream);
/* The same on host arrays (FP64 interleaved complex), blocking. */
SKB_API int skb_cs_vertical_schedule(skb_cs_vertical* p, double* arena3, double* arena1);
SKB_API void* skb_cs_vertical_stream(skb_cs_vertical* p);

/* ------------------------------------------------------ serving loop */
/* A continuous-batching request loop over flux size classes (no counterpart
 * in the reference, which has no serving path).  Each class gets one or more
 * slots — a flux pipeline for `max_batch` members on its own stream — while
 * they fit `hbm_budget_bytes`; queued requests of a class join the next free
 * slot's batch, and slots of all classes run concurrently.  Inputs are host
 * FP64 complex arrays of one member ([mode][field][j]) or resident states
 * loaded once; results are written to the caller's host array (pinned memory
 * keeps the copy asynchronous).  A member's result does not depend on the
 * other requests in its batch.  Slot streams carry priorities by class size
 * (the class with the least work per request highest), so a small request's
 * kernels are dispatched ahead of the waiting CTAs of a larger class's batch.
 * slot_bytes is the sum of the slots' own device allocations. */
typedef struct skb_server_class {
    uint64_t n, nz, targets, max_batch;
    int32_t mode; /* SKB_FLUX_* */
} skb_server_class;

typedef struct skb_server_stats {
    uint64_t submitted, completed, batches, slots, resident_states;
    uint64_t slot_bytes, state_bytes, budget_bytes;
} skb_server_stats;

typedef struct skb_server skb_server;
SKB_API int skb_server_create(const skb_server_class* classes, uint64_t class_count, uint64_t hbm_budget_bytes,
                              int max_slots_per_class, skb_server** out);
SKB_API int skb_server_destroy(skb_server* s);
SKB_API int skb_server_sizes(skb_server* s, int size_class, uint64_t* input_elements, uint64_t* output_elements);
SKB_API int skb_server_submit(skb_server* s, int size_class, const skb_complex* input, skb_complex* output,
                              uint64_t* ticket);
/* Admission by HBM footprint: SKB_ERR_OUT_OF_MEMORY when the state does not fit. */
SKB_API int skb_server_load_state(skb_server* s, int size_class, const skb_complex* input, int64_t* state);
SKB_API int skb_server_release_state(skb_server* s, int64_t state);
SKB_API int skb_server_submit_state(skb_server* s, int64_t state, skb_complex* output, uint64_t* ticket);
/* *done = 1 when finished within timeout_seconds; latency = submit -> result in host memory. */
SKB_API int skb_server_wait(skb_server* s, uint64_t ticket, double timeout_seconds, int* done, double* latency_ms);
SKB_API int skb_server_get_stats(skb_server* s, skb_server_stats* stats);
/* held = 1: queued requests wait and no new batch starts (running batches
 * finish); held = 0 releases them, so a burst submitted meanwhile is batched. */
SKB_API int skb_server_hold(skb_server* s, int held);

/* --------------------------------------------------------------- timing */
/* Events on a handle's stream, for benchmark harnesses. */
typedef struct skb_timer skb_timer;
SKB_API int skb_timer_create(skb_timer** out);
SKB_API int skb_timer_destroy(skb_timer* t);
SKB_API int skb_timer_start(skb_timer* t, void* stream);
SKB_API int skb_timer_stop(skb_timer* t, void* stream);
SKB_API int skb_timer_elapsed_ms(skb_timer* t, double* ms);
/* The stream a handle enqueues on (for callers that time around it). */
SKB_API void* skb_fft_stream(skb_fft_provider* p);
SKB_API void* skb_pruned_stream(skb_pruned_provider* p);
SKB_API void* skb_vertical_stream(skb_vertical_provider* p);
SKB_API void* skb_pointwise_stream(skb_pointwise_executor* p);
SKB_API void* skb_flux_stream(skb_flux* p);
SKB_API void* skb_vertical_wvm_stream(skb_vertical_wvm_provider* p);

/* Device buffers for callers without their own allocator (tests, bindings). */
SKB_API int skb_device_alloc(uint64_t bytes, void** ptr);
SKB_API int skb_device_free(void* ptr);
SKB_API int skb_host_alloc_pinned(uint64_t bytes, void** ptr);
SKB_API int skb_host_free_pinned(void* ptr);
SKB_API int skb_copy_to_device(void* dst, const void* src, uint64_t bytes, void* stream);
SKB_API int skb_copy_to_host(void* dst, const void* src, uint64_t bytes, void* stream);
SKB_API int skb_stream_synchronize(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SKB_CUDA_H */
