"""ctypes binding of libskb_cuda.so (include/skb_cuda.h).

Mirrors the reference's provider classes (include/skbench/skbench.hpp) with
numpy arrays on the host side:

    FFTProvider               FFTWProvider               (skbench.hpp:364-421)
    PrunedProvider            FFTWPrunedProvider /
                              FFTWStreamingPrunedSplitProvider (skbench.hpp:467-624)
    VerticalGemmProvider      VerticalGemmProvider       (skbench.hpp:152-218)
    PointwiseAdvectionExecutor PointwiseAdvectionExecutor (pointwise_advection.hpp:18-43)
    Flux                      the 15 -> 4 executeAll composition (benchmark.cpp:4405-4424)
    ConstantStratificationVertical
                              the type-I (REDFT00 / RODFT00) vertical plans of the
                              constant-stratification kernel
                              (constant_stratification.cpp:95-379)

Errors map to the reference's exception classes: ValueError for
std::invalid_argument, RuntimeError for std::runtime_error, LogicError for
std::logic_error and MemoryError for std::bad_alloc.  There is no fallback: if
the library is missing or no GPU is present, calls fail loudly.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(os.path.dirname(HERE), "libskb_cuda.so")

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_RUNTIME = -2
ERR_LOGIC = -3
ERR_OUT_OF_MEMORY = -4

FP64 = 0
FP32 = 1
GEMM_FP64, GEMM_FP32, GEMM_TF32X3, GEMM_BF16X3 = 0, 1, 2, 3
INTERLEAVED, SPLIT = 0, 1
BIDIRECTIONAL, FORWARD_ONLY, INVERSE_ONLY = 0, 1, 2
FAMILY_COMMON_DCT2, FAMILY_K2_ROTATION, FAMILY_STURM_LIOUVILLE = 0, 1, 2
TYPE1_DCT, TYPE1_DST = 0, 1
FLUX_FP64_PLAIN, FLUX_FP32, FLUX_SPLIT_TF32X3, FLUX_SPLIT_BF16X3 = 0, 1, 2, 3
FIXTURES = ("impulse", "sinusoid", "random", "dc", "nyquist")


class LogicError(RuntimeError):
    """std::logic_error: wrong layout or direction for this handle."""


class Workload(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64), ("nz", ctypes.c_uint64),
                ("fields", ctypes.c_uint64), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("antialias", ctypes.c_int32)]

    def __init__(self, nx, ny, nz, fields, lx=1.0, ly=1.0, antialias=True):
        super().__init__(nx, ny, nz, fields, lx, ly, 1 if antialias else 0)

    @property
    def planes(self):
        return self.nz * self.fields

    @property
    def nx_half(self):
        return self.nx // 2 + 1

    @property
    def nj(self):
        return 0 if self.nz < 2 else 2 * (self.nz - 1) // 3

    @property
    def real_elements(self):
        return self.nx * self.ny * self.planes

    @property
    def spectrum_elements(self):
        return self.nx_half * self.ny * self.planes


class RetainedMode(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int64), ("l", ctypes.c_int64), ("stored_kx", ctypes.c_uint64),
                ("stored_ky", ctypes.c_uint64), ("conjugates_stored_value", ctypes.c_int32),
                ("radial_mode", ctypes.c_double)]


class ModeGroup(ctypes.Structure):
    _fields_ = [("squared_mode_key", ctypes.c_uint64), ("first_mode", ctypes.c_uint64),
                ("mode_count", ctypes.c_uint64)]


class FieldView(ctypes.Structure):
    _fields_ = [("real", ctypes.c_void_p), ("imag", ctypes.c_void_p), ("mode_stride", ctypes.c_uint64)]


class ProviderInfo(ctypes.Structure):
    _fields_ = [("allocation_seconds", ctypes.c_double), ("planning_seconds", ctypes.c_double),
                ("other_setup_seconds", ctypes.c_double), ("persistent_bytes", ctypes.c_uint64),
                ("scratch_bytes", ctypes.c_uint64), ("planning_bytes", ctypes.c_uint64),
                ("active_kx", ctypes.c_uint64), ("full_kx", ctypes.c_uint64),
                ("row_transforms_per_direction", ctypes.c_uint64),
                ("column_transforms_per_direction", ctypes.c_uint64),
                ("omitted_column_transforms_per_direction", ctypes.c_uint64),
                ("launches_per_execution", ctypes.c_uint64), ("precision", ctypes.c_int32),
                ("destroys_native_input", ctypes.c_int32), ("library_identity", ctypes.c_char * 128),
                ("version", ctypes.c_char * 64)]

    def as_dict(self):
        out = {name: getattr(self, name) for name, _ in self._fields_}
        out["library_identity"] = self.library_identity.decode()
        out["version"] = self.version.decode()
        return out


class StageTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("ms", ctypes.c_double), ("launches", ctypes.c_uint64),
                ("algorithmic_bytes", ctypes.c_double), ("flops", ctypes.c_double)]


class FluxOptions(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("nz", ctypes.c_uint64), ("targets", ctypes.c_uint64),
                ("members", ctypes.c_uint64), ("mode", ctypes.c_int32), ("family", ctypes.c_int32),
                ("family_seed", ctypes.c_uint64)]


_LIB = None


def library():
    """Load libskb_cuda.so; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError("libskb_cuda.so is not built (run __graft_entry__.build() or "
                               "spectral-kernel-benchmarks_b200/build.py): " + LIBRARY_PATH)
        lib = ctypes.CDLL(LIBRARY_PATH)
        lib.skb_last_error.restype = ctypes.c_char_p
        lib.skb_version.restype = ctypes.c_char_p
        for name in ("skb_fft_stream", "skb_pruned_stream", "skb_vertical_stream", "skb_pointwise_stream",
                     "skb_flux_stream", "skb_vertical_wvm_stream", "skb_pipeline_stream", "skb_cs_vertical_stream"):
            getattr(lib, name).restype = ctypes.c_void_p
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        _LIB = lib
    return _LIB


def check(rc):
    if rc == OK:
        return
    msg = library().skb_last_error().decode()
    if rc == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == ERR_LOGIC:
        raise LogicError(msg)
    if rc == ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _u64(v):
    return ctypes.c_uint64(int(v))


def version():
    return library().skb_version().decode()


def device_count():
    n = ctypes.c_int(0)
    check(library().skb_device_count(ctypes.byref(n)))
    return n.value


def set_device(device):
    check(library().skb_set_device(ctypes.c_int(device)))


def synchronize():
    check(library().skb_device_synchronize())


def simt_peaks():
    """Measured FP32 and FP64 SIMT FMA throughput of the current device,
    (fp32_tflops, fp64_tflops)."""
    f32, f64 = ctypes.c_double(), ctypes.c_double()
    check(library().skb_measure_simt_peaks(ctypes.byref(f32), ctypes.byref(f64)))
    return f32.value, f64.value


# ------------------------------------------------------------------ model

def retained_modes(w: Workload):
    lib = library()
    n = ctypes.c_uint64()
    check(lib.skb_retained_modes(ctypes.byref(w), None, _u64(0), ctypes.byref(n)))
    arr = (RetainedMode * max(1, n.value))()
    check(lib.skb_retained_modes(ctypes.byref(w), arr, _u64(n.value), ctypes.byref(n)))
    return list(arr)[: n.value]


def squared_wavenumber_groups(w: Workload):
    lib = library()
    n = ctypes.c_uint64()
    check(lib.skb_squared_wavenumber_groups(ctypes.byref(w), None, _u64(0), ctypes.byref(n)))
    arr = (ModeGroup * max(1, n.value))()
    check(lib.skb_squared_wavenumber_groups(ctypes.byref(w), arr, _u64(n.value), ctypes.byref(n)))
    return list(arr)[: n.value]


def order_hashes(w: Workload, wvm=True):
    bufs = [ctypes.create_string_buffer(32) for _ in range(3)]
    check(library().skb_order_hashes(ctypes.byref(w), bufs[0], bufs[1], bufs[2] if wvm else None))
    return tuple(b.value.decode() for b in bufs)


def make_fixture(w: Workload, kind, seed):
    k = FIXTURES.index(kind) if isinstance(kind, str) else int(kind)
    out = np.empty(w.real_elements)
    check(library().skb_make_fixture(ctypes.byref(w), ctypes.c_int(k), _u64(seed), _p(out)))
    return out


def vertical_family(w: Workload, family=FAMILY_K2_ROTATION, seed=0):
    lib = library()
    groups = ctypes.c_uint64()
    ident = ctypes.create_string_buffer(96)
    check(lib.skb_vertical_family(ctypes.byref(w), ctypes.c_int(family), _u64(seed), None, None, _u64(0),
                                  ctypes.byref(groups), ident))
    size = groups.value * w.nj * w.nz
    fwd = np.empty(size)
    inv = np.empty(size)
    check(lib.skb_vertical_family(ctypes.byref(w), ctypes.c_int(family), _u64(seed), _p(fwd), _p(inv), _u64(size),
                                  ctypes.byref(groups), ident))
    return fwd, inv, ident.value.decode()


def _info(fn, handle):
    info = ProviderInfo()
    check(fn(handle, ctypes.byref(info)))
    return info.as_dict()


# ---------------------------------------------------------- device memory

class DeviceArray:
    """An owned device allocation with numpy upload / download."""

    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        ptr = ctypes.c_void_p()
        check(library().skb_device_alloc(_u64(max(1, self.nbytes)), ctypes.byref(ptr)))
        self.ptr = ptr.value

    @classmethod
    def from_numpy(cls, array, stream=None):
        a = np.ascontiguousarray(array)
        d = cls(a.nbytes)
        d.upload(a, stream)
        return d

    def upload(self, array, stream=None):
        a = np.ascontiguousarray(array)
        assert a.nbytes <= self.nbytes
        check(library().skb_copy_to_device(ctypes.c_void_p(self.ptr), _p(a), _u64(a.nbytes), ctypes.c_void_p(stream)))
        check(library().skb_stream_synchronize(ctypes.c_void_p(stream)))

    def download(self, dtype, count, stream=None):
        out = np.empty(count, dtype=dtype)
        check(library().skb_copy_to_host(_p(out), ctypes.c_void_p(self.ptr), _u64(out.nbytes), ctypes.c_void_p(stream)))
        check(library().skb_stream_synchronize(ctypes.c_void_p(stream)))
        return out

    def free(self):
        if self.ptr:
            check(library().skb_device_free(ctypes.c_void_p(self.ptr)))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedArray:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, dtype, count):
        self.dtype = np.dtype(dtype)
        self.count = int(count)
        ptr = ctypes.c_void_p()
        check(library().skb_host_alloc_pinned(_u64(max(1, self.count * self.dtype.itemsize)), ctypes.byref(ptr)))
        self.ptr = ptr.value
        buf = (ctypes.c_char * (self.count * self.dtype.itemsize)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=self.count)

    def free(self):
        if self.ptr:
            self.array = None
            check(library().skb_host_free_pinned(ctypes.c_void_p(self.ptr)))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Timer:
    """CUDA events recorded on a given stream."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(library().skb_timer_create(ctypes.byref(h)))
        self.h = h

    def start(self, stream):
        check(library().skb_timer_start(self.h, ctypes.c_void_p(stream)))

    def stop(self, stream):
        check(library().skb_timer_stop(self.h, ctypes.c_void_p(stream)))

    def elapsed_ms(self):
        ms = ctypes.c_double()
        check(library().skb_timer_elapsed_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            library().skb_timer_destroy(self.h)
        except Exception:
            pass


def field_views(views):
    """[(real_ptr, imag_ptr_or_None, mode_stride), ...] -> FieldView array."""
    arr = (FieldView * max(1, len(views)))()
    for i, (re, im, stride) in enumerate(views):
        arr[i] = FieldView(re, im, stride)
    return arr, len(views)


def _complex(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


# -------------------------------------------------------------------- FFT

class FFTProvider:
    """FFTWProvider drop-in: batched 2-D r2c/c2r in WVM frequency-major order."""

    def __init__(self, workload: Workload, precision=FP64):
        self.w = workload
        self.precision = precision
        h = ctypes.c_void_p()
        check(library().skb_fft_create(ctypes.byref(workload), ctypes.c_int(precision), ctypes.byref(h)))
        self.h = h

    @property
    def stream(self):
        return library().skb_fft_stream(self.h)

    def info(self):
        return _info(library().skb_fft_info, self.h)

    def forward(self, real):
        real = np.ascontiguousarray(real, dtype=np.float64)
        assert real.size == self.w.real_elements
        out = np.empty(self.w.spectrum_elements, np.complex128)
        check(library().skb_fft_forward(self.h, _p(real), _p(out)))
        return out

    def inverse(self, spectrum):
        spec = _complex(spectrum).copy()
        assert spec.size == self.w.spectrum_elements
        out = np.empty(self.w.real_elements)
        check(library().skb_fft_inverse(self.h, _p(spec), _p(out)))
        return out

    def forward_split(self, real):
        real = np.ascontiguousarray(real, dtype=np.float64)
        re = np.empty(self.w.spectrum_elements)
        im = np.empty(self.w.spectrum_elements)
        check(library().skb_fft_forward_split(self.h, _p(real), _p(re), _p(im)))
        return re, im

    def inverse_split(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64).copy()
        im = np.ascontiguousarray(im, dtype=np.float64).copy()
        out = np.empty(self.w.real_elements)
        check(library().skb_fft_inverse_split(self.h, _p(re), _p(im), _p(out)))
        return out

    def _modes(self):
        if not hasattr(self, "_mode_count"):
            self._mode_count = len(retained_modes(self.w))
        return self._mode_count

    def gather_retained(self, spectrum):
        spec = _complex(spectrum)
        out = np.empty(self._modes() * self.w.planes, np.complex128)
        check(library().skb_fft_gather_retained(self.h, _p(spec), _p(out)))
        return out

    def embed_retained(self, retained):
        ret = _complex(retained)
        out = np.empty(self.w.spectrum_elements, np.complex128)
        check(library().skb_fft_embed_retained(self.h, _p(ret), _p(out)))
        return out

    def gather_retained_to_split(self, spectrum, scale=1.0):
        spec = _complex(spectrum)
        n = self._modes() * self.w.planes
        re, im = np.empty(n), np.empty(n)
        check(library().skb_fft_gather_retained_to_split(self.h, _p(spec), _p(re), _p(im), ctypes.c_double(scale)))
        return re, im

    def embed_retained_from_split(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        out = np.empty(self.w.spectrum_elements, np.complex128)
        check(library().skb_fft_embed_retained_from_split(self.h, _p(re), _p(im), _p(out)))
        return out

    def forward_device(self, real_ptr, spectrum_ptr, stream=None):
        check(library().skb_fft_forward_device(self.h, ctypes.c_void_p(real_ptr), ctypes.c_void_p(spectrum_ptr),
                                               ctypes.c_void_p(stream)))

    def inverse_device(self, spectrum_ptr, real_ptr, stream=None):
        check(library().skb_fft_inverse_device(self.h, ctypes.c_void_p(spectrum_ptr), ctypes.c_void_p(real_ptr),
                                               ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_fft_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------- pruned

class PrunedProvider:
    """FFTWPrunedProvider / FFTWStreamingPrunedSplitProvider drop-in."""

    def __init__(self, workload: Workload, precision=FP64):
        self.w = workload
        self.precision = precision
        h = ctypes.c_void_p()
        check(library().skb_pruned_create(ctypes.byref(workload), ctypes.c_int(precision), ctypes.byref(h)))
        self.h = h
        self.modes = len(retained_modes(workload))

    @property
    def stream(self):
        return library().skb_pruned_stream(self.h)

    def info(self):
        return _info(library().skb_pruned_info, self.h)

    def active_kx_count(self):
        return self.info()["active_kx"]

    def forward(self, real):
        real = np.ascontiguousarray(real, dtype=np.float64)
        out = np.empty(self.modes * self.w.planes, np.complex128)
        check(library().skb_pruned_forward(self.h, _p(real), _p(out)))
        return out

    def forward_split(self, real, scale=1.0):
        real = np.ascontiguousarray(real, dtype=np.float64)
        n = self.modes * self.w.planes
        re, im = np.empty(n), np.empty(n)
        check(library().skb_pruned_forward_split(self.h, _p(real), _p(re), _p(im), ctypes.c_double(scale)))
        return re, im

    def inverse(self, retained):
        ret = _complex(retained)
        out = np.empty(self.w.real_elements)
        check(library().skb_pruned_inverse(self.h, _p(ret), _p(out)))
        return out

    def inverse_split(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        out = np.empty(self.w.real_elements)
        check(library().skb_pruned_inverse_split(self.h, _p(re), _p(im), _p(out)))
        return out

    def forward_split_fields(self, real, fields, scale=1.0):
        """fields: list of (real_array, imag_array, mode_stride) host arrays, written in place."""
        real = np.ascontiguousarray(real, dtype=np.float64)
        views, n = field_views([(f[0].ctypes.data, f[1].ctypes.data, f[2]) for f in fields])
        check(library().skb_pruned_forward_split_fields(self.h, _p(real), views, _u64(n), ctypes.c_double(scale)))

    def inverse_split_fields(self, fields):
        views, n = field_views([(f[0].ctypes.data, f[1].ctypes.data, f[2]) for f in fields])
        out = np.empty(self.w.real_elements)
        check(library().skb_pruned_inverse_split_fields(self.h, views, _u64(n), _p(out)))
        return out

    def forward_device(self, real_ptr, views, scale=1.0, stream=None):
        arr, n = field_views(views)
        check(library().skb_pruned_forward_device(self.h, ctypes.c_void_p(real_ptr), arr, _u64(n),
                                                  ctypes.c_double(scale), ctypes.c_void_p(stream)))

    def inverse_device(self, views, real_ptr, stream=None):
        arr, n = field_views(views)
        check(library().skb_pruned_inverse_device(self.h, arr, _u64(n), ctypes.c_void_p(real_ptr),
                                                  ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_pruned_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------- vertical

class VerticalGemmProvider:
    """VerticalGemmProvider drop-in over a K^2 (or common) operator family."""

    def __init__(self, workload: Workload, groups, forward, inverse, layout=INTERLEAVED, buffer_policy=BIDIRECTIONAL,
                 gemm_precision=GEMM_FP64):
        self.w = workload
        self.layout = layout
        garr = (ModeGroup * len(groups))(*[ModeGroup(g.squared_mode_key, g.first_mode, g.mode_count)
                                           for g in groups])
        self.modes = sum(g.mode_count for g in groups)
        self.columns = self.modes * workload.fields
        fwd = np.ascontiguousarray(forward, dtype=np.float64)
        inv = np.ascontiguousarray(inverse, dtype=np.float64)
        h = ctypes.c_void_p()
        check(library().skb_vertical_create(ctypes.byref(workload), garr, _u64(len(groups)), _p(fwd), _p(inv),
                                            ctypes.c_int(layout), ctypes.c_int(buffer_policy),
                                            ctypes.c_int(gemm_precision), ctypes.byref(h)))
        self.h = h

    @property
    def stream(self):
        return library().skb_vertical_stream(self.h)

    def info(self):
        return _info(library().skb_vertical_info, self.h)

    def load_physical_input(self, x):
        x = _complex(x)
        check(library().skb_vertical_load_physical_input(self.h, _p(x)))

    def load_modal_input(self, x):
        x = _complex(x)
        check(library().skb_vertical_load_modal_input(self.h, _p(x)))

    def load_physical_input_split(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        check(library().skb_vertical_load_physical_input_split(self.h, _p(re), _p(im)))

    def load_modal_input_split(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        check(library().skb_vertical_load_modal_input_split(self.h, _p(re), _p(im)))

    def execute_forward(self):
        check(library().skb_vertical_execute_forward(self.h))

    def execute_inverse(self):
        check(library().skb_vertical_execute_inverse(self.h))

    def copy_forward_output(self):
        out = np.empty(self.columns * self.w.nj, np.complex128)
        check(library().skb_vertical_copy_forward_output(self.h, _p(out)))
        return out

    def copy_inverse_output(self):
        out = np.empty(self.columns * self.w.nz, np.complex128)
        check(library().skb_vertical_copy_inverse_output(self.h, _p(out)))
        return out

    def copy_forward_output_split(self):
        re, im = np.empty(self.columns * self.w.nj), np.empty(self.columns * self.w.nj)
        check(library().skb_vertical_copy_forward_output_split(self.h, _p(re), _p(im)))
        return re, im

    def copy_inverse_output_split(self):
        re, im = np.empty(self.columns * self.w.nz), np.empty(self.columns * self.w.nz)
        check(library().skb_vertical_copy_inverse_output_split(self.h, _p(re), _p(im)))
        return re, im

    def forward_device(self, in_re, in_im, out_re, out_im, stream=None):
        check(library().skb_vertical_forward_device(self.h, ctypes.c_void_p(in_re), ctypes.c_void_p(in_im),
                                                    ctypes.c_void_p(out_re), ctypes.c_void_p(out_im),
                                                    ctypes.c_void_p(stream)))

    def inverse_device(self, in_re, in_im, out_re, out_im, stream=None):
        check(library().skb_vertical_inverse_device(self.h, ctypes.c_void_p(in_re), ctypes.c_void_p(in_im),
                                                    ctypes.c_void_p(out_re), ctypes.c_void_p(out_im),
                                                    ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_vertical_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -------------------------------------------------------------- pointwise

class WvmDirectVerticalProvider:
    """WvmDirectVerticalGemmProvider drop-in: per-mode grouped GEMM on full
    WVM-order spectra [ky][kx][field][z] <-> modal spectra [ky][kx][field][j],
    with the kx = 0 boundary copy; output cells without a retained mode are
    left as they are."""

    def __init__(self, workload: Workload, groups, forward, inverse, buffer_policy=BIDIRECTIONAL,
                 gemm_precision=GEMM_FP64):
        self.w = workload
        self.precision = gemm_precision
        garr = (ModeGroup * len(groups))(*[ModeGroup(g.squared_mode_key, g.first_mode, g.mode_count)
                                           for g in groups])
        fwd = np.ascontiguousarray(forward, dtype=np.float64)
        inv = np.ascontiguousarray(inverse, dtype=np.float64)
        h = ctypes.c_void_p()
        check(library().skb_vertical_wvm_create(ctypes.byref(workload), garr, _u64(len(groups)), _p(fwd), _p(inv),
                                                ctypes.c_int(buffer_policy), ctypes.c_int(gemm_precision),
                                                ctypes.byref(h)))
        self.h = h
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(library().skb_vertical_wvm_sizes(self.h, ctypes.byref(a), ctypes.byref(b)))
        self.spectrum_elements, self.modal_elements = a.value, b.value

    @property
    def stream(self):
        return library().skb_vertical_wvm_stream(self.h)

    @property
    def device_dtype(self):
        return np.complex128 if self.precision == GEMM_FP64 else np.complex64

    def info(self):
        return _info(library().skb_vertical_wvm_info, self.h)

    def forward(self, spectrum, out=None):
        x = _complex(spectrum)
        y = np.zeros(self.modal_elements, np.complex128) if out is None else _complex(out).copy()
        check(library().skb_vertical_wvm_forward(self.h, _p(x), _p(y)))
        return y

    def inverse(self, modal, out=None):
        x = _complex(modal)
        y = np.zeros(self.spectrum_elements, np.complex128) if out is None else _complex(out).copy()
        check(library().skb_vertical_wvm_inverse(self.h, _p(x), _p(y)))
        return y

    def forward_device(self, spectrum_ptr, modal_ptr, stream=None):
        check(library().skb_vertical_wvm_forward_device(self.h, ctypes.c_void_p(spectrum_ptr),
                                                        ctypes.c_void_p(modal_ptr), ctypes.c_void_p(stream)))

    def inverse_device(self, modal_ptr, spectrum_ptr, stream=None):
        check(library().skb_vertical_wvm_inverse_device(self.h, ctypes.c_void_p(modal_ptr),
                                                        ctypes.c_void_p(spectrum_ptr), ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_vertical_wvm_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def modal_weights(w: Workload):
    """syntheticModalWorkWeights: [mode][field][j] doubles."""
    out = np.empty(len(retained_modes(w)) * w.fields * w.nj)
    check(library().skb_modal_weights(ctypes.byref(w), _p(out)))
    return out


class SpectralPipeline:
    """The spectral-pipeline round trip: r2c + retention, K^2 vertical forward,
    synthetic modal work, vertical inverse, embedding + c2r (unnormalised)."""

    def __init__(self, workload: Workload, precision=FP64):
        self.w = workload
        self.precision = precision
        h = ctypes.c_void_p()
        check(library().skb_pipeline_create(ctypes.byref(workload), ctypes.c_int(precision), ctypes.byref(h)))
        self.h = h

    @property
    def stream(self):
        return library().skb_pipeline_stream(self.h)

    @property
    def device_dtype(self):
        return np.float64 if self.precision == FP64 else np.float32

    def info(self):
        return _info(library().skb_pipeline_info, self.h)

    def execute(self, real):
        x = np.ascontiguousarray(real, dtype=np.float64)
        assert x.size == self.w.real_elements
        out = np.empty_like(x)
        check(library().skb_pipeline_execute(self.h, _p(x), _p(out)))
        return out

    def execute_device(self, in_ptr, out_ptr, stream=None):
        check(library().skb_pipeline_execute_device(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                                    ctypes.c_void_p(stream)))

    def profile(self, in_ptr, out_ptr):
        stages = (StageTime * 16)()
        n = ctypes.c_uint64()
        check(library().skb_pipeline_profile(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), stages,
                                             _u64(16), ctypes.byref(n)))
        return [{"name": stages[i].name.decode(), "ms": stages[i].ms, "launches": stages[i].launches,
                 "bytes": stages[i].algorithmic_bytes} for i in range(n.value)]

    def close(self):
        if self.h:
            check(library().skb_pipeline_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_cache():
    """The autotuner's cache: {key: (value, ms)}."""
    lib = library()
    n = ctypes.c_uint64()
    check(lib.skb_tune_cache_size(ctypes.byref(n)))
    out = {}
    key = ctypes.create_string_buffer(1024)
    value = ctypes.c_int()
    ms = ctypes.c_double()
    for i in range(n.value):
        check(lib.skb_tune_cache_entry(_u64(i), key, _u64(len(key)), ctypes.byref(value), ctypes.byref(ms)))
        out[key.value.decode()] = (value.value, ms.value)
    return out


def tune_cache_store(key, value, ms=0.0):
    check(library().skb_tune_cache_store(key.encode(), ctypes.c_int(value), ctypes.c_double(ms)))


def tune_cache_lookup(key):
    """The cached value for key, or None."""
    value = ctypes.c_int()
    found = ctypes.c_int()
    check(library().skb_tune_cache_lookup(key.encode(), ctypes.byref(value), ctypes.byref(found)))
    return value.value if found.value else None


def tune_cache_clear():
    check(library().skb_tune_cache_clear())


def tune_cache_load(path):
    n = ctypes.c_uint64()
    check(library().skb_tune_cache_load(os.fsencode(path), ctypes.byref(n)))
    return n.value


def tune_cache_save(path):
    n = ctypes.c_uint64()
    check(library().skb_tune_cache_save(os.fsencode(path), ctypes.byref(n)))
    return n.value


class ConstantStratificationVertical:
    """Type-I vertical transforms of the constant-stratification kernel, in
    place on complex [row][storage_channels][nz] arrays (z adjacent).

    transform(..., kind=TYPE1_DCT) is FFTW's REDFT00 over all nz points,
    kind=TYPE1_DST its RODFT00 over the nz-2 interior points (endpoints left
    as they are); normalize=True appends the WVM forward normalisation
    (normalizeForwardDct / normalizeForwardDst).  schedule() is the
    production call graph executeCompleteVerticalGraph: 15 inverse channel
    transforms on a 3-channel arena and 4 normalised forward transforms on a
    1-channel arena."""

    def __init__(self, rows, nz, precision=FP64):
        self.rows = int(rows)
        self.nz = int(nz)
        self.precision = precision
        h = ctypes.c_void_p()
        check(library().skb_cs_vertical_create(_u64(rows), _u64(nz), ctypes.c_int(precision), ctypes.byref(h)))
        self.h = h

    @property
    def stream(self):
        return library().skb_cs_vertical_stream(self.h)

    @property
    def device_dtype(self):
        return np.float64 if self.precision == FP64 else np.float32

    def info(self):
        return _info(library().skb_cs_vertical_info, self.h)

    def _host(self, data, storage):
        x = np.ascontiguousarray(data, dtype=np.complex128).copy()
        assert x.size == self.rows * storage * self.nz
        return x

    def transform(self, data, kind, storage_channels, first_channel, channels, normalize=False):
        """Host array in, transformed copy out (complex128)."""
        x = self._host(data, storage_channels)
        check(library().skb_cs_vertical_transform(self.h, ctypes.c_int(kind), _u64(storage_channels),
                                                  _u64(first_channel), _u64(channels), ctypes.c_int(int(normalize)),
                                                  _p(x)))
        return x

    def transform_device(self, ptr, kind, storage_channels, first_channel, channels, normalize=False, stream=None):
        check(library().skb_cs_vertical_transform_device(self.h, ctypes.c_int(kind), _u64(storage_channels),
                                                         _u64(first_channel), _u64(channels),
                                                         ctypes.c_int(int(normalize)), ctypes.c_void_p(ptr),
                                                         ctypes.c_void_p(stream)))

    def normalize_device(self, ptr, kind, storage_channels, first_channel, channels, stream=None):
        check(library().skb_cs_vertical_normalize_device(self.h, ctypes.c_int(kind), _u64(storage_channels),
                                                         _u64(first_channel), _u64(channels), ctypes.c_void_p(ptr),
                                                         ctypes.c_void_p(stream)))

    def schedule(self, arena3, arena1):
        """Host arrays in, (arena3, arena1) after the production schedule out."""
        a3 = self._host(arena3, 3)
        a1 = self._host(arena1, 1)
        check(library().skb_cs_vertical_schedule(self.h, _p(a3), _p(a1)))
        return a3, a1

    def schedule_device(self, arena3_ptr, arena1_ptr, stream=None):
        check(library().skb_cs_vertical_schedule_device(self.h, ctypes.c_void_p(arena3_ptr),
                                                        ctypes.c_void_p(arena1_ptr), ctypes.c_void_p(stream)))

    def close(self):
        if getattr(self, "h", None):
            library().skb_cs_vertical_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PointwiseAdvectionExecutor:
    """PointwiseAdvectionExecutor drop-in: target = -scale*(u qx + v qy + w qz)."""

    def __init__(self, volume, scale, precision=FP64):
        self.volume = int(volume)
        h = ctypes.c_void_p()
        check(library().skb_pointwise_create(_u64(volume), ctypes.c_double(scale), ctypes.c_int(precision),
                                             ctypes.byref(h)))
        self.h = h

    @property
    def stream(self):
        return library().skb_pointwise_stream(self.h)

    def execute(self, shared, derivative):
        s = np.ascontiguousarray(shared, dtype=np.float64)
        d = np.ascontiguousarray(derivative, dtype=np.float64)
        out = np.empty(self.volume)
        check(library().skb_pointwise_execute(self.h, _p(s), _p(d), _p(out)))
        return out

    def execute_device(self, shared_ptr, derivative_ptr, target_ptr, stream=None):
        check(library().skb_pointwise_execute_device(self.h, ctypes.c_void_p(shared_ptr),
                                                     ctypes.c_void_p(derivative_ptr), ctypes.c_void_p(target_ptr),
                                                     ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_pointwise_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------- flux

class FluxFamilies(ctypes.Structure):
    _fields_ = [("groups", ctypes.c_uint64), ("group_modes", ctypes.POINTER(ctypes.c_uint64)),
                ("forward", ctypes.POINTER(ctypes.c_double) * 2), ("inverse", ctypes.POINTER(ctypes.c_double) * 2),
                ("input_family", ctypes.c_uint32 * 15), ("target_family", ctypes.c_uint32 * 4)]


class Flux:
    """The composed 15 -> 4 (targets=4) or 12 -> 3 (targets=3) flux.

    `families` (the authoritative WVM form): a dict with 'group_modes' (modes
    per operator group, retained-mode order), 'forward' / 'inverse' (per family
    [group][j][z] / [group][z][j]), 'input_family' (15) and 'target_family' (4),
    e.g. from skb_cuda.fixture.load; `family` is then ignored."""

    def __init__(self, n, nz, targets=4, members=1, mode=FLUX_FP64_PLAIN, family=FAMILY_K2_ROTATION, family_seed=0,
                 families=None):
        opts = FluxOptions(n, nz, targets, members, mode, family, family_seed)
        h = ctypes.c_void_p()
        if families is None:
            check(library().skb_flux_create(ctypes.byref(opts), ctypes.byref(h)))
        else:
            keep = [np.ascontiguousarray(families["group_modes"], dtype=np.uint64).reshape(-1)]
            groups, nj = len(keep[0]), (2 * (nz - 1) // 3 if nz >= 2 else 0)
            # The C ABI copies groups * Nj * Nz values from each matrix pointer:
            # refuse arrays of another shape here, before C reads past them.
            expect = {"forward": (groups, nj, nz), "inverse": (groups, nz, nj)}
            for name in ("forward", "inverse"):
                if len(families[name]) != 2:
                    raise ValueError(f"families['{name}'] must hold the wave-f and wave-g matrices (2 entries)")
                for f in range(2):
                    a = np.ascontiguousarray(families[name][f], dtype=np.float64)
                    if a.size != int(np.prod(expect[name])) or (a.ndim == 3 and a.shape != expect[name]):
                        raise ValueError(f"families['{name}'][{f}] has shape {a.shape}; expected {expect[name]} "
                                         f"([group][{'j][z' if name == 'forward' else 'z][j'}] for {groups} groups, "
                                         f"Nz={nz}, Nj={nj})")
                    keep.append(a)
            for name, count in (("input_family", 15), ("target_family", 4)):
                if len(families[name]) != count:
                    raise ValueError(f"families['{name}'] must map {count} slots to a family; got "
                                     f"{len(families[name])}")
            fam = FluxFamilies()
            fam.groups = len(keep[0])
            fam.group_modes = keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
            for f in range(2):
                fam.forward[f] = keep[1 + f].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                fam.inverse[f] = keep[3 + f].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            fam.input_family[:] = [int(v) for v in families["input_family"]]
            fam.target_family[:] = [int(v) for v in families["target_family"]]
            check(library().skb_flux_create_families(ctypes.byref(opts), ctypes.byref(fam), ctypes.byref(h)))
        self.h = h
        self.n, self.nz, self.targets, self.members, self.mode = n, nz, targets, members, mode
        m, nj, i, o = (ctypes.c_uint64() for _ in range(4))
        check(library().skb_flux_sizes(self.h, ctypes.byref(m), ctypes.byref(nj), ctypes.byref(i), ctypes.byref(o)))
        self.modes, self.nj, self.input_elements, self.output_elements = m.value, nj.value, i.value, o.value

    @property
    def stream(self):
        return library().skb_flux_stream(self.h)

    @property
    def device_dtype(self):
        return np.complex128 if self.mode == FLUX_FP64_PLAIN else np.complex64

    def info(self):
        return _info(library().skb_flux_info, self.h)

    def execute(self, modal_input):
        x = _complex(modal_input)
        assert x.size == self.input_elements
        out = np.empty(self.output_elements, np.complex128)
        check(library().skb_flux_execute(self.h, _p(x), _p(out)))
        return out

    def execute_host_ptr(self, in_ptr, out_ptr):
        check(library().skb_flux_execute(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr)))

    def execute_device(self, in_ptr, out_ptr, stream=None, members=None):
        if members is None:
            check(library().skb_flux_execute_device(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                                    ctypes.c_void_p(stream)))
        else:
            check(library().skb_flux_execute_device_members(self.h, ctypes.c_void_p(in_ptr),
                                                            ctypes.c_void_p(out_ptr), _u64(members),
                                                            ctypes.c_void_p(stream)))

    def profile(self, in_ptr, out_ptr):
        """One device execution with per-stage event timing -> list of dicts."""
        arr = (StageTime * 32)()
        n = ctypes.c_uint64()
        check(library().skb_flux_profile(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), arr, _u64(32),
                                         ctypes.byref(n)))
        return [dict(name=a.name.decode(), ms=a.ms, launches=a.launches, bytes=a.algorithmic_bytes, flops=a.flops)
                for a in arr[: n.value]]

    def check_device(self):
        check(library().skb_flux_check_device(self.h))

    def capture_graph(self, in_ptr, out_ptr):
        check(library().skb_flux_capture_graph(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr)))

    def autotune(self, in_ptr, out_ptr):
        """Project autotuner: measure the fused path's launch shapes on these
        device buffers (cached per shape and device), apply them and leave the
        flux in out_ptr.  Returns {key: (value, ms)}; a captured graph is
        dropped (capture again afterwards)."""
        buf = ctypes.create_string_buffer(8192)
        check(library().skb_flux_autotune(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), buf,
                                          _u64(len(buf))))
        out = {}
        for line in buf.value.decode().splitlines():
            key, _, rest = line.rpartition(" = ")
            value, _, ms = rest.partition(" (")
            out[key] = (int(value), float(ms.split(" ")[0]))
        return out

    def replay_graph(self, stream=None):
        check(library().skb_flux_replay_graph(self.h, ctypes.c_void_p(stream)))

    def close(self):
        if self.h:
            check(library().skb_flux_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ serving loop

class ServerClass(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("nz", ctypes.c_uint64), ("targets", ctypes.c_uint64),
                ("max_batch", ctypes.c_uint64), ("mode", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in ("submitted", "completed", "batches", "slots", "resident_states",
                                                     "slot_bytes", "state_bytes", "budget_bytes")]


class Server:
    """Continuous-batching flux request loop over size classes.

    classes: list of (n, nz, targets, max_batch, mode).  Outputs are written
    into caller arrays; keep them alive until wait() returns."""

    def __init__(self, classes, hbm_budget_bytes, max_slots_per_class=2):
        arr = (ServerClass * len(classes))(*[ServerClass(*c) for c in classes])
        h = ctypes.c_void_p()
        check(library().skb_server_create(arr, _u64(len(classes)), _u64(hbm_budget_bytes),
                                          ctypes.c_int(max_slots_per_class), ctypes.byref(h)))
        self.h = h
        self.sizes = []
        for i in range(len(classes)):
            a, b = ctypes.c_uint64(), ctypes.c_uint64()
            check(library().skb_server_sizes(self.h, ctypes.c_int(i), ctypes.byref(a), ctypes.byref(b)))
            self.sizes.append((a.value, b.value))
        self._keep = {}

    def submit(self, size_class, modal_input, output=None):
        x = _complex(modal_input)
        assert x.size == self.sizes[size_class][0]
        out = output if output is not None else np.empty(self.sizes[size_class][1], np.complex128)
        t = ctypes.c_uint64()
        check(library().skb_server_submit(self.h, ctypes.c_int(size_class), _p(x), _p(out), ctypes.byref(t)))
        self._keep[t.value] = (x, out)
        return t.value

    def load_state(self, size_class, modal_input):
        x = _complex(modal_input)
        sid = ctypes.c_int64()
        check(library().skb_server_load_state(self.h, ctypes.c_int(size_class), _p(x), ctypes.byref(sid)))
        return sid.value

    def release_state(self, state):
        check(library().skb_server_release_state(self.h, ctypes.c_int64(state)))

    def submit_state(self, state, output):
        t = ctypes.c_uint64()
        check(library().skb_server_submit_state(self.h, ctypes.c_int64(state), _p(output), ctypes.byref(t)))
        self._keep[t.value] = (None, output)
        return t.value

    def wait(self, ticket, timeout=60.0):
        """-> (output array, latency_ms); raises TimeoutError if not finished."""
        done, lat = ctypes.c_int(), ctypes.c_double()
        check(library().skb_server_wait(self.h, _u64(ticket), ctypes.c_double(timeout), ctypes.byref(done),
                                        ctypes.byref(lat)))
        if not done.value:
            raise TimeoutError(f"request {ticket} not finished within {timeout} s")
        _, out = self._keep.pop(ticket)
        return out, lat.value

    def hold(self, held=True):
        """While held, no new batch starts; release with hold(False)."""
        check(library().skb_server_hold(self.h, 1 if held else 0))

    def stats(self):
        st = ServerStats()
        check(library().skb_server_get_stats(self.h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            check(library().skb_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
