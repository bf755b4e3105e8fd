"""Python mirror of the reference's fcwt module (src/fcwt/fcwt.i, fcwt.py,
boilerplate.py of fastlib/fCWT) over the C ABI of libfcwt_b200.so.

Same names, arguments, in-place output conventions and errors as the SWIG
module, so code and tests written for ``import fcwt`` run against
``import fcwt_b200 as fcwt``. Inputs and outputs may be numpy arrays (host) or
torch CUDA tensors (device-resident; nothing is copied, work is enqueued on
torch's current stream). torch is imported only when a tensor is passed.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

from . import _lib
from ._lib import (FCWT_EXACT_SUPPORT, FCWT_NORM, FCWT_OUT_BF16, FCWT_OUT_C64, FCWT_OUT_F16,
                   FCWT_SCALAR_TRUNC, FCWT_STRICT, FcwtError)

# enum SCALETYPE (src/fcwt/fcwt.h:65)
FCWT_LINSCALES = 0
FCWT_LOGSCALES = 1
FCWT_LINFREQS = 2

_FFTW_FLAGS = {"FFTW_MEASURE": 1, "FFTW_PATIENT": 2, "FFTW_EXHAUSTIVE": 3, "FFTW_ESTIMATE": 0}


def _strict(strict) -> bool:
    """Strict Nyquist checks: the `strict` argument, else FCWT_STRICT=1 in the
    environment (the reference's asserts, src/fcwt/fcwt.cpp:148,167,184, are
    compiled out of its release builds, so the default accepts f1 > fs/2)."""
    if strict is not None:
        return bool(strict)
    v = os.environ.get("FCWT_STRICT", "")
    return bool(v) and v != "0"


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _positive(name: str, v) -> None:
    # fcwt.i:28-32: %typemap(check) float f0, float f1, int fn
    if v <= 0:
        raise ValueError("Expected a non-zero, positive value.")


def _as_int(name: str, v) -> int:
    if isinstance(v, (bool, np.bool_)):
        raise TypeError(f"argument '{name}' must be an int")
    if isinstance(v, (int, np.integer)):
        return int(v)
    if isinstance(v, (float, np.floating)) and float(v).is_integer():
        return int(v)
    raise TypeError(f"argument '{name}' must be an int")


class Wavelet:
    """Base class of the reference's wavelet interface (src/fcwt/fcwt.h:67-79)."""

    def __init__(self):
        self.width = 0
        self.four_wavelen = 0.0
        self.imag_frequency = False
        self.doublesided = False
        self.mother = None

    def generate(self, *args):
        raise NotImplementedError("Override this virtual class")

    def getSupport(self, scale):
        raise NotImplementedError("Override this virtual class")

    def getWavelet(self, scale, pwav):
        raise NotImplementedError("Override this virtual class")


class Morlet(Wavelet):
    """Morlet(bandwidth) (src/fcwt/fcwt.cpp:41-49)."""

    def __init__(self, bandwidth):
        super().__init__()
        self.fb = float(np.float32(bandwidth))
        self.four_wavelen = float(np.float32(0.9876))

    def generate(self, *args):
        """generate(size): frequency-domain mother table of length size, computed
        on the GPU (src/fcwt/fcwt.cpp:51-67); stored in ``self.mother``.
        generate(real, imag, size, scale): time-domain wavelet written into the
        float32 arrays real/imag (2*getSupport(scale)+1 taps, fcwt.cpp:68-84)."""
        if len(args) == 1:
            size = _as_int("size", args[0])
            self.width = size
            out = np.zeros(max(size, 0), np.float32)
            if size > 0:
                _lib.call("fcwt_morlet_mother", _lib.context().handle, ctypes.c_float(self.fb), size, _ptr(out))
            self.mother = out
            return None
        if len(args) == 4:
            real, imag, size, scale = args
            w = self.getSupport(scale)
            for a in (real, imag):
                if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                    raise TypeError("real/imag must be contiguous float32 arrays")
                if a.size < 2 * w + 1:
                    raise ValueError("real/imag must hold 2*getSupport(scale)+1 values")
            self.width = w
            _lib.call("fcwt_morlet_time", ctypes.c_float(self.fb), ctypes.c_float(scale), _as_int("size", size),
                      _ptr(real), _ptr(imag))
            return None
        raise TypeError("generate() takes (size) or (real, imag, size, scale)")

    def getSupport(self, scale) -> int:
        return _lib.load().fcwt_morlet_support(ctypes.c_float(self.fb), ctypes.c_float(scale))

    def getWavelet(self, scale, pwav) -> None:
        """Fill the complex64 array pwav in place (src/fcwt/fcwt.cpp:86-105)."""
        if not (isinstance(pwav, np.ndarray) and pwav.dtype == np.complex64 and pwav.flags.c_contiguous
                and pwav.ndim == 1):
            raise TypeError("pwav must be a contiguous 1-D complex64 array")
        _lib.call("fcwt_morlet_wavelet", ctypes.c_float(self.fb), ctypes.c_float(scale), _ptr(pwav), pwav.size)



class Paul(Wavelet):
    """Paul wavelet of order m (analytic, single-sided, real in frequency).

    The reference defines only Morlet; its test suite names Paul
    (tests/test_fcwt.py:185-211, commented out). In the reference's
    frequency variable x = 2 w (2 pi / N) of table entry w (Morlet's is
    t = fb (x - 2 pi), src/fcwt/fcwt.cpp:51-67) this table is

        mother[w] = A * y^m * exp(m (1 - y)),   y = x / (2 pi) = 2 w / N,

    a Paul spectrum x^m e^{-x} stretched so its peak sits at x = 2 pi like the
    Morlet's, so that Scales maps scale s to frequency fs / s for it too; A is
    the Morlet table's peak value. The transform runs through the
    caller-supplied-wavelet path (fcwt_cwt_mother)."""

    def __init__(self, order: int = 4):
        super().__init__()
        self.m = int(order)
        if self.m < 1:
            raise ValueError("order must be >= 1")
        self.four_wavelen = 1.0

    def generate(self, *args):
        if len(args) != 1:
            raise NotImplementedError("Paul provides the frequency-domain table generate(size) only")
        size = _as_int("size", args[0])
        w = np.arange(max(size, 0), dtype=np.float64)
        y = 2.0 * w / max(size, 1)
        amp = np.sqrt(2.0 * np.pi) * 0.75112554446
        with np.errstate(under="ignore"):
            t = amp * np.exp(self.m * np.log(np.maximum(y, 1e-300)) + self.m * (1.0 - y))
        t[y == 0] = 0.0
        self.width = size
        self.mother = t.astype(np.float32)
        return None

class DOG(Wavelet):
    """Derivative-of-Gaussian wavelet of order m (real in time, so its
    spectrum is two-sided: doublesided; odd orders are imaginary in
    frequency: imag_frequency). The reference names DOG(order) in its test
    suite and main.cpp (tests/test_fcwt.py:156-182, src/main.cpp:68, both
    commented out) but defines no class; this one follows the published
    spectrum psi^(w) = -i^m / sqrt(Gamma(m + 1/2)) w^m exp(-w^2/2) (Torrence &
    Compo 1998), stretched like Paul so the peak of |psi^| sits where the
    Morlet's does (table entry w = N/2, so Scales maps scale s to fs / s):

        mother[w] = A * s_m * y^m * exp(m (1 - y^2) / 2),   y = 2 w / N,

    A the Morlet table's peak value and s_m the sign of -i^m once the factor
    i of odd orders is left to imag_frequency (s_m = -1, 1, 1, -1 for
    m = 1, 2, 3, 4, period 4). The transform runs through the caller-wavelet
    path with FCWT_DOUBLESIDED (and FCWT_IMAG_FREQUENCY for odd m), the
    reference's own semantics for those flags (src/fcwt/fcwt.cpp:232-273)."""

    def __init__(self, order: int = 2):
        super().__init__()
        self.m = int(order)
        if self.m < 1:
            raise ValueError("order must be >= 1")
        self.four_wavelen = 1.0
        self.imag_frequency = self.m % 2 == 1
        self.doublesided = True

    def generate(self, *args):
        if len(args) != 1:
            raise NotImplementedError("DOG provides the frequency-domain table generate(size) only")
        size = _as_int("size", args[0])
        w = np.arange(max(size, 0), dtype=np.float64)
        y = 2.0 * w / max(size, 1)
        amp = np.sqrt(2.0 * np.pi) * 0.75112554446
        sign = -1.0 if (self.m % 4) in (0, 1) else 1.0
        with np.errstate(under="ignore"):
            t = sign * amp * np.exp(self.m * np.log(np.maximum(y, 1e-300)) + 0.5 * self.m * (1.0 - y * y))
        t[y == 0] = 0.0
        self.width = size
        self.mother = t.astype(np.float32)
        return None


class Scales:
    """Scales(wavelet, scaletype, fs, f0, f1, fn) (src/fcwt/fcwt.cpp:111-190).
    strict=True (or FCWT_STRICT=1) raises ValueError for f1 > fs/2."""

    def __init__(self, pwav, st, fs, f0, f1, fn, strict=None):
        fs = _as_int("fs", fs)
        fn = _as_int("fn", fn)
        _positive("f0", f0)
        _positive("f1", f1)
        _positive("fn", fn)
        st = _as_int("st", st)
        self.fs = fs
        self.fourwavl = float(getattr(pwav, "four_wavelen", np.float32(0.9876)))
        self.nscales = fn
        self.scales = np.zeros(fn, np.float32)
        flags = FCWT_STRICT if _strict(strict) else 0
        rc = _lib.load().fcwt_scales_checked(st, fs, ctypes.c_float(f0), ctypes.c_float(f1), fn, flags,
                                             _ptr(self.scales))
        if rc == _lib.FCWT_ERR_INVALID:
            raise ValueError(_lib.load().fcwt_last_error().decode())
        _lib.check(rc)

    def getScales(self, pfreqs) -> None:
        pfreqs = _inplace_f32(pfreqs)
        n = min(pfreqs.size, self.scales.size)
        pfreqs[:n] = self.scales[:n]

    def getFrequencies(self, pfreqs) -> None:
        pfreqs = _inplace_f32(pfreqs)
        n = pfreqs.size
        if n > self.scales.size:
            raise ValueError("array longer than the number of scales")
        _lib.call("fcwt_frequencies", _ptr(self.scales), n, self.fs, _ptr(pfreqs))


def _inplace_f32(a) -> np.ndarray:
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous and a.ndim == 1):
        raise TypeError("Array of type 'float' required (contiguous, 1-D)")
    return a


def _scales_array(scales) -> np.ndarray:
    if isinstance(scales, Scales):
        return scales.scales
    return np.ascontiguousarray(scales, np.float32)


class FCWT:
    """FCWT(wavelet, threads, use_optimalization_schemes, use_normalization)
    (src/fcwt/fcwt.h:114-152). ``threads`` keeps its reference meaning for
    the result: it sets the per-scale truncation length (fcwt.cpp:213-214)."""

    def __init__(self, pwav, pthreads, puse_optimalization_schemes, puse_normalization, device: int = 0,
                 strict=None, compat_align_shift: bool = False):
        self.wavelet = pwav
        self.threads = _as_int("pthreads", pthreads)
        self.use_optimalization_schemes = bool(puse_optimalization_schemes)
        self.use_normalization = bool(puse_normalization)
        self.device = device
        # compat_align_shift: reproduce the reference's odd-n row shift (src/fcwt/fcwt.cpp:418-426)
        self.flags = (FCWT_NORM if self.use_normalization else 0) | (FCWT_STRICT if _strict(strict) else 0) | \
            (_lib.FCWT_COMPAT_ALIGN if compat_align_shift else 0)

    # -- tuning files (src/fcwt/fcwt.cpp:313-393)
    def create_FFT_optimization_plan(self, pmaxsize, poptimizationflags) -> None:
        if isinstance(poptimizationflags, str):
            if poptimizationflags not in _FFTW_FLAGS:
                print(f"Unknown flag: {poptimizationflags}", file=sys.stderr)
                return
            level = _FFTW_FLAGS[poptimizationflags]
        else:
            f = _as_int("poptimizationflags", poptimizationflags)
            # FFTW flag bits: ESTIMATE 1<<6, EXHAUSTIVE 1<<3, PATIENT 1<<5, MEASURE 0
            level = 0 if f & (1 << 6) else 3 if f & (1 << 3) else 2 if f & (1 << 5) else 1
        pmaxsize = _as_int("pmaxsize", pmaxsize)
        if _lib.load().fcwt_find2power(pmaxsize) <= 10:
            print("Maxsize is too small (<=1024)... please use a larger number", file=sys.stderr)
        _lib.call("fcwt_create_optimization_plan", _lib.context(self.device).handle, pmaxsize, self.threads,
                  level, None)

    def _load_plan(self, n: int) -> None:
        if not self.use_optimalization_schemes:
            return
        N = 1 << _lib.load().fcwt_find2power(n)
        if N <= 1024:
            print("Inputsize is too small (N <= 1024) to use optimization.")
            return
        rc = _lib.load().fcwt_load_optimization_plan(_lib.context(self.device).handle, n, self.threads, None)
        if rc != 0:
            print(f"WARNING: Optimization scheme 'n{N}_t{self.threads}.wis' was not found, "
                  "fallback to calculation without optimization.")

    def cwt(self, pinput, scales, poutput, out_type: int = FCWT_OUT_C64) -> None:
        """FCWT::cwt(input, n, scales, output, n1, n2) (fcwt.cpp:540-543):
        real input; output [fn, n] complex64 written in place."""
        self._run(pinput, scales, poutput, False, out_type)

    def ccwt(self, pcinput, scales, poutput, out_type: int = FCWT_OUT_C64) -> None:
        """FCWT::cwt(complex input, ...) (fcwt.cpp:545-548)."""
        self._run(pcinput, scales, poutput, True, out_type)

    def _run_table(self, x, sc, out, complex_input: bool, out_type: int) -> None:
        """Any other Wavelet subclass: the transform runs on its mother table."""
        ctx = _lib.context(self.device)
        if _is_torch(x) or _is_torch(out):
            import torch

            n = x.numel()
            table = _table_of(self.wavelet, n)
            ctx.set_stream(torch.cuda.current_stream(out.device).cuda_stream)
            try:
                _lib.call("fcwt_cwt_mother", ctx.handle, ctypes.c_void_p(x.data_ptr()), n, 1 if complex_input else 0,
                          _ptr(table), table.size, _ptr(sc), sc.size, self.threads,
                          self.flags | _kind_flags(self.wavelet), ctypes.c_void_p(out.data_ptr()), out_type)
            finally:
                ctx.set_stream(None)
            return
        xin = _host_input(x, complex_input)
        n = xin.size
        table = _table_of(self.wavelet, n)
        _check_host_output(out, sc.size, n, out_type)
        _lib.call("fcwt_cwt_mother", ctx.handle, _ptr(xin), n, 1 if complex_input else 0, _ptr(table), table.size,
                  _ptr(sc), sc.size, self.threads, self.flags | _kind_flags(self.wavelet), _ptr(out), out_type)

    def _run(self, x, scales, out, complex_input: bool, out_type: int) -> None:
        sc = _scales_array(scales)
        if not isinstance(self.wavelet, Morlet):
            self._run_table(x, sc, out, complex_input, out_type)
            return
        fb = self.wavelet.fb
        ctx = _lib.context(self.device)
        fname = "fcwt_ccwt" if complex_input else "fcwt_cwt"
        if _is_torch(x) or _is_torch(out):
            _run_torch(ctx, fname, x, sc, out, complex_input, fb, self.threads, self.flags, out_type)
            return
        xin = _host_input(x, complex_input)
        n = xin.size
        self._load_plan(n)
        _check_host_output(out, sc.size, n, out_type)
        _lib.call(fname, ctx.handle, _ptr(xin), n, ctypes.c_float(fb), _ptr(sc), sc.size, self.threads,
                  self.flags, _ptr(out), out_type)


def _kind_flags(wavelet) -> int:
    """FCWT_IMAG_FREQUENCY / FCWT_DOUBLESIDED from the wavelet's fields (the
    reference passes them to its product, src/fcwt/fcwt.cpp:396-429)."""
    f = 0
    if getattr(wavelet, "imag_frequency", False):
        f |= _lib.FCWT_IMAG_FREQUENCY
    if getattr(wavelet, "doublesided", False):
        f |= _lib.FCWT_DOUBLESIDED
    return f


def _table_of(wavelet, n: int) -> np.ndarray:
    """The frequency-domain table wavelet.generate(N) fills, N = 2^find2power(n)
    (the reference reads wavelet->mother after generate, fcwt.cpp:504-505)."""
    N = 1 << _lib.load().fcwt_find2power(int(n))
    wavelet.generate(N)
    t = getattr(wavelet, "mother", None)
    if t is None or np.asarray(t).size != N:
        raise ValueError(f"generate({N}) must leave a {N}-entry table in .mother")
    return np.ascontiguousarray(t, np.float32)


def _host_input(x, complex_input: bool) -> np.ndarray:
    x = np.asarray(x)
    if x.ndim != 1:
        raise ValueError("Array must be 1-dimensional")
    if complex_input:
        if not np.iscomplexobj(x) and x.dtype.kind not in "fiu":
            raise TypeError("Array of type 'complex float' required")
        return np.ascontiguousarray(x, np.complex64)
    if np.iscomplexobj(x):
        raise TypeError("Array of type 'float' required")
    return np.ascontiguousarray(x, np.float32)


_OUT_DTYPES = {FCWT_OUT_C64: (np.complex64,), FCWT_OUT_BF16: (np.uint32, np.float32), FCWT_OUT_F16: (np.uint32, np.float32)}


def _check_host_output(out, fn: int, n: int, out_type: int) -> None:
    if not isinstance(out, np.ndarray):
        raise TypeError("output must be a numpy array or a torch CUDA tensor")
    if not out.flags.c_contiguous:
        raise TypeError("Array must be contiguous.")
    if out_type == FCWT_OUT_C64:
        if out.dtype != np.complex64:
            raise TypeError("Array of type 'complex float' required")
        if out.size != fn * n:
            raise ValueError(f"output must hold nscales*n = {fn}*{n} values")
    else:
        if out.nbytes != fn * n * 4:
            raise ValueError(f"output must hold nscales*n*4 bytes for a 16-bit complex type")


def _run_torch(ctx, fname, x, sc, out, complex_input, fb, threads, flags, out_type) -> None:
    import torch

    if not (isinstance(x, torch.Tensor) and isinstance(out, torch.Tensor)):
        raise TypeError("pass both input and output as torch tensors for the device path")
    if not (x.is_cuda and out.is_cuda):
        raise TypeError("torch tensors must live on a CUDA device")
    if x.dim() != 1:
        raise ValueError("Array must be 1-dimensional")
    want = torch.complex64 if complex_input else torch.float32
    if x.dtype != want:
        raise TypeError(f"input must be {want}")
    if not x.is_contiguous() or not out.is_contiguous():
        raise TypeError("tensors must be contiguous")
    n = x.numel()
    esz = 8 if out_type == FCWT_OUT_C64 else 4
    if out.numel() * out.element_size() != sc.size * n * esz:
        raise ValueError("output has the wrong size")
    if out.device.index != ctx.device:
        ctx = _lib.context(out.device.index)
    ctx.set_stream(torch.cuda.current_stream(out.device).cuda_stream)
    try:
        _lib.call(fname, ctx.handle, ctypes.c_void_p(x.data_ptr()), n, ctypes.c_float(fb), _ptr(sc), sc.size,
                  threads, flags, ctypes.c_void_p(out.data_ptr()), out_type)
    finally:
        ctx.set_stream(None)


class Plan:
    """A reusable device plan (fcwt_plan_create): all shape-, scale- and
    flag-dependent work done once; ``execute`` runs one transform.

    rows=(begin, end) selects a shard of the scale rows (multi-GPU sharding);
    the reference's stale-bin semantics still follow all rows.
    row_stride / time_stride: fused decimation (fcwt_plan_create_strided):
    every row_stride-th row of the shard and every time_stride-th sample
    (a power of two), output [ceil(rows / row_stride), ceil(n / time_stride)]."""

    def __init__(self, n: int, scales, fb: float = 2.0, threads: int = 1, norm: bool = True,
                 complex_input: bool = False, rows: tuple[int, int] | None = None, device: int = 0,
                 exact_support: bool = False, scalar_trunc: bool = False, row_stride: int = 1,
                 time_stride: int = 1, compat_align_shift: bool = False):
        self.ctx = _lib.context(device)
        self.device = device
        self.scales = _scales_array(scales).copy()
        self.n = int(n)
        self.fn = self.scales.size
        self.rows = rows if rows is not None else (0, self.fn)
        self.complex_input = complex_input
        flags = (FCWT_NORM if norm else 0) | (FCWT_EXACT_SUPPORT if exact_support else 0) | \
            (FCWT_SCALAR_TRUNC if scalar_trunc else 0) | (_lib.FCWT_COMPAT_ALIGN if compat_align_shift else 0)
        h = ctypes.c_void_p()
        if row_stride == 1 and time_stride == 1:
            _lib.call("fcwt_plan_create", self.ctx.handle, self.n, 1 if complex_input else 0, ctypes.c_float(fb),
                      _ptr(self.scales), self.fn, int(threads), flags, int(self.rows[0]), int(self.rows[1]),
                      ctypes.byref(h))
        else:
            _lib.call("fcwt_plan_create_strided", self.ctx.handle, self.n, 1 if complex_input else 0,
                      ctypes.c_float(fb), _ptr(self.scales), self.fn, int(threads), flags, int(self.rows[0]),
                      int(self.rows[1]), int(row_stride), int(time_stride), ctypes.byref(h))
        self.handle = h
        r, c = ctypes.c_int(), ctypes.c_int()
        _lib.call("fcwt_plan_output_shape", self.handle, ctypes.byref(r), ctypes.byref(c))
        self.out_shape = (r.value, c.value)

    @property
    def n_rows(self) -> int:
        return self.out_shape[0]

    def execute(self, x, out, out_type: int = FCWT_OUT_C64, stream=None) -> None:
        """x, out: numpy arrays (host; synchronous) or torch CUDA tensors (enqueued
        on `stream` or torch's current stream)."""
        if _is_torch(x) or _is_torch(out):
            import torch

            st = stream if stream is not None else torch.cuda.current_stream(self.device)
            self.ctx.set_stream(st.cuda_stream)
            try:
                _lib.call("fcwt_plan_execute", self.handle, ctypes.c_void_p(x.data_ptr()),
                          ctypes.c_void_p(out.data_ptr()), out_type)
            finally:
                self.ctx.set_stream(None)
            return
        xin = _host_input(x, self.complex_input)
        if xin.size != self.n:
            raise ValueError("input length differs from the plan")
        _check_host_output(out, self.out_shape[0], self.out_shape[1], out_type)
        _lib.call("fcwt_plan_execute", self.handle, _ptr(xin), _ptr(out), out_type)

    def stats(self) -> dict:
        """Rows of the plan and how many run on the tensor-core engine."""
        r, t = ctypes.c_int(), ctypes.c_int()
        _lib.call("fcwt_plan_stats", self.handle, ctypes.byref(r), ctypes.byref(t))
        return {"rows": r.value, "tensor_core_rows": t.value}

    def execute_ptr(self, x_ptr: int, out_ptr: int, out_type: int = FCWT_OUT_C64, stream_ptr: int | None = None) -> None:
        """Raw-pointer form (device or host pointers); stream_ptr None = the
        context's own stream, 0 = legacy default stream."""
        self.ctx.set_stream(stream_ptr)
        try:
            _lib.call("fcwt_plan_execute", self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(out_ptr), out_type)
        finally:
            self.ctx.set_stream(None)

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().fcwt_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """Many signals (different lengths and scale grids, one Morlet(fb)) in one
    plan: one forward-FFT launch sequence per padded length and a single
    persistent row-engine launch for all rows of all signals
    (fcwt_plan_create_batched). ``execute(..., graph=True)`` replays the whole
    sequence from a CUDA graph (device tensors only)."""

    def __init__(self, ns, scales_list, fb: float = 2.0, threads: int = 1, norm: bool = True,
                 complex_input: bool = False, device: int = 0, exact_support: bool = False,
                 continuous: bool = False):
        self.ctx = _lib.context(device)
        self.device = device
        self.ns = [int(v) for v in ns]
        self.scales = [_scales_array(sc).copy() for sc in scales_list]
        if len(self.ns) != len(self.scales):
            raise ValueError("one scale grid per signal")
        self.fns = [sc.size for sc in self.scales]
        self.complex_input = complex_input
        nsig = len(self.ns)
        flags = (FCWT_NORM if norm else 0) | (FCWT_EXACT_SUPPORT if exact_support else 0) | \
            (_lib.FCWT_CONTINUOUS if continuous else 0)
        ns_arr = (ctypes.c_int * nsig)(*self.ns)
        fns_arr = (ctypes.c_int * nsig)(*self.fns)
        sc_arr = (ctypes.c_void_p * nsig)(*[sc.ctypes.data for sc in self.scales])
        h = ctypes.c_void_p()
        _lib.call("fcwt_plan_create_batched", self.ctx.handle, nsig, ns_arr, 1 if complex_input else 0,
                  ctypes.c_float(fb), sc_arr, fns_arr, int(threads), flags, ctypes.byref(h))
        self.handle = h

    def stats(self) -> dict:
        """Rows of the plan and how many run on the tensor-core engine."""
        r, t = ctypes.c_int(), ctypes.c_int()
        _lib.call("fcwt_plan_stats", self.handle, ctypes.byref(r), ctypes.byref(t))
        return {"rows": r.value, "tensor_core_rows": t.value}

    def outputs_like(self, device=None, out_dtype=None):
        """Allocate torch outputs [fn_s, n_s] (complex64) for every signal."""
        import torch

        dev = device if device is not None else f"cuda:{self.device}"
        return [torch.empty((fn, n), dtype=torch.complex64, device=dev) for fn, n in zip(self.fns, self.ns)]

    def execute(self, inputs, outputs, out_type: int = FCWT_OUT_C64, graph: bool = False, stream=None) -> None:
        nsig = len(self.ns)
        if len(inputs) != nsig or len(outputs) != nsig:
            raise ValueError("one input and one output per signal")
        torch_mode = any(_is_torch(v) for v in list(inputs) + list(outputs))
        keep = []
        ins, outs = [], []
        for s in range(nsig):
            x, o = inputs[s], outputs[s]
            if _is_torch(x):
                ins.append(x.data_ptr())
            else:
                xx = _host_input(x, self.complex_input)
                keep.append(xx)
                ins.append(xx.ctypes.data)
            outs.append(o.data_ptr() if _is_torch(o) else o.ctypes.data)
        in_arr = (ctypes.c_void_p * nsig)(*ins)
        out_arr = (ctypes.c_void_p * nsig)(*outs)
        fname = "fcwt_plan_execute_graph" if graph else "fcwt_plan_execute_batched"
        if torch_mode:
            import torch

            st = stream if stream is not None else torch.cuda.current_stream(self.device)
            self.ctx.set_stream(st.cuda_stream)
            try:
                _lib.call(fname, self.handle, in_arr, out_arr, out_type)
            finally:
                self.ctx.set_stream(None)
        else:
            _lib.call(fname, self.handle, in_arr, out_arr, out_type)

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().fcwt_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synchronize(device: int = 0) -> None:
    """Wait for the device work of this process's context and raise on device errors."""
    _lib.context(device).synchronize()


def row_truncation(n: int, scales, threads: int = 1, exact_support: bool = False, scalar_trunc: bool = False,
                   fb: float = 2.0):
    """Per-row truncation length of the reference (bit-exact) and the bin window
    [lo, hi) the device engine evaluates for Morlet(fb). Host only."""
    sc = _scales_array(scales)
    proc = np.zeros(sc.size, np.int32)
    lo = np.zeros(sc.size, np.int32)
    hi = np.zeros(sc.size, np.int32)
    flags = (FCWT_EXACT_SUPPORT if exact_support else 0) | (FCWT_SCALAR_TRUNC if scalar_trunc else 0)
    _lib.call("fcwt_row_truncation", int(n), ctypes.c_float(fb), _ptr(sc), sc.size, int(threads), flags, _ptr(proc),
              _ptr(lo), _ptr(hi))
    return proc, lo, hi


def mother_host(fb: float, N: int) -> np.ndarray:
    """Morlet::generate(int) evaluated by the library's host code (no GPU)."""
    out = np.zeros(N, np.float32)
    _lib.call("fcwt_morlet_mother_host", ctypes.c_float(fb), int(N), _ptr(out))
    return out


# ---------------------------------------------------------------- boilerplate

def cwt(input, fs, f0, f1, fn, nthreads=1, scaling="lin", fast=False, norm=True):
    """fcwt.cwt (src/fcwt/boilerplate.py:5-33): Morlet(2.0), LINFREQS for
    scaling="lin" else LOGSCALES; returns (freqs float32[fn], out complex64[fn, n])."""
    if _is_torch(input):
        return cwt_device(input, fs, f0, f1, fn, nthreads=nthreads, scaling=scaling, norm=norm)
    input = np.asarray(input)
    if input.ndim > 1:
        raise ValueError("Input must be a vector")
    if input.dtype != np.float32:
        input = input.astype(np.float32)
    morl = Morlet(2.0)
    if scaling == "lin":
        scales = Scales(morl, FCWT_LINFREQS, fs, f0, f1, fn)
    else:
        scales = Scales(morl, FCWT_LOGSCALES, fs, f0, f1, fn)
    fcwt = FCWT(morl, nthreads, fast, norm)
    output = np.zeros((fn, input.size), dtype=np.complex64)
    freqs = np.zeros((fn), dtype=np.float32)
    fcwt.cwt(input, scales, output)
    scales.getFrequencies(freqs)
    return freqs, output


def cwt_device(input, fs, f0, f1, fn, nthreads=1, scaling="lin", norm=True, out_dtype=None, fb: float = 2.0):
    """Device-resident form of fcwt.cwt for a torch CUDA tensor: returns
    (freqs numpy float32[fn], out torch tensor [fn, n]) without host copies.
    out_dtype: torch.complex64 (default) or torch.bfloat16 / torch.float16 for
    interleaved 16-bit (re, im) pairs, shape [fn, n, 2]."""
    import torch

    x = input
    if x.dim() != 1:
        raise ValueError("Input must be a vector")
    if x.dtype != torch.float32:
        x = x.float()
    x = x.contiguous()
    morl = Morlet(fb)
    st = FCWT_LINFREQS if scaling == "lin" else FCWT_LOGSCALES
    scales = Scales(morl, st, fs, f0, f1, fn)
    n = x.numel()
    if out_dtype is None or out_dtype == torch.complex64:
        out = torch.empty((fn, n), dtype=torch.complex64, device=x.device)
        ot = FCWT_OUT_C64
    elif out_dtype in (torch.bfloat16, torch.float16):
        out = torch.empty((fn, n, 2), dtype=out_dtype, device=x.device)
        ot = FCWT_OUT_BF16 if out_dtype == torch.bfloat16 else FCWT_OUT_F16
    else:
        raise TypeError("out_dtype must be complex64, bfloat16 or float16")
    FCWT(morl, nthreads, False, norm, device=x.device.index or 0).cwt(x, scales, out, out_type=ot)
    freqs = np.zeros(fn, np.float32)
    scales.getFrequencies(freqs)
    return freqs, out
