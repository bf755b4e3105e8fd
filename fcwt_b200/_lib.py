"""ctypes binding of libfcwt_b200.so (the C ABI declared in include/fcwt_b200.h).

The library is the product: it must exist (``python -m fcwt_b200.build``) and
load; there is no Python or CPU fallback for the transform.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfcwt_b200.so")

FCWT_OK = 0
FCWT_ERR_INVALID = 1
FCWT_ERR_CUDA = 2
FCWT_ERR_NOMEM = 3
FCWT_ERR_UNSUPPORTED = 4
FCWT_ERR_DEVICE = 5
FCWT_ERR_IO = 6

FCWT_NORM = 1 << 0
FCWT_SCALAR_TRUNC = 1 << 1
FCWT_EXACT_SUPPORT = 1 << 2
FCWT_CONTINUOUS = 1 << 3
FCWT_STRICT = 1 << 4
FCWT_IMAG_FREQUENCY = 1 << 5
FCWT_DOUBLESIDED = 1 << 6
FCWT_COMPAT_ALIGN = 1 << 7

FCWT_OUT_C64 = 0
FCWT_OUT_BF16 = 1
FCWT_OUT_F16 = 2
FCWT_OUT_POWER = 3
FCWT_OUT_DB = 4

FCWT_ENGINE_AUTO = 0
FCWT_ENGINE_CUDA_CORES = 1
FCWT_ENGINE_TENSOR_CORES = 2

# Every symbol include/fcwt_b200.h declares: name -> (restype, argtypes)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_u = ctypes.c_uint
_f = ctypes.c_float
SIGNATURES = {
    "fcwt_version": (_i, []),
    "fcwt_last_error": (ctypes.c_char_p, []),
    "fcwt_context_create": (_i, [_i, ctypes.POINTER(_vp)]),
    "fcwt_context_destroy": (_i, [_vp]),
    "fcwt_context_set_stream": (_i, [_vp, _vp]),
    "fcwt_synchronize": (_i, [_vp]),
    "fcwt_context_set_engine": (_i, [_vp, _i]),
    "fcwt_profile_enable": (_i, [_vp, _i]),
    "fcwt_profile_read": (_i, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "fcwt_find2power": (_i, [_i]),
    "fcwt_scales": (_i, [_i, _i, _f, _f, _i, _vp]),
    "fcwt_scales_checked": (_i, [_i, _i, _f, _f, _i, _u, _vp]),
    "fcwt_frequencies": (_i, [_vp, _i, _i, _vp]),
    "fcwt_morlet_support": (_i, [_f, _f]),
    "fcwt_morlet_time": (_i, [_f, _f, _i, _vp, _vp]),
    "fcwt_morlet_wavelet": (_i, [_f, _f, _vp, _i]),
    "fcwt_morlet_mother_host": (_i, [_f, _i, _vp]),
    "fcwt_row_truncation": (_i, [_i, _f, _vp, _i, _i, _u, _vp, _vp, _vp]),
    "fcwt_morlet_mother": (_i, [_vp, _f, _i, _vp]),
    "fcwt_cwt": (_i, [_vp, _vp, _i, _f, _vp, _i, _i, _u, _vp, _i]),
    "fcwt_ccwt": (_i, [_vp, _vp, _i, _f, _vp, _i, _i, _u, _vp, _i]),
    "fcwt_plan_create": (_i, [_vp, _i, _i, _f, _vp, _i, _i, _u, _i, _i, ctypes.POINTER(_vp)]),
    "fcwt_plan_execute": (_i, [_vp, _vp, _vp, _i]),
    "fcwt_plan_create_strided": (_i, [_vp, _i, _i, _f, _vp, _i, _i, _u, _i, _i, _i, _i, ctypes.POINTER(_vp)]),
    "fcwt_plan_output_shape": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "fcwt_plan_destroy": (_i, [_vp]),
    "fcwt_plan_stats": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "fcwt_plan_create_mother": (_i, [_vp, _i, _i, _vp, _i, _vp, _i, _i, _u, _i, _i, ctypes.POINTER(_vp)]),
    "fcwt_cwt_mother": (_i, [_vp, _vp, _i, _i, _vp, _i, _vp, _i, _i, _u, _vp, _i]),
    "fcwt_plan_create_batched": (_i, [_vp, _i, _vp, _i, _f, _vp, _vp, _i, _u, ctypes.POINTER(_vp)]),
    "fcwt_plan_execute_batched": (_i, [_vp, _vp, _vp, _i]),
    "fcwt_plan_execute_graph": (_i, [_vp, _vp, _vp, _i]),
    "fcwt_create_optimization_plan": (_i, [_vp, _i, _i, _i, ctypes.c_char_p]),
    "fcwt_load_optimization_plan": (_i, [_vp, _i, _i, ctypes.c_char_p]),
    "fcwt_morlet_cwt_backward": (_i, [_vp, _vp, _i, _i, _f, _vp, _i, _f, _u, _vp, _vp,
                                      ctypes.POINTER(ctypes.c_double), _vp]),
    "fcwt_cwt_noalloc": (_i, [_vp, _i, _f, _vp, _i, _i, _u, _vp, _vp, ctypes.POINTER(_i)]),
}


class FcwtError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[fcwt status {code}] {message}")
        self.code = code


_lib = None
_lock = threading.RLock()


def load() -> ctypes.CDLL:
    """Load libfcwt_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} not found: build the CUDA library first (python -m fcwt_b200.build)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc: int) -> None:
    if rc != FCWT_OK:
        msg = load().fcwt_last_error()
        raise FcwtError(rc, msg.decode() if msg else "unknown error")


def call(name: str, *args) -> int:
    rc = getattr(load(), name)(*args)
    check(rc)
    return rc


class Context:
    """Owns an fcwt_context (one device, one stream, workspace, plan cache)."""

    def __init__(self, device: int = 0):
        self.device = device
        h = ctypes.c_void_p()
        call("fcwt_context_create", device, ctypes.byref(h))
        self.handle = h

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            load().fcwt_context_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None) -> None:
        """stream_ptr: a cudaStream_t value; 0 is the legacy default stream
        (what torch reports for its default stream); None restores the
        context's own stream."""
        if stream_ptr is None:
            h = 0
        elif stream_ptr == 0:
            h = 1  # cudaStreamLegacy
        else:
            h = stream_ptr
        call("fcwt_context_set_stream", self.handle, ctypes.c_void_p(h))

    def synchronize(self) -> None:
        call("fcwt_synchronize", self.handle)

    def set_engine(self, mode: int) -> None:
        """FCWT_ENGINE_AUTO, FCWT_ENGINE_CUDA_CORES or FCWT_ENGINE_TENSOR_CORES
        for plans built afterwards (drops this context's plan cache)."""
        call("fcwt_context_set_engine", self.handle, int(mode))

    def profile_enable(self, enable: bool = True) -> None:
        call("fcwt_profile_enable", self.handle, 1 if enable else 0)

    def profile_read(self) -> tuple[float, int, int]:
        """(row-engine device ms, row-engine launches, kernels launched) since the last read."""
        ms = ctypes.c_double()
        el = ctypes.c_int()
        kl = ctypes.c_int()
        call("fcwt_profile_read", self.handle, ctypes.byref(ms), ctypes.byref(el), ctypes.byref(kl))
        return ms.value, el.value, kl.value


_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    """Process-wide context of a device (created on first use)."""
    c = _contexts.get(device)
    if c is None:
        with _lock:
            c = _contexts.get(device)
            if c is None:
                c = Context(device)
                _contexts[device] = c
    return c
