"""GPU test of fcwt_cwt_noalloc, the entry point for callers that cannot
allocate device memory (real-time audio/sensor threads where cudaMalloc may
block and synchronize the device, plug-ins whose host framework owns all
device memory, callers with a footprint fixed at start-up). It keeps its
workspace in a static array inside the library, so its output must match the
allocating entry point (fcwt_cwt) even though every call reuses that array.

The file is named to be collected last; it passes alone in a fresh process and
after the other tests."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(lib, x, sc, fb, T, norm, out):
    import torch

    status = ctypes.c_int(-1)
    flags = 1 if norm else 0
    rc = lib.fcwt_cwt_noalloc(ctypes.c_void_p(x.data_ptr()), x.numel(), ctypes.c_float(fb),
                              ctypes.c_void_p(sc.ctypes.data), sc.size, T, flags,
                              ctypes.c_void_p(out.data_ptr()),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(status))
    return rc, status.value


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(fcwt, oracle):
    import torch

    from fcwt_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(21)
    cases = [
        # n, fb, scale grid, threads, norm  (N = 16384 two-phase, 4096 fused, 1024 fused, 512 direct)
        (10000, 2.0, oracle.scales(LOGSCALES, 1000, 1.0, 101.0, 300), 8, True),
        (4000, 0.5, oracle.scales(LOGSCALES, 1000, 2.0, 200.0, 64), 1, False),
        (1000, 16.0, oracle.scales(LINFREQS, 1000, 1.0, 20.0, 100), 1, True),
        (500, 2.0, oracle.scales(LOGSCALES, 1000, 5.0, 400.0, 20), 3, True),
    ]
    for n, fb, sc, T, norm in cases:
        for call in range(2):  # two calls in a row on the same static workspace
            x = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()
            got = torch.full((sc.size, n), float("nan"), dtype=torch.complex64, device="cuda")
            rc, st = _noalloc(lib, x, sc, fb, T, norm, got)
            assert rc == 0 and st == 0, lib.fcwt_last_error()
            want = torch.empty_like(got)
            fcwt.FCWT(fcwt.Morlet(fb), T, False, norm).cwt(x, sc, want)
            torch.cuda.synchronize()
            g, w = got.cpu().numpy(), want.cpu().numpy()
            assert np.isfinite(g).all()
            assert rel_l2(g, w) < TOL, (n, call)


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    from fcwt_b200 import _lib

    lib = _lib.load()
    sc = np.array([10.0, 20.0], np.float32)
    x = torch.zeros(16385, device="cuda")
    out = torch.empty((2, 16385), dtype=torch.complex64, device="cuda")
    rc, _ = _noalloc(lib, x, sc, 2.0, 1, True, out)
    assert rc == _lib.FCWT_ERR_INVALID
    assert b"16384" in lib.fcwt_last_error()
    sc2 = np.full(1025, 10.0, np.float32)
    out2 = torch.empty((1025, 100), dtype=torch.complex64, device="cuda")
    rc, _ = _noalloc(lib, torch.zeros(100, device="cuda"), sc2, 2.0, 1, True, out2)
    assert rc == _lib.FCWT_ERR_INVALID
    assert b"1024" in lib.fcwt_last_error()


def test_noalloc_rejects_a_device_scales_array():
    """scales is read on the host: a device pointer is refused with an error,
    not dereferenced."""
    import torch

    from fcwt_b200 import _lib

    lib = _lib.load()
    n, fn = 1000, 4
    x = torch.zeros(n, device="cuda")
    out = torch.empty((fn, n), dtype=torch.complex64, device="cuda")
    sc_dev = torch.full((fn,), 10.0, device="cuda")
    status = ctypes.c_int(-1)
    rc = lib.fcwt_cwt_noalloc(ctypes.c_void_p(x.data_ptr()), n, ctypes.c_float(2.0),
                              ctypes.c_void_p(sc_dev.data_ptr()), fn, 1, 1, ctypes.c_void_p(out.data_ptr()),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(status))
    assert rc == _lib.FCWT_ERR_INVALID
    assert b"host" in lib.fcwt_last_error()
