"""CPU tests of the product's host side: the C-ABI library loads and exports
every symbol include/fcwt_b200.h declares, the host arithmetic is bit-exact
with the reference golden vectors, argument errors behave like the reference
binding, and the planner's bin windows drop only negligible weights. No GPU
compute is called here."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    text = open(os.path.join(ROOT, "include", "fcwt_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fcwt_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from fcwt_b200 import _lib

    names = _header_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding binds exactly the declared set
    assert set(_lib.SIGNATURES) == set(names)


def test_cpp_api_symbols_exported():
    """The C++ drop-in classes of include/fcwt.h are compiled into the library."""
    from fcwt_b200 import _lib

    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    for sym in ["_ZN6MorletC1Ef", "_ZN6ScalesC1EP7Wavelet9SCALETYPEiffi", "_ZN4FCWTC1EP7Waveletibb",
                "_ZN4FCWT3cwtEPfiPSt7complexIfEP6Scales", "_ZN6Scales14getFrequenciesEPfi"]:
        assert sym in out, sym


def test_scales_bit_exact(golden, fcwt):
    for k, (st, fs, f0, f1, fn) in enumerate(golden["scale_cases"]):
        s = fcwt.Scales(fcwt.Morlet(2.0), int(st), int(fs), float(f0), float(f1), int(fn))
        assert np.array_equal(s.scales.view(np.uint32), golden[f"scales_{k}"].view(np.uint32)), k
        fr = np.zeros(int(fn), np.float32)
        s.getFrequencies(fr)
        assert np.array_equal(fr.view(np.uint32), golden[f"freqs_{k}"].view(np.uint32)), k
        sc = np.zeros(int(fn), np.float32)
        s.getScales(sc)
        assert np.array_equal(sc, s.scales)


def test_host_mother_bit_exact(golden, fcwt):
    for k, (fb, N) in enumerate(golden["mother_cases"]):
        m = fcwt.mother_host(float(fb), int(N))
        assert np.array_equal(m.view(np.uint32), golden[f"mother_{k}"].view(np.uint32)), k


def test_truncation_bit_exact(golden, fcwt):
    for k, (n, si, T) in enumerate(golden["trunc_cases"]):
        proc, lo, hi = fcwt.row_truncation(int(n), golden[f"scales_{si}"], int(T))
        assert np.array_equal(proc, golden[f"proc_{k}"]), k
        N = fcwt.api._lib.load().fcwt_find2power(int(n))
        assert np.all(lo >= 0) and np.all(hi <= max((1 << N) // 2, 1)) and np.all(lo <= hi)


def test_wavelet_and_support(golden, fcwt):
    for k, (fb, scale) in enumerate(golden["wavelet_cases"]):
        m = fcwt.Morlet(float(fb))
        g = golden[f"wavelet_{k}"]
        assert m.getSupport(float(scale)) * 2 + 1 == g.size
        w = np.zeros(g.size, np.complex64)
        m.getWavelet(float(scale), w)
        assert np.array_equal(w.view(np.uint32), g.view(np.uint32)), k
        re_, im_ = np.zeros(g.size, np.float32), np.zeros(g.size, np.float32)
        m.generate(re_, im_, g.size, float(scale))
        assert np.array_equal(re_, g.real) and np.array_equal(im_, g.imag)


def test_binding_argument_errors(fcwt):
    m = fcwt.Morlet(2.0)
    with pytest.raises(ValueError):
        fcwt.Scales(m, fcwt.FCWT_LINFREQS, 1000, 0.0, 10.0, 10)
    with pytest.raises(ValueError):
        fcwt.Scales(m, fcwt.FCWT_LINFREQS, 1000, 1.0, -1.0, 10)
    with pytest.raises(ValueError):
        fcwt.Scales(m, fcwt.FCWT_LINFREQS, 1000, 1.0, 10.0, 0)
    with pytest.raises(TypeError):
        fcwt.Scales(m, fcwt.FCWT_LINFREQS, 1000.5, 1.0, 10.0, 10)
    with pytest.raises(fcwt.FcwtError):
        fcwt.row_truncation(100, np.ones(3, np.float32), threads=0)
    with pytest.raises(fcwt.FcwtError):
        fcwt.row_truncation(100, np.array([1.0, -2.0], np.float32), threads=1)
    with pytest.raises(ValueError):
        fcwt.cwt(np.zeros((2, 2), np.float32), 1000, 1, 10, 5)


def test_c_abi_rejects_bad_arguments():
    from fcwt_b200 import _lib

    lib = _lib.load()
    out = np.zeros(4, np.float32)
    assert lib.fcwt_scales(7, 1000, ctypes.c_float(1.0), ctypes.c_float(2.0), 4,
                           ctypes.c_void_p(out.ctypes.data)) == _lib.FCWT_ERR_INVALID
    assert b"scale type" in lib.fcwt_last_error()
    assert lib.fcwt_frequencies(None, 4, 1000, None) == _lib.FCWT_ERR_INVALID
    assert lib.fcwt_find2power(100000) == 17
    assert lib.fcwt_find2power(0) == 0 and lib.fcwt_find2power(1) == 0
    assert lib.fcwt_plan_execute(None, None, None, 0) == _lib.FCWT_ERR_INVALID
    assert lib.fcwt_synchronize(None) == _lib.FCWT_ERR_INVALID


def test_context_creation_fails_cleanly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from fcwt_b200 import _lib

    h = ctypes.c_void_p()
    rc = _lib.load().fcwt_context_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value


@pytest.mark.parametrize("fb,case", [(2.0, 0), (0.5, 0), (6.0, 4), (2.0, 1)])
def test_bin_window_drops_only_negligible_weights(oracle, fcwt, golden, fb, case):
    """Bins outside the planner's [lo, hi) window carry weight below 2^-36 of
    the mother peak (the trimming bound), for own and stale bins alike."""
    st, fs, f0, f1, fn = golden["scale_cases"][case]
    sc = golden[f"scales_{case}"][:: max(1, int(fn) // 60)].copy()
    n = 10000
    N = oracle.padded(n)
    for T in (1, 8):
        _, lo, hi = fcwt.row_truncation(n, sc, T, fb=fb)
        W, _ = oracle.weights(N, sc, T, oracle.mother(fb, N))
        peak = oracle.mother(fb, N).max()
        for i in range(sc.size):
            mask = np.ones(N // 2, bool)
            mask[lo[i]:hi[i]] = False
            if mask.any():
                assert W[i][mask].max(initial=0.0) < 2.0 ** -36 * peak * (1 + 1e-6), (i, T)
        # exact mode keeps every nonzero bin
        _, lo_e, hi_e = fcwt.row_truncation(n, sc, T, exact_support=True, fb=fb)
        for i in range(sc.size):
            nz = np.nonzero(W[i])[0]
            if nz.size:
                assert lo_e[i] <= nz[0] and hi_e[i] > nz[-1]


def test_strict_nyquist_is_opt_in(fcwt, monkeypatch):
    """The reference asserts f1 <= fs/2 (src/fcwt/fcwt.cpp:148,167,184) but
    its release builds compile the asserts out, so by default f1 > fs/2 is
    accepted (the published benchmark runs fs=100 with f1=101). Strict mode,
    by argument or FCWT_STRICT=1, refuses it for Scales and for transforms."""
    monkeypatch.delenv("FCWT_STRICT", raising=False)
    m = fcwt.Morlet(2.0)
    s = fcwt.Scales(m, fcwt.FCWT_LINFREQS, 100, 1.0, 101.0, 50)  # accepted, like the release build
    with pytest.raises(ValueError, match="Nyquist"):
        fcwt.Scales(m, fcwt.FCWT_LINFREQS, 100, 1.0, 101.0, 50, strict=True)
    fcwt.Scales(m, fcwt.FCWT_LOGSCALES, 100, 1.0, 50.0, 50, strict=True)  # f1 = fs/2 is fine
    monkeypatch.setenv("FCWT_STRICT", "1")
    with pytest.raises(ValueError):
        fcwt.Scales(m, fcwt.FCWT_LOGSCALES, 1000, 1.0, 600.0, 20)
    monkeypatch.setenv("FCWT_STRICT", "0")
    fcwt.Scales(m, fcwt.FCWT_LOGSCALES, 1000, 1.0, 600.0, 20)
    # transforms: a scale below 2 is a centre frequency above fs/2
    from fcwt_b200 import _lib

    lib = _lib.load()
    sc = np.ascontiguousarray(s.scales)
    proc = np.zeros(sc.size, np.int32)
    assert sc.min() < 2.0
    assert lib.fcwt_row_truncation(10000, ctypes.c_float(2.0), sc.ctypes.data, sc.size, 1, 0,
                                   proc.ctypes.data, None, None) == 0
    rc = lib.fcwt_row_truncation(10000, ctypes.c_float(2.0), sc.ctypes.data, sc.size, 1, _lib.FCWT_STRICT,
                                 proc.ctypes.data, None, None)
    assert rc == _lib.FCWT_ERR_INVALID and b"Nyquist" in lib.fcwt_last_error()
