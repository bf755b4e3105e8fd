"""GPU tests of caller-supplied wavelets (the reference's Wavelet
interface): the Paul wavelet and a user subclass through FCWT.cwt / ccwt,
numpy and torch buffers, both row engines, against the float64 oracle run on
the same mother table (rel-L2 <= 1e-5); unsupported kinds are refused."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


class GaussBump:
    """A user wavelet: single-sided Gaussian bump around x = 2 pi."""

    def __init__(self, width):
        self.width = 0
        self.four_wavelen = 1.0
        self.imag_frequency = False
        self.doublesided = False
        self.mother = None
        self.s = width

    def generate(self, size):
        x = 2.0 * np.arange(size) * (2 * np.pi / size)
        self.mother = (1.5 * np.exp(-0.5 * ((x - 2 * np.pi) * self.s) ** 2)).astype(np.float32)


@pytest.fixture
def ctx(fcwt):
    from fcwt_b200 import _lib

    c = _lib.context(0)
    yield c
    c.set_engine(_lib.FCWT_ENGINE_AUTO)


@pytest.mark.parametrize("mode", ["auto", "cuda_cores"])
@pytest.mark.parametrize("n", [3000, 40000])
def test_paul_matches_oracle(fcwt, oracle, ctx, mode, n):
    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_AUTO if mode == "auto" else _lib.FCWT_ENGINE_CUDA_CORES)
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 0.05)).astype(np.float32)
    paul = fcwt.Paul(4)
    sc = fcwt.Scales(paul, fcwt.FCWT_LOGSCALES, 1000, 2.0, 300.0, 48)
    out = np.zeros((48, n), np.complex64)
    fcwt.FCWT(paul, 2, False, True).cwt(x, sc, out)
    ref = oracle.cwt_fp64(x, sc.scales, 2.0, 2, True, mother=paul.mother)
    assert rel_l2(out, ref) < TOL


def test_user_wavelet_complex_input_and_torch(fcwt, oracle):
    import torch

    n = 20000
    rng = np.random.default_rng(4)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    w = GaussBump(3.0)
    sc = oracle.scales(LINFREQS, 1000, 5.0, 120.0, 32)
    f = fcwt.FCWT(w, 1, False, True)
    out = np.zeros((32, n), np.complex64)
    f.ccwt(x, sc, out)
    ref = oracle.cwt_fp64(x, sc, 2.0, 1, True, mother=w.mother)
    assert rel_l2(out, ref) < TOL
    xd = torch.from_numpy(x).cuda()
    od = torch.empty((32, n), dtype=torch.complex64, device="cuda")
    f.ccwt(xd, sc, od)
    torch.cuda.synchronize()
    assert rel_l2(od.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("mode", ["auto", "cuda_cores"])
@pytest.mark.parametrize("imag,double", [(True, False), (False, True), (True, True)])
def test_imag_frequency_and_doublesided_kinds(fcwt, oracle, ctx, mode, imag, double):
    """The reference's other wavelet kinds (Wavelet::imag_frequency and
    ::doublesided, AVX product of src/fcwt/fcwt.cpp:232-273) on a user table,
    real and complex input, numpy and torch buffers, both engines; sigma small
    enough that reused bins matter."""
    import torch

    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_AUTO if mode == "auto" else _lib.FCWT_ENGINE_CUDA_CORES)
    for n, cplx in [(30000, False), (20000, True), (3000, False)]:
        rng = np.random.default_rng(n + 7 * imag + 3 * double)
        x = rng.standard_normal(n) + np.sin(np.arange(n) * 0.04)
        if cplx:
            x = x + 1j * rng.standard_normal(n)
        x = x.astype(np.complex64 if cplx else np.float32)
        w = GaussBump(1.5)
        w.imag_frequency, w.doublesided = imag, double
        sc = oracle.scales(LOGSCALES, 1000, 3.0, 250.0, 24)
        f = fcwt.FCWT(w, 3, False, True)
        out = np.zeros((24, n), np.complex64)
        (f.ccwt if cplx else f.cwt)(x, sc, out)
        ref = oracle.cwt_fp64(x, sc, 2.0, 3, True, mother=w.mother, imaginary=imag, doublesided=double)
        assert rel_l2(out, ref) < TOL, (n, cplx)
        xd = torch.from_numpy(x).cuda()
        od = torch.empty((24, n), dtype=torch.complex64, device="cuda")
        (f.ccwt if cplx else f.cwt)(xd, sc, od)
        torch.cuda.synchronize()
        assert rel_l2(od.cpu().numpy(), ref) < TOL, (n, cplx, "torch")


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_dog_wavelet(fcwt, oracle, order):
    """DOG(m): doublesided, imaginary for odd m; against the float64 oracle on
    the same table, and the peak-frequency check of the reference's
    (commented-out) test_dog (tests/test_fcwt.py:156-182)."""
    fs, n = 64, 10000
    hz = 5.3
    x = np.sin(2 * np.pi * hz * (np.arange(n) / fs)).astype(np.float32)
    dog = fcwt.DOG(order)
    assert dog.doublesided and dog.imag_frequency == (order % 2 == 1)
    sc = fcwt.Scales(dog, fcwt.FCWT_LINFREQS, fs, 1.0, 32.0, 300)
    freqs = np.zeros(300, np.float32)
    sc.getFrequencies(freqs)
    out = np.zeros((300, n), np.complex64)
    fcwt.FCWT(dog, 8, False, True).cwt(x, sc, out)
    ref = oracle.cwt_fp64(x, sc.scales, 2.0, 8, True, mother=dog.mother, imaginary=dog.imag_frequency,
                          doublesided=True)
    assert rel_l2(out, ref) < TOL
    peak = float(freqs[int(np.argmax(np.mean(np.abs(out), axis=1)))])
    assert abs(peak - hz) < 0.5


def test_unsupported_outputs_are_refused(fcwt, oracle):
    """A mother table of the wrong length, and a doublesided wavelet with a
    16-bit output (doublesided rows are combined in complex64), are refused."""
    import ctypes

    import torch

    from fcwt_b200 import _lib
    from fcwt_b200._lib import FcwtError

    sc = oracle.scales(LOGSCALES, 1000, 2.0, 300.0, 8)
    w = GaussBump(3.0)
    w.doublesided = True
    x = torch.ones(1000, device="cuda")
    o16 = torch.empty((8, 1000, 2), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(FcwtError) as ei:
        fcwt.FCWT(w, 1, False, True).cwt(x, sc, o16, out_type=fcwt.FCWT_OUT_BF16)
    assert ei.value.args[0] == _lib.FCWT_ERR_UNSUPPORTED or "complex64" in str(ei.value)
    bad = np.ones(100, np.float32)  # N for n = 1000 is 1024
    with pytest.raises(FcwtError):
        _lib.call("fcwt_cwt_mother", _lib.context(0).handle, ctypes.c_void_p(np.ones(1000, np.float32).ctypes.data),
                  1000, 0, ctypes.c_void_p(bad.ctypes.data), bad.size, ctypes.c_void_p(sc.ctypes.data), sc.size, 1,
                  1, ctypes.c_void_p(np.zeros((8, 1000), np.complex64).ctypes.data), 0)
