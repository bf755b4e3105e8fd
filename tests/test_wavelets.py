"""Caller-supplied wavelets on the CPU: the oracle restatement with a
mother table equals the reference's own FCWT::cwt driven by a Wavelet
subclass that returns the same table (the reference's Wavelet interface,
src/fcwt/fcwt.h:67-79); the Paul table's shape."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LOGSCALES, Reference, Restatement, rel_l2


def _paul_table(N: int, m: int) -> np.ndarray:
    import fcwt_b200 as fcwt

    p = fcwt.Paul(m)
    p.generate(N)
    return p.mother


def test_paul_table_peak_and_decay():
    t = _paul_table(4096, 4)
    assert int(np.argmax(t)) == 2048
    assert t[2048] == pytest.approx(np.sqrt(2 * np.pi) * 0.75112554446, rel=1e-6)
    assert t[0] == 0.0 and np.all(t >= 0)
    y = 2.0 * np.arange(4096) / 4096
    A = np.sqrt(2 * np.pi) * 0.75112554446
    np.testing.assert_allclose(t[1:], (A * y[1:] ** 4 * np.exp(4 * (1 - y[1:]))).astype(np.float32), rtol=2e-6)


@pytest.mark.skipif(not Reference.available(), reason="reference build missing")
@pytest.mark.parametrize("kind", ["paul4", "morlet_table"])
def test_table_restatement_matches_reference(kind):
    o = Restatement()
    ref = Reference()
    rng = np.random.default_rng(3)
    n = 6000
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 0.03)).astype(np.float32)
    sc = o.scales(LOGSCALES, 1000, 2.0, 300.0, 40)
    N = o.padded(n)
    table = _paul_table(N, 4) if kind == "paul4" else o.mother(2.0, N)
    got = o.cwt_fp64(x, sc, 2.0, 4, True, mother=table)
    want = ref.cwt_table(x, table, sc, threads=4, norm=True)
    assert rel_l2(want, got) < 5e-7
    if kind == "morlet_table":
        # the same table through the Morlet path of the reference
        assert rel_l2(ref.cwt(x, sc, 2.0, 1000, 4, True), want) < 1e-7


@pytest.mark.skipif(not Reference.available(), reason="reference build missing")
@pytest.mark.parametrize("imag,double", [(True, False), (False, True), (True, True)])
def test_wavelet_kinds_restatement_matches_reference(imag, double):
    """imag_frequency and doublesided: the oracle's restatement of the AVX
    product (src/fcwt/fcwt.cpp:232-273, mirror of fcwt.cpp:507-510) against
    the reference's own FCWT::cwt with a Wavelet subclass setting those
    fields; real and complex input, small sigma (reused bins carry weight)."""
    o = Restatement()
    ref = Reference()
    rng = np.random.default_rng(11)
    n = 5000
    sc = o.scales(LOGSCALES, 1000, 2.0, 300.0, 40)
    N = o.padded(n)
    table = o.mother(0.7, N)
    for cplx in (False, True):
        x = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
        x = x.astype(np.complex64 if cplx else np.float32)
        want = ref.cwt_table(x, table, sc, threads=3, norm=True, imaginary=imag, doublesided=double)
        got = o.cwt_fp64(x, sc, 2.0, 3, True, mother=table, imaginary=imag, doublesided=double)
        assert rel_l2(want, got) < 5e-7, cplx


def test_dog_table():
    """DOG(m) tables: peak at the Morlet's peak entry N/2 with the Morlet's
    peak magnitude, sign of -i^m (the factor i of odd orders left to
    imag_frequency), zero at w = 0, two-sided."""
    import fcwt_b200 as fcwt

    A = np.sqrt(2 * np.pi) * 0.75112554446
    for m, sign in [(1, -1), (2, 1), (3, 1), (4, -1), (5, -1)]:
        d = fcwt.DOG(m)
        d.generate(4096)
        t = d.mother
        assert d.doublesided and d.imag_frequency == (m % 2 == 1)
        assert int(np.argmax(np.abs(t))) == 2048 and t[0] == 0.0
        assert t[2048] == pytest.approx(sign * A, rel=1e-6)
