"""Pins the CPU oracle (oracle/) to the reference: golden vectors produced by
the reference's own CPU build (tests/golden/make_golden.py), and, where the
reference build is present, direct comparisons. CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LOGSCALES, rel_l2


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_scales_bit_exact(golden, oracle):
    for k, (st, fs, f0, f1, fn) in enumerate(golden["scale_cases"]):
        s = oracle.scales(int(st), int(fs), float(f0), float(f1), int(fn))
        assert np.array_equal(_bits(s), _bits(golden[f"scales_{k}"])), k
        f = oracle.frequencies(s, int(fs))
        assert np.array_equal(_bits(f), _bits(golden[f"freqs_{k}"])), k


def test_mother_bit_exact(golden, oracle):
    for k, (fb, N) in enumerate(golden["mother_cases"]):
        m = oracle.mother(float(fb), int(N))
        assert np.array_equal(_bits(m), _bits(golden[f"mother_{k}"])), k


def test_truncation_and_indices(golden, oracle):
    """Truncation lengths and mother-table indices of the restatement equal
    the ones read back from the reference's own daughter product (every scale
    case, threads 1, 8 and 16)."""
    assert {int(T) for _, _, T in golden["trunc_cases"]} == {1, 8, 16}
    assert len({int(si) for _, si, _ in golden["trunc_cases"]}) == len(golden["scale_cases"])
    for k, (n, si, T) in enumerate(golden["trunc_cases"]):
        sc = golden[f"scales_{si}"]
        N = oracle.padded(int(n))
        proc = golden[f"proc_{k}"]
        assert np.array_equal(oracle.procs(N, sc, int(T)), proc), k
        rows = [0, len(sc) // 2, len(sc) - 1]
        idx = np.stack([oracle.indices(N, float(sc[r]), 64) for r in rows])
        g = golden[f"index_{k}"]
        for j, r in enumerate(rows):
            m = min(64, int(proc[r]))
            assert np.all(g[j, m:] == -1), (k, r)  # bins the reference does not write
            assert np.array_equal(idx[j, :m], g[j, :m]), (k, r)


def test_daughter_weights_with_reused_bins(golden, oracle):
    """Per-bin daughter weights of the restatement, including the bins a row
    inherits from earlier rows through the reused O1 buffer, equal the
    reference's daughter product row after row (mother[w] = w, so each weight
    is its mother-table index)."""
    for k, (n, si, T) in enumerate(golden["dw_cases"]):
        sc = golden[f"scales_{si}"]
        rows = golden[f"dw_rows_{k}"]
        _, W = oracle.weights_rows(int(n), sc, int(T), np.arange(int(n), dtype=np.float32), rows)
        assert np.array_equal(W[:, : int(n) // 2].astype(np.int32), golden[f"dw_{k}"]), k


def test_reference_truncation_reads_back_directly(reference, oracle):
    """Direct check against the reference build (when present): proc_i for a
    grid the goldens do not hold."""
    sc = oracle.scales(LOGSCALES, 44100, 20.0, 20000.0, 200)
    for T in (1, 4, 32):
        proc, _ = reference.truncation(65536, sc, T)
        assert np.array_equal(proc, oracle.procs(65536, sc, T)), T


def test_wavelet_time_domain(golden, oracle):
    for k, (fb, scale) in enumerate(golden["wavelet_cases"]):
        g = golden[f"wavelet_{k}"]
        w = oracle.wavelet(float(fb), float(scale), g.size)
        assert np.array_equal(w.view(np.uint32), g.view(np.uint32)), k


def test_fp64_oracle_matches_reference_rows(golden, oracle):
    # reference FP32 (FFTW) vs float64 restatement: FP32 rounding only
    out = oracle.cwt_fp64(golden["c1_signal"], golden["scales_0"], 2.0, threads=8, norm=True,
                          rows=golden["c1_rows"])
    assert rel_l2(golden["c1_out"], out) < 1e-6


def test_fp64_oracle_stale_bins(golden, oracle):
    # σ = 0.5: the reused-O1 bins carry percent-level energy; the restatement
    # must reproduce them (ignoring them costs ~1e-2 rel-L2)
    out = oracle.cwt_fp64(golden["s05_signal"], golden["s05_scales"], 0.5, threads=1, norm=False,
                          rows=golden["s05_rows"])
    assert rel_l2(golden["s05_out"], out) < 1e-6


def test_oracle_vs_reference_random(oracle, reference):
    rng = np.random.default_rng(3)
    for n, fb, fn, T in [(3000, 1.0, 40, 2), (2048, 4.0, 33, 8), (778, 2.0, 20, 1)]:
        x = rng.standard_normal(n).astype(np.float32)
        sc = oracle.scales(LOGSCALES, 1000, 2.0, 400.0, fn)
        assert rel_l2(reference.cwt(x, sc, fb, 1000, T), oracle.cwt_fp64(x, sc, fb, T)) < 2e-6


def test_oracle_complex_input(oracle, reference):
    rng = np.random.default_rng(4)
    n = 4096
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    sc = oracle.scales(LOGSCALES, 1000, 2.0, 400.0, 24)
    assert rel_l2(reference.cwt(x, sc, 2.0, 1000, 4), oracle.cwt_fp64(x, sc, 2.0, 4)) < 2e-6


@pytest.mark.parametrize("n", [1000, 1001])
def test_reference_row_alignment_quirk(oracle, reference, n):
    """Documents the reference's std::align shift (src/fcwt/fcwt.cpp:425-426):
    for odd n, rows whose start address is 8 mod 16 are written one sample to
    the right. The product writes unshifted rows; this test pins the quirk."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 2.0, 400.0, 6)
    out = reference.cwt(x, sc, 2.0, 1000, 1)
    ref64 = oracle.cwt_fp64(x, sc, 2.0, 1)
    base = out.ctypes.data
    for i in range(sc.size - 1):
        shifted = (base + 8 * i * n) % 16 != 0
        if shifted:
            assert rel_l2(out[i, 1:], ref64[i, :-1]) < 2e-6
        else:
            assert rel_l2(out[i], ref64[i]) < 2e-6
    assert rel_l2(out[-1], ref64[-1]) < 2e-6
