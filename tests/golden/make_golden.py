"""Generates tests/golden/golden.npz from the reference's own CPU build.

Run here, where the reference sources exist:
    oracle/build_ref.sh && python tests/golden/make_golden.py
The fixtures are produced by oracle/_ref/libfcwt_ref.so (src/fcwt/fcwt.cpp of
fastlib/fCWT compiled with its shipped FFTW), so they pin both the oracle
restatement and the GPU path to the reference's behaviour:
  - scale grids and frequencies of the three Scales types;
  - Morlet mother tables (Morlet::generate(int));
  - per-row truncation lengths and mother-table indices for threads 1, 8 and
    16 on every scale case, read back from the reference's own
    FCWT::daughter_wavelet_multiplication (input 1, mother[w] = w);
  - per-bin daughter weights as mother-table indices, O1 reused row after
    row as FCWT::cwt does (stale bins included), for the device test that
    pushes a delta through a mother[w] = w wavelet;
  - time-domain wavelets (getWavelet);
  - coefficient rows of the reference transform for a 10k x 300 case
    (σ=2, LOGSCALES 1-101 Hz at 1 kHz) and a stale-bin-heavy σ=0.5 case.
Signals are seeded; the script is deterministic.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import LINFREQS, LINSCALES, LOGSCALES, Reference  # noqa: E402

SCALE_CASES = [
    # (scaletype, fs, f0, f1, fn)
    (LOGSCALES, 1000, 1.0, 101.0, 300),
    (LINFREQS, 1000, 1.0, 101.0, 3000),
    (LINSCALES, 1000, 1.0, 101.0, 300),
    (LINFREQS, 1000, 1.0, 20.0, 1000),
    (LOGSCALES, 100, 0.01, 10.0, 300),
    (LOGSCALES, 200000, 10.0, 80000.0, 1024),
    (LOGSCALES, 30000, 1.0, 5000.0, 77),
    (LINFREQS, 100, 1.0, 101.0, 300),
]
MOTHER_CASES = [(0.5, 1024), (2.0, 1024), (2.0, 16384), (6.0, 16384), (16.0, 4096)]
# signal length per scale case (odd lengths included); every case runs with threads 1, 8 and 16
TRUNC_N = [10000, 100000, 10000, 1001, 6000, 2 ** 20, 123457, 10000]
TRUNC_CASES = [(TRUNC_N[si], si, T) for si in range(len(SCALE_CASES)) for T in (1, 8, 16)]
# per-bin weight indices: (n = N, scale case, threads, rows)
DW_CASES = [
    (16384, 0, 8, [0, 1, 100, 299]),
    (32768, 6, 16, [0, 38, 76]),
    (16384, 4, 1, [0, 150, 299]),
]


def c1_signal(n=10000, fs=1000, seed=1):
    t = np.arange(n)
    rng = np.random.default_rng(seed)
    x = np.sin(2 * np.pi * (1 + 20 * t / n) * t / fs) + rng.normal(0, 0.1, n)
    return x.astype(np.float32)


def main():
    ref = Reference()
    g = {}
    for k, (st, fs, f0, f1, fn) in enumerate(SCALE_CASES):
        g[f"scales_{k}"] = ref.scales(st, fs, f0, f1, fn)
        g[f"freqs_{k}"] = ref.frequencies(st, fs, f0, f1, fn)
    g["scale_cases"] = np.array(SCALE_CASES, dtype=np.float64)
    for k, (fb, N) in enumerate(MOTHER_CASES):
        g[f"mother_{k}"] = ref.mother(fb, N)
    g["mother_cases"] = np.array(MOTHER_CASES, dtype=np.float64)
    for k, (n, si, T) in enumerate(TRUNC_CASES):
        sc = g[f"scales_{si}"]
        N = ref.padded(n)
        proc, idx = ref.truncation(N, sc, T)
        g[f"proc_{k}"] = proc
        rows = [0, len(sc) // 2, len(sc) - 1]
        g[f"index_{k}"] = idx[rows]
    g["trunc_cases"] = np.array(TRUNC_CASES, dtype=np.int64)
    for k, (n, si, T, rows) in enumerate(DW_CASES):
        sc = g[f"scales_{si}"]
        O = ref.daughter(n, sc, T)  # input 1, mother[w] = w, O1 kept across rows
        g[f"dw_{k}"] = O[rows, : n // 2].real.astype(np.int32)
        g[f"dw_rows_{k}"] = np.array(rows, np.int32)
    g["dw_cases"] = np.array([c[:3] for c in DW_CASES], dtype=np.int64)
    for k, (fb, scale) in enumerate([(2.0, 2.0), (2.0, 10.0), (16.0, 3.5)]):
        pn = 2 * ref.support(fb, scale) + 1
        g[f"wavelet_{k}"] = ref.wavelet(fb, scale, pn)
    g["wavelet_cases"] = np.array([(2.0, 2.0), (2.0, 10.0), (16.0, 3.5)])

    # coefficient rows: 10k x 300, σ = 2, LOGSCALES 1-101 Hz, threads 8, norm on
    x = c1_signal()
    sc = g["scales_0"]
    out = ref.cwt(x, sc, 2.0, fs=1000, threads=8, norm=True)
    rows = np.array([0, 37, 150, 299])
    g["c1_signal"] = x
    g["c1_rows"] = rows
    g["c1_out"] = out[rows]
    g["c1_absmean"] = np.abs(out).mean(axis=1).astype(np.float32)
    # stale-heavy: σ = 0.5, n = 4096, 64 LOGSCALES 2-200 Hz at 1 kHz, threads 1, norm off
    rng = np.random.default_rng(7)
    x2 = rng.standard_normal(4096).astype(np.float32)
    sc2 = ref.scales(LOGSCALES, 1000, 2.0, 200.0, 64)
    out2 = ref.cwt(x2, sc2, 0.5, fs=1000, threads=1, norm=False)
    rows2 = np.array([0, 1, 20, 63])
    g["s05_signal"] = x2
    g["s05_scales"] = sc2
    g["s05_rows"] = rows2
    g["s05_out"] = out2[rows2]
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **g)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
