"""The MATLAB MEX gateway (fcwt_b200/mex/fcwtmex.cpp, calling convention of
the reference's src/MEX/fcwtmex.cpp). MATLAB is not installed, so the
gateway is compiled against a declarations-only stand-in of the mx/mex API
(tests/mex/mex.h) on the CPU, and on a GPU it is linked with a heap-backed
fake of that API (tests/mex/fake_mx.cpp), called like MATLAB would, and its
n x fn output is checked against the float64 oracle."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import LOGSCALES, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GW = os.path.join(ROOT, "fcwt_b200", "mex", "fcwtmex.cpp")
LIBDIR = os.path.join(ROOT, "fcwt_b200", "lib")
INC = ["-I" + os.path.join(ROOT, "tests", "mex"), "-I" + os.path.join(ROOT, "include")]


def test_gateway_compiles_against_the_mex_api(tmp_path):
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-c", GW, *INC, "-o", str(tmp_path / "gw.o")],
                   check=True, capture_output=True)


@pytest.mark.gpu
def test_gateway_transform(oracle, tmp_path):
    exe = str(tmp_path / "fake_mex")
    subprocess.run(["g++", "-std=c++17", GW, os.path.join(ROOT, "tests", "mex", "fake_mx.cpp"), *INC,
                    "-L" + LIBDIR, "-lfcwt_b200", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True, capture_output=True)
    n, fs, f0, f1, fn, c0 = 20000, 1000, 1.0, 100.0, 120, 2.0
    rng = np.random.default_rng(9)
    x = (np.sin(2 * np.pi * 12.0 * np.arange(n) / fs) + 0.2 * rng.standard_normal(n)).astype(np.float32)
    xin = tmp_path / "x.f32"
    x.tofile(xin)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(xin), str(n), str(c0), str(fs), str(f0), str(f1), str(fn), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, np.uint8)
    tfm = raw[: 8 * n * fn].view(np.complex64).reshape(fn, n)  # column-major n x fn = row-major fn x n
    freqs = raw[8 * n * fn:].view(np.float32)
    sc = oracle.scales(LOGSCALES, fs, f0, f1, fn)
    assert np.array_equal(freqs, oracle.frequencies(sc, fs))
    ref = oracle.cwt_fp64(x, sc, c0, threads=1, norm=True)
    assert rel_l2(tfm, ref) < 1e-5
