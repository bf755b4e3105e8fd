"""The C++ drop-in (include/fcwt.h + libfcwt_b200.so) exercised the way a
user of the reference's C++ API would: the README's example program
(fastlib/fCWT README.md:139-214) is compiled with g++ against our header and
linked against our library, unchanged apart from writing its results to a
file. Host-only parts run on the CPU; the transform itself is a GPU test,
checked against the float64 oracle."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "readme_example.cpp")
LIBDIR = os.path.join(ROOT, "fcwt_b200", "lib")


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "readme_example")
    subprocess.run(["g++", "-std=c++17", "-O1", SRC, "-I" + os.path.join(ROOT, "include"), "-L" + LIBDIR,
                    "-lfcwt_b200", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True, capture_output=True)
    return exe


def _run(exe, mode, out, strict=False, cwd=None):
    env = dict(os.environ)
    env.pop("FCWT_STRICT", None)
    if strict:
        env["FCWT_STRICT"] = "1"
    return subprocess.run([exe, mode, out], env=env, cwd=cwd, capture_output=True, text=True, timeout=600)


def test_readme_program_host_parts(example, oracle, tmp_path):
    out = str(tmp_path / "host.bin")
    for strict in (False, True):
        r = _run(example, "host", out, strict)
        assert r.returncode == 0, r.stderr
        raw = open(out, "rb").read()
        sc = np.frombuffer(raw[:1200], np.float32)
        fr = np.frombuffer(raw[1200:2400], np.float32)
        ref_sc = oracle.scales(LOGSCALES, 1000, 1.0, 101.0, 300)
        assert np.array_equal(sc.view(np.uint32), ref_sc.view(np.uint32))
        assert np.array_equal(fr.view(np.uint32), oracle.frequencies(ref_sc, 1000).view(np.uint32))
        sup = int(np.frombuffer(raw[2400:2404], np.int32)[0])
        assert sup == oracle.support(2.0, 10.0)
        m = 2 * sup + 1
        re = np.frombuffer(raw[2404:2404 + 4 * m], np.float32)
        im = np.frombuffer(raw[2404 + 4 * m:2404 + 8 * m], np.float32)
        w = oracle.wavelet(2.0, 10.0, m)
        assert np.array_equal(re, w.real) and np.array_equal(im, w.imag)
        threw = int(np.frombuffer(raw[2404 + 8 * m:2408 + 8 * m], np.int32)[0])
        assert threw == (1 if strict else 0)


@pytest.mark.gpu
def test_readme_program_transform(example, oracle, tmp_path):
    out = str(tmp_path / "gpu.bin")
    r = _run(example, "gpu", out, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    # optplan = true with no tuning file: the reference's warning, then the transform
    assert "n131072_t8.wis" in r.stdout
    n, fn = 100000, 3000
    raw = np.fromfile(out, np.uint8)
    sig = raw[: 4 * n].view(np.float32)
    sc = raw[4 * n: 4 * n + 4 * fn].view(np.float32)
    rows = raw[4 * n + 4 * fn:].view(np.complex64).reshape(3, n)
    assert np.array_equal(sc, oracle.scales(LINFREQS, 1000, 1.0, 32.0, fn))
    ref = oracle.cwt_fp64(sig, sc, 2.0, threads=8, norm=False, rows=[0, fn // 2, fn - 1])
    assert rel_l2(rows, ref) < 1e-5
