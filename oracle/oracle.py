"""CPU oracle for the fCWT transform path. TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed CPU baseline. The product
(``fcwt_b200``) never imports it.

Two oracles live here:

* ``Restatement`` — oracle/fcwt_oracle.c (plain C, float32 operation order of
  the reference) for the scale grids, the mother table, the truncation lengths
  and the per-row daughter weights including the reused-O1 "stale" bins, plus
  float64 numpy FFTs for the transform itself (``cwt_fp64``). The reference
  computes its FFTs with FFTW 3.3.10 in float32 (src/fcwt/fcwt.cpp:486-502);
  float64 here is the accuracy yardstick.
* ``Reference`` — the reference's own CPU path (src/fcwt/fcwt.cpp compiled by
  oracle/build_ref.sh into oracle/_ref/libfcwt_ref.so, FFTW + AVX + OpenMP),
  driven through oracle/ref_shim.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libfcwt_ref.so")

LINSCALES, LOGSCALES, LINFREQS = 0, 1, 2

_c_float = ctypes.c_float
_vp = ctypes.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def build(force: bool = False) -> str:
    """Compile oracle/fcwt_oracle.c into oracle/_build/liboracle.so (plain gcc,
    no contraction, no fast-math, glibc libm like the reference)."""
    src = os.path.join(HERE, "fcwt_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
                           "-fPIC", "-shared", src, "-lm", "-o", tmp])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def build_reference(reference_root: str | None = None) -> str | None:
    """Build oracle/_ref/libfcwt_ref.so from the reference sources, when they
    are present on this machine. The source tree is `reference_root`, else
    $FCWT_REFERENCE_ROOT, else the default of oracle/build_ref.sh. Returns the
    library path, or None when neither the sources nor a built library exist."""
    root = reference_root or os.environ.get("FCWT_REFERENCE_ROOT")
    args = ["bash", os.path.join(HERE, "build_ref.sh")] + ([root] if root else [])
    if subprocess.run(args, capture_output=True).returncode != 0:
        return REF_LIB_PATH if os.path.exists(REF_LIB_PATH) else None
    return REF_LIB_PATH


class Restatement:
    """ctypes front-end of oracle/fcwt_oracle.c."""

    def __init__(self):
        self.lib = ctypes.CDLL(build())
        L = self.lib
        L.or_find2power.restype = ctypes.c_int
        L.or_proc.restype = ctypes.c_int
        L.or_proc.argtypes = [ctypes.c_int, _c_float, ctypes.c_int, ctypes.c_int]
        L.or_index.restype = ctypes.c_int
        L.or_index.argtypes = [ctypes.c_int, _c_float, ctypes.c_int]
        L.or_scales.argtypes = [ctypes.c_int, ctypes.c_int, _c_float, _c_float, ctypes.c_int, _vp]
        L.or_frequencies.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp]
        L.or_mother.argtypes = [_c_float, ctypes.c_int, _vp]
        L.or_support.restype = ctypes.c_int
        L.or_support.argtypes = [_c_float, _c_float]
        L.or_get_wavelet.argtypes = [_c_float, _c_float, ctypes.c_int, _vp]
        L.or_weights.argtypes = [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                 _vp, _vp]
        L.or_weights_rows.argtypes = [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                      _vp, ctypes.c_int, _vp]

    def find2power(self, n: int) -> int:
        return self.lib.or_find2power(int(n))

    def padded(self, n: int) -> int:
        return 1 << self.find2power(n)

    def scales(self, scaletype: int, fs: int, f0: float, f1: float, fn: int) -> np.ndarray:
        out = np.zeros(fn, np.float32)
        self.lib.or_scales(scaletype, int(fs), f0, f1, fn, _ptr(out))
        return out

    def frequencies(self, scales: np.ndarray, fs: int) -> np.ndarray:
        scales = np.ascontiguousarray(scales, np.float32)
        out = np.zeros(scales.size, np.float32)
        self.lib.or_frequencies(_ptr(scales), scales.size, int(fs), _ptr(out))
        return out

    def mother(self, fb: float, N: int) -> np.ndarray:
        out = np.zeros(N, np.float32)
        self.lib.or_mother(fb, N, _ptr(out))
        return out

    def support(self, fb: float, scale: float) -> int:
        return self.lib.or_support(fb, scale)

    def wavelet(self, fb: float, scale: float, pn: int) -> np.ndarray:
        out = np.zeros(pn, np.complex64)
        self.lib.or_get_wavelet(fb, scale, pn, _ptr(out))
        return out

    def proc(self, N: int, scale: float, threads: int, avx: bool = True) -> int:
        return self.lib.or_proc(N, scale, threads, 1 if avx else 0)

    def procs(self, N: int, scales, threads: int, avx: bool = True) -> np.ndarray:
        return np.array([self.proc(N, float(s), threads, avx) for s in np.asarray(scales, np.float32)],
                        np.int32)

    def indices(self, N: int, scale: float, count: int) -> np.ndarray:
        return np.array([self.lib.or_index(N, scale, q) for q in range(count)], np.int32)

    def weights(self, N: int, scales, threads: int, mother: np.ndarray, avx: bool = True):
        scales = np.ascontiguousarray(scales, np.float32)
        fn = scales.size
        W = np.zeros((fn, max(N // 2, 1)), np.float32)
        procs = np.zeros(fn, np.int32)
        mother = np.ascontiguousarray(mother, np.float32)
        self.lib.or_weights(N, _ptr(scales), fn, threads, 1 if avx else 0, _ptr(mother), _ptr(W),
                            _ptr(procs))
        return W, procs

    def weights_rows(self, N: int, scales, threads: int, mother: np.ndarray, rows, avx: bool = True):
        scales = np.ascontiguousarray(scales, np.float32)
        sel = np.ascontiguousarray(sorted(int(r) for r in rows), np.int32)
        W = np.zeros((sel.size, max(N // 2, 1)), np.float32)
        mother = np.ascontiguousarray(mother, np.float32)
        self.lib.or_weights_rows(N, _ptr(scales), scales.size, threads, 1 if avx else 0, _ptr(mother),
                                 _ptr(sel), sel.size, _ptr(W))
        return sel, W

    def cwt_fp64(self, x, scales, fb: float, threads: int = 1, norm: bool = True,
                 avx: bool = True, rows=None, mother=None, imaginary: bool = False,
                 doublesided: bool = False) -> np.ndarray:
        """Float64 restatement of FCWT::cwt (src/fcwt/fcwt.cpp:447-529) with the
        reference's exact truncation, indices and stale-bin weights, and
        float64 FFTs. `mother` replaces the Morlet(fb) table by a caller's
        frequency-domain table of N entries (the Wavelet::generate(N) result,
        fcwt.cpp:504-505). imaginary / doublesided: the wavelet's
        imag_frequency / doublesided fields with the AVX product's semantics
        (fcwt.cpp:232-273): products times i; bins b in [N - proc, N) of the
        mirrored spectrum (fcwt.cpp:507-510) weighted by the row's weight at
        N - 1 - b (reused bins included). Returns complex128 [fn, n], or
        [len(rows), n] for the selected rows (ascending)."""
        x = np.asarray(x)
        n = x.size
        N = self.padded(n)
        xp = np.zeros(N, np.complex128)
        xp[:n] = x.astype(np.complex128) if np.iscomplexobj(x) else x.astype(np.float64)
        Ihat = np.fft.fft(xp)
        scales = np.ascontiguousarray(scales, np.float32)
        sel = list(range(scales.size)) if rows is None else sorted(int(r) for r in rows)
        table = self.mother(fb, N) if mother is None else np.ascontiguousarray(mother, np.float32)
        _, W = self.weights_rows(N, scales, threads, table, sel, avx)
        half = N // 2
        out = np.zeros((len(sel), n), np.complex128)
        if doublesided and N > 1:
            Im = Ihat.copy()
            i = np.arange(1, half)
            Im[N - i] = np.conj(Ihat[i])
        for k in range(len(sel)):
            O1 = np.zeros(N, np.complex128)
            O1[:half] = Ihat[:half] * W[k, :half].astype(np.float64)
            if doublesided and N > 1:
                b = np.arange(half, N)
                O1[half:] = Im[half:] * W[k, N - 1 - b].astype(np.float64)
            if imaginary:
                O1 *= 1j
            y = np.fft.ifft(O1)  # includes the 1/N
            if not norm:
                y = y * N
            out[k] = y[:n]
        return out


class Reference:
    """The reference's own CPU path, oracle/_ref/libfcwt_ref.so."""

    def __init__(self, path: str = REF_LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path}")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_scales.argtypes = [_c_float, ctypes.c_int, ctypes.c_int, _c_float, _c_float,
                                 ctypes.c_int, _vp]
        L.ref_frequencies.argtypes = L.ref_scales.argtypes
        L.ref_mother.argtypes = [_c_float, ctypes.c_int, _vp]
        L.ref_support.restype = ctypes.c_int
        L.ref_support.argtypes = [_c_float, _c_float]
        L.ref_wavelet.argtypes = [_c_float, _c_float, _vp, ctypes.c_int]
        L.ref_cwt.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _c_float, _vp, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]
        L.ref_find2power.restype = ctypes.c_int
        L.ref_cwt_table.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]
        L.ref_daughter.argtypes = [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, _vp, _vp, _vp]

    def padded(self, n: int) -> int:
        """1 << find2power(n) (src/fcwt/fcwt.h:154-165)."""
        return 1 << self.lib.ref_find2power(int(n))

    @staticmethod
    def available(path: str = REF_LIB_PATH) -> bool:
        return os.path.exists(path)

    def scales(self, scaletype: int, fs: int, f0: float, f1: float, fn: int, fb: float = 2.0):
        out = np.zeros(fn, np.float32)
        self.lib.ref_scales(fb, scaletype, int(fs), f0, f1, fn, _ptr(out))
        return out

    def frequencies(self, scaletype: int, fs: int, f0: float, f1: float, fn: int, fb: float = 2.0):
        out = np.zeros(fn, np.float32)
        self.lib.ref_frequencies(fb, scaletype, int(fs), f0, f1, fn, _ptr(out))
        return out

    def mother(self, fb: float, N: int) -> np.ndarray:
        out = np.zeros(N, np.float32)
        self.lib.ref_mother(fb, N, _ptr(out))
        return out

    def cwt_table(self, x, table, scales, threads: int = 1, norm: bool = True, imaginary: bool = False,
                  doublesided: bool = False) -> np.ndarray:
        """FCWT::cwt with a wavelet whose generate(N) returns `table` and whose
        imag_frequency / doublesided fields are set as given."""
        x = np.asarray(x)
        cplx = np.iscomplexobj(x)
        xin = np.ascontiguousarray(x, np.complex64 if cplx else np.float32)
        sc = np.ascontiguousarray(scales, np.float32)
        t = np.ascontiguousarray(table, np.float32)
        out = np.zeros((sc.size, xin.size), np.complex64)
        kind = (1 if imaginary else 0) | (2 if doublesided else 0)
        self.lib.ref_cwt_table(_ptr(xin), xin.size, 1 if cplx else 0, _ptr(t), t.size, _ptr(sc), sc.size,
                               int(threads), 1 if norm else 0, kind, _ptr(out))
        return out

    def daughter(self, N: int, scales, threads: int, mother=None, inp=None, imaginary: bool = False,
                 doublesided: bool = False, reset: bool = False) -> np.ndarray:
        """O1 after FCWT::daughter_wavelet_multiplication of each scale in turn
        (src/fcwt/fcwt.cpp:197-311), complex64 [fn, N]. Defaults: input all
        (1 + 0i), mother[w] = w (exact in float32 for N <= 2^24), so a written
        bin holds its mother-table index. reset: NaN-fill O1 before each row."""
        sc = np.ascontiguousarray(scales, np.float32)
        m = np.arange(N, dtype=np.float32) if mother is None else np.ascontiguousarray(mother, np.float32)
        x = np.ones(N, np.complex64) if inp is None else np.ascontiguousarray(inp, np.complex64)
        out = np.zeros((sc.size, N), np.complex64)
        self.lib.ref_daughter(int(N), _ptr(sc), sc.size, int(threads), 1 if imaginary else 0, 1 if doublesided else 0,
                              1 if reset else 0, _ptr(x), _ptr(m), _ptr(out))
        return out

    def truncation(self, N: int, scales, threads: int, nidx: int = 64):
        """The reference's own truncation lengths proc_i (bins its product
        writes) and mother-table indices idx_i(q) for q < min(nidx, proc_i)
        (-1 beyond), read back from daughter_wavelet_multiplication."""
        O = self.daughter(N, scales, threads, reset=True)
        half = max(N // 2, 1)
        written = ~np.isnan(O[:, :half].real)
        proc = np.where(written.all(axis=1), half, np.argmin(written, axis=1)).astype(np.int32)
        idx = np.full((O.shape[0], nidx), -1, np.int32)
        for i in range(O.shape[0]):
            k = min(nidx, int(proc[i]))
            idx[i, :k] = O[i, :k].real.astype(np.int32)
        return proc, idx

    def support(self, fb: float, scale: float) -> int:
        return self.lib.ref_support(fb, scale)

    def wavelet(self, fb: float, scale: float, pn: int) -> np.ndarray:
        out = np.zeros(pn, np.complex64)
        self.lib.ref_wavelet(fb, scale, _ptr(out), pn)
        return out

    def cwt(self, x, scales, fb: float, fs: int = 1000, threads: int = 1, norm: bool = True,
            out: np.ndarray | None = None) -> np.ndarray:
        """FCWT(Morlet(fb), threads, false, norm).cwt(x, n, out, scales)."""
        x = np.asarray(x)
        is_complex = np.iscomplexobj(x)
        x = np.ascontiguousarray(x, np.complex64 if is_complex else np.float32)
        scales = np.ascontiguousarray(scales, np.float32)
        n, fn = x.size, scales.size
        if out is None:
            out = np.zeros((fn, n), np.complex64)
        self.lib.ref_cwt(_ptr(x), n, 1 if is_complex else 0, fb, _ptr(scales), fn, int(fs),
                         int(threads), 0, 1 if norm else 0, _ptr(out))
        return out


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2 in float64."""
    a = np.asarray(a).astype(np.complex128).ravel()
    b = np.asarray(b).astype(np.complex128).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
