"""The two row engines on the same inputs: the tcgen05 tensor-core engine
(split-FP16 phase-1 GEMM, rows whose window spans <= 16 blocks of 1024 bins,
N >= 16384; for 16-bit outputs also the column DFTs, as two radix-32 GEMM
stages) and the CUDA-core engine. Both against the float64 oracle at
rel-L2 <= 1e-5 (complex64) and <= 3e-3 (16-bit outputs), and against each
other. Cases cover the reference's stale bins (sigma 0.5), norm off, complex
input, odd n, several signals in one plan (plain stores instead of tensor-map
stores) and the continuous Morlet of the differentiable operator."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture
def ctx(fcwt):
    from fcwt_b200 import _lib

    c = _lib.context(0)
    yield c
    c.set_engine(_lib.FCWT_ENGINE_AUTO)


def _tc_rows(fcwt, n, sc, fb, T, exact=False):
    """Rows the tensor-core engine takes (host-side rule of the planner)."""
    _, lo, hi = fcwt.row_truncation(n, sc, threads=T, exact_support=exact, fb=fb)
    N = 1 << int(np.ceil(np.log2(n)))
    if N < 16384:
        return np.zeros(len(sc), bool)
    L = np.where(hi > lo, (lo // 1024) * 1024, 0)
    kw = np.where(hi > lo, (hi - L + 1023) // 1024, 0)
    return kw <= 16


def _plan_run(fcwt, ctx, mode, x, sc, fb, T, norm, complex_input=False, out_type=0):
    ctx.set_engine(mode)
    p = fcwt.Plan(x.size, sc, fb=fb, threads=T, norm=norm, complex_input=complex_input)
    if out_type == 0:
        out = np.zeros((len(sc), x.size), np.complex64)
    else:
        out = np.zeros((len(sc), x.size, 2), np.uint16)
    p.execute(x, out, out_type=out_type)
    p.close()
    return out


def _to_complex(out16, out_type):
    import torch

    t = torch.from_numpy(out16.view(np.int16))
    f = t.view(torch.bfloat16 if out_type == 1 else torch.float16).float().numpy()
    return f[..., 0] + 1j * f[..., 1]


CASES = [
    # n, fb, scaletype, fs, f0, f1, fn, threads, norm
    (100000, 2.0, LINFREQS, 1000, 1.0, 101.0, 64, 1, True),
    (16384, 2.0, LOGSCALES, 1000, 2.0, 200.0, 64, 8, True),
    (30000, 0.5, LOGSCALES, 1000, 2.0, 300.0, 48, 2, False),
    (65536, 6.0, LINFREQS, 30000, 1.0, 5000.0, 40, 8, True),
    (54321, 4.0, LOGSCALES, 200000, 10.0, 80000.0, 40, 1, True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}_fb{c[1]}_T{c[7]}")
def test_engines_match_oracle(fcwt, oracle, ctx, case):
    from fcwt_b200 import _lib

    n, fb, st, fs, f0, f1, fn, T, norm = case
    rng = np.random.default_rng(n + fn)
    x = (rng.standard_normal(n) + 2 * np.sin(np.arange(n) * 0.01)).astype(np.float32)
    sc = oracle.scales(st, fs, f0, f1, fn)
    assert _tc_rows(fcwt, n, sc, fb, T).any()
    ref = oracle.cwt_fp64(x, sc, fb, T, norm)
    tc = _plan_run(fcwt, ctx, _lib.FCWT_ENGINE_TENSOR_CORES, x, sc, fb, T, norm)
    cc = _plan_run(fcwt, ctx, _lib.FCWT_ENGINE_CUDA_CORES, x, sc, fb, T, norm)
    assert rel_l2(tc, ref) < TOL
    assert rel_l2(cc, ref) < TOL
    assert rel_l2(tc, cc) < 2 * TOL
    # row by row, for rows carrying energy
    e = np.linalg.norm(ref, axis=1)
    for i in np.nonzero(e > 1e-3 * e.max())[0]:
        assert rel_l2(tc[i], ref[i]) < 4 * TOL


def test_tensor_engine_complex_input_odd_n(fcwt, oracle, ctx):
    from fcwt_b200 import _lib

    n = 40001
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    sc = oracle.scales(LOGSCALES, 1000, 1.0, 450.0, 36)
    tc = _plan_run(fcwt, ctx, _lib.FCWT_ENGINE_TENSOR_CORES, x, sc, 2.0, 4, True, complex_input=True)
    ref = oracle.cwt_fp64(x, sc, 2.0, 4, True)
    assert rel_l2(tc, ref) < TOL


@pytest.mark.parametrize("n", [100000, 40002, 16384], ids=["tensor_map_stores", "plain_stores", "smallest_N"])
@pytest.mark.parametrize("out_type", [1, 2], ids=["bf16", "f16"])
def test_tensor_engine_16bit_outputs(fcwt, oracle, ctx, out_type, n):
    """16-bit outputs: tensor-map stores when n is a multiple of 4 (16-byte row
    stride), plain stores otherwise; N = 16384 is the smallest padded length of
    the tensor-core engine (16 columns, two groups per row)."""
    from fcwt_b200 import _lib

    rng = np.random.default_rng(3)
    x = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 32)
    out = _plan_run(fcwt, ctx, _lib.FCWT_ENGINE_TENSOR_CORES, x, sc, 2.0, 1, True, out_type=out_type)
    ref = oracle.cwt_fp64(x, sc, 2.0, 1, True)
    assert rel_l2(_to_complex(out, out_type), ref) < 3e-3


def test_tensor_engine_batched_plan(fcwt, oracle, ctx):
    """Several signals of different lengths and grids in one plan (the
    tensor-core engine stores through SMEM staging, no tensor map)."""
    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_TENSOR_CORES)
    rng = np.random.default_rng(11)
    ns = [20000, 70000, 16385]
    grids = [oracle.scales(LOGSCALES, 30000, 1.0, 5000.0, k) for k in (24, 40, 16)]
    xs = [rng.standard_normal(n).astype(np.float32) for n in ns]
    bp = fcwt.BatchPlan(ns, grids, fb=6.0, threads=1, norm=True)
    outs = [np.zeros((len(g), n), np.complex64) for g, n in zip(grids, ns)]
    bp.execute(xs, outs)
    bp.close()
    for x, g, o in zip(xs, grids, outs):
        assert rel_l2(o, oracle.cwt_fp64(x, g, 6.0, 1, True)) < TOL


def test_tensor_engine_device_tensors_repeat(fcwt, oracle, ctx):
    """Device-resident input and output, several executions of one plan."""
    import torch
    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_TENSOR_CORES)
    n = 100000
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 300)
    p = fcwt.Plan(n, sc, fb=2.0, threads=1, norm=True)
    xd = torch.from_numpy(x).cuda()
    out = torch.empty((300, n), dtype=torch.complex64, device="cuda")
    for _ in range(3):
        out.zero_()
        p.execute(xd, out)
    torch.cuda.synchronize()
    p.close()
    assert rel_l2(out.cpu().numpy(), oracle.cwt_fp64(x, sc, 2.0, 1, True)) < TOL


@pytest.mark.parametrize("out_type", [1, 2], ids=["bf16", "f16"])
def test_tensor_engine_16bit_repeat_bit_identical(fcwt, ctx, out_type):
    """16-bit outputs (column DFTs on the tensor cores) over many rows: every
    execution gives the same bits (no race between the CTA halves, the
    staging reuse and the stage MMAs) and matches the complex64 transform of
    the same plan within the 16-bit tolerance."""
    import torch
    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_TENSOR_CORES)
    n, fn = 100000, 600
    rng = np.random.default_rng(8)
    x = rng.standard_normal(n).astype(np.float32)
    sc = fcwt.Scales(fcwt.Morlet(2.0), fcwt.FCWT_LINFREQS, 1000, 1.0, 101.0, fn)
    p = fcwt.Plan(n, sc, fb=2.0, threads=1, norm=True)
    assert p.stats()["tensor_core_rows"] == fn
    xd = torch.from_numpy(x).cuda()
    dt = torch.bfloat16 if out_type == 1 else torch.float16
    outs = []
    for _ in range(3):
        o = torch.full((fn, n, 2), float("nan"), dtype=dt, device="cuda")
        p.execute(xd, o, out_type=out_type)
        outs.append(o)
    ref = torch.empty((fn, n), dtype=torch.complex64, device="cuda")
    p.execute(xd, ref)
    torch.cuda.synchronize()
    p.close()
    for o in outs[1:]:
        assert torch.equal(o.view(torch.int16), outs[0].view(torch.int16))
    got = torch.complex(outs[0][..., 0].double(), outs[0][..., 1].double())
    ref64 = ref.to(torch.complex128)
    err = float(torch.linalg.vector_norm(got - ref64) / torch.linalg.vector_norm(ref64))
    assert err < 3e-3


def test_tuner_records_engine_choice(fcwt, oracle, ctx, tmp_path, monkeypatch):
    """create_FFT_optimization_plan times both row engines for lengths the
    tensor-core engine can take and writes its choice into the plan file;
    transforms that load the file use it and stay within tolerance."""
    monkeypatch.chdir(tmp_path)
    f = fcwt.FCWT(fcwt.Morlet(2.0), 1, True, True)
    f.create_FFT_optimization_plan(20000, "FFTW_MEASURE")
    lines = dict(ln.split() for ln in open("n32768_t1.wis").read().splitlines()[1:])
    assert lines["engine"] in ("0", "1") and int(lines["N"]) == 32768
    rng = np.random.default_rng(4)
    x = rng.standard_normal(20000).astype(np.float32)
    sc = fcwt.Scales(fcwt.Morlet(2.0), fcwt.FCWT_LOGSCALES, 1000, 1.0, 400.0, 64)
    out = np.zeros((64, 20000), np.complex64)
    f.cwt(x, sc, out)
    assert rel_l2(out, oracle.cwt_fp64(x, sc.scales, 2.0, 1, True)) < TOL


@pytest.mark.parametrize("mode", ["tensor_cores", "cuda_cores"])
@pytest.mark.parametrize("n", [100000, 30001], ids=["tensor_map_stores", "plain_stores"])
def test_power_and_db_epilogues(fcwt, oracle, ctx, mode, n):
    """FCWT_OUT_POWER (|W|^2) and FCWT_OUT_DB (10 log10 |W|^2) written by the
    row kernels: both equal |W|^2 of the same plan's complex64 output W up to
    the epilogue's own float32 rounding, and the squared magnitude of the
    float64 oracle within the float32 transform's error. That error is absolute
    (about 1e-7 of the row's peak amplitude), so the dB comparison with the
    oracle covers the elements within 40 dB of the peak, where it is below
    1e-3 dB; the comparison with W covers every element above 1e-30."""
    from fcwt_b200 import _lib

    m = _lib.FCWT_ENGINE_TENSOR_CORES if mode == "tensor_cores" else _lib.FCWT_ENGINE_CUDA_CORES
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 0.02)).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 24)
    ref = np.abs(oracle.cwt_fp64(x, sc, 2.0, 1, True)) ** 2
    ctx.set_engine(m)
    p = fcwt.Plan(n, sc, fb=2.0, threads=1, norm=True)
    w = np.zeros((24, n), np.complex64)
    pw = np.zeros((24, n), np.float32)
    db = np.zeros((24, n), np.float32)
    p.execute(x, w)
    p.execute(x, pw, out_type=fcwt.FCWT_OUT_POWER)
    p.execute(x, db, out_type=fcwt.FCWT_OUT_DB)
    p.close()
    w2 = np.abs(w.astype(np.complex128)) ** 2
    assert np.max(np.abs(pw - w2) / np.maximum(w2, 1e-30)) < 1e-5
    own = w2 > 1e-30
    assert np.max(np.abs(db[own] - 10 * np.log10(w2[own]))) < 1e-4
    assert np.linalg.norm(pw - ref) / np.linalg.norm(ref) < 2e-5
    mask = ref > 1e-4 * ref.max()
    assert np.max(np.abs(db[mask] - 10 * np.log10(ref[mask]))) < 1e-3


@pytest.mark.parametrize("mode", ["tensor_cores", "cuda_cores"])
def test_maximum_padded_length(fcwt, oracle, ctx, mode):
    """n just above 2^22 (N = 2^23, the largest supported): 8192 columns per
    row, the w_M table read from global memory, 1024 column groups."""
    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_TENSOR_CORES if mode == "tensor_cores" else _lib.FCWT_ENGINE_CUDA_CORES)
    n = (1 << 22) + 1000
    rng = np.random.default_rng(23)
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 1e-3)).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 0.5, 1.5, 6)  # windows of <= 16 blocks of 1024 bins
    p = fcwt.Plan(n, sc, fb=2.0, threads=1, norm=True)
    if mode == "tensor_cores":
        assert p.stats()["tensor_core_rows"] == 6
    out = np.zeros((6, n), np.complex64)
    p.execute(x, out)
    p.close()
    assert rel_l2(out, oracle.cwt_fp64(x, sc, 2.0, 1, True)) < TOL
