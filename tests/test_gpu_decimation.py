"""GPU tests of the fused decimation epilogues (fcwt_plan_create_strided):
every row_stride-th scale and every time_stride-th sample, computed directly
(the four-step inverse transform skips the columns it does not keep). Each
decimated output equals the same samples of the undecimated transform (rel-L2
<= 1e-6, float32 twiddle paths differ) and of the float64 oracle (<= 1e-5),
for both row engines, complex64 / BF16 / power outputs and odd lengths.
Reference behaviour decimated: FCWT::cwt, src/fcwt/fcwt.cpp:447-529."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx(fcwt):
    from fcwt_b200 import _lib

    c = _lib.context(0)
    yield c
    c.set_engine(_lib.FCWT_ENGINE_AUTO)


def _signal(n, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(n) / 1000.0
    return (np.sin(2 * np.pi * (5 + 20 * t / t[-1]) * t) + 0.3 * rng.standard_normal(n)).astype(np.float32)


@pytest.mark.parametrize("mode", ["auto", "cuda_cores"])
@pytest.mark.parametrize("n,fn,D,R", [
    (100000, 300, 2, 1), (100000, 300, 16, 3), (40001, 97, 8, 2), (5000, 50, 32, 1), (600, 20, 4, 3),
    (20000, 40, 2, 5),
])
def test_strided_plan_equals_decimated_transform(fcwt, oracle, ctx, mode, n, fn, D, R):
    import torch

    from fcwt_b200 import _lib

    ctx.set_engine(_lib.FCWT_ENGINE_AUTO if mode == "auto" else _lib.FCWT_ENGINE_CUDA_CORES)
    x = _signal(n, n + D)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, fn)
    xd = torch.from_numpy(x).cuda()
    full = torch.empty((fn, n), dtype=torch.complex64, device="cuda")
    fcwt.Plan(n, sc, fb=2.0, threads=4, norm=True).execute(xd, full)
    p = fcwt.Plan(n, sc, fb=2.0, threads=4, norm=True, row_stride=R, time_stride=D)
    rows_out, n_out = -(-fn // R), -(-n // D)
    assert p.out_shape == (rows_out, n_out)
    out = torch.full((rows_out, n_out), float("nan"), dtype=torch.complex64, device="cuda")
    p.execute(xd, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    want = full.cpu().numpy()[::R, ::D]
    assert np.isfinite(got).all()
    assert rel_l2(got, want) < 1e-6
    sel = [0, rows_out // 2, rows_out - 1]
    ref = oracle.cwt_fp64(x, sc, 2.0, 4, True, rows=[R * r for r in sel])[:, ::D]
    assert rel_l2(got[sel], ref) < 1e-5
    if mode == "auto" and n >= 20000:
        st = p.stats()
        assert st["rows"] == rows_out
    # 16-bit and power epilogues on the same decimated plan
    o16 = torch.empty((rows_out, n_out, 2), dtype=torch.bfloat16, device="cuda")
    p.execute(xd, o16, out_type=fcwt.FCWT_OUT_BF16)
    g16 = torch.complex(o16[..., 0].double(), o16[..., 1].double()).cpu().numpy()
    assert rel_l2(g16, want) < 3e-3
    pw = torch.empty((rows_out, n_out), dtype=torch.float32, device="cuda")
    p.execute(xd, pw, out_type=fcwt.FCWT_OUT_POWER)
    assert rel_l2(pw.cpu().numpy(), np.abs(want) ** 2) < 1e-5


def test_strided_plan_with_row_shard_and_host_buffers(fcwt, oracle):
    """Row shard [37, 211) decimated by 4 rows and 8 samples, numpy buffers."""
    n, fn = 70000, 256
    x = _signal(n, 5)
    sc = oracle.scales(LOGSCALES, 1000, 1.0, 200.0, fn)
    p = fcwt.Plan(n, sc, fb=2.0, threads=2, norm=True, rows=(37, 211), row_stride=4, time_stride=8)
    rows_out, n_out = -(-(211 - 37) // 4), -(-n // 8)
    out = np.zeros((rows_out, n_out), np.complex64)
    p.execute(x, out)
    rows = list(range(37, 211, 4))
    ref = oracle.cwt_fp64(x, sc, 2.0, 2, True, rows=rows)[:, ::8]
    assert rel_l2(out, ref) < 1e-5


def test_time_stride_limits(fcwt, oracle):
    from fcwt_b200._lib import FcwtError

    sc = oracle.scales(LOGSCALES, 1000, 2.0, 200.0, 8)
    with pytest.raises(FcwtError):  # not a power of two
        fcwt.Plan(10000, sc, time_stride=3)
    with pytest.raises(FcwtError):  # N = 16384 > 8192 allows at most 2
        fcwt.Plan(10000, sc, time_stride=4)
    with pytest.raises(FcwtError):
        fcwt.Plan(10000, sc, row_stride=0)
    fcwt.Plan(10000, sc, time_stride=2)
    fcwt.Plan(8000, sc, time_stride=64)  # N = 8192: whole-row path, any power of two
