"""GPU parity: the CUDA path (through the C ABI) against the reference's golden
vectors and the float64 oracle. Tolerance: rel-L2 <= 1e-5 for complex64
output, 3e-3 for 16-bit outputs; truncation lengths,
scale grids and mother-table indices bit-exact (covered in test_host.py)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LINSCALES, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _run(fcwt, x, sc, fb, T, norm, complex_input=False, exact=False):
    x = np.asarray(x)
    out = np.zeros((len(sc), x.size), np.complex64)
    if exact:
        p = fcwt.Plan(x.size, sc, fb=fb, threads=T, norm=norm, complex_input=complex_input, exact_support=True)
        p.execute(x, out)
        p.close()
        return out
    f = fcwt.FCWT(fcwt.Morlet(fb), T, False, norm)
    (f.ccwt if complex_input else f.cwt)(x, sc, out)
    return out


def test_golden_c1_rows(fcwt, golden, oracle):
    x, sc = golden["c1_signal"], golden["scales_0"]
    out = _run(fcwt, x, sc, 2.0, 8, True)
    assert rel_l2(out[golden["c1_rows"]], golden["c1_out"]) < TOL
    assert rel_l2(out, oracle.cwt_fp64(x, sc, 2.0, 8, True)) < TOL
    assert np.allclose(np.abs(out).mean(axis=1), golden["c1_absmean"], rtol=1e-4, atol=1e-7)


def test_golden_stale_bins_sigma_half(fcwt, golden, oracle):
    x, sc = golden["s05_signal"], golden["s05_scales"]
    out = _run(fcwt, x, sc, 0.5, 1, False)
    assert rel_l2(out[golden["s05_rows"]], golden["s05_out"]) < TOL
    assert rel_l2(out, oracle.cwt_fp64(x, sc, 0.5, 1, False)) < TOL


CASES = [
    # n, fb, scaletype, fs, f0, f1, fn, threads, norm
    (1, 2.0, LOGSCALES, 1000, 1.0, 100.0, 5, 1, True),
    (2, 2.0, LOGSCALES, 1000, 1.0, 100.0, 5, 1, True),
    (3, 2.0, LINFREQS, 1000, 1.0, 100.0, 5, 1, False),
    (5, 2.0, LINFREQS, 1000, 1.0, 100.0, 5, 1, True),
    (17, 1.0, LOGSCALES, 1000, 10.0, 400.0, 9, 1, True),
    (100, 2.0, LOGSCALES, 1000, 5.0, 450.0, 20, 8, True),
    (511, 0.5, LINSCALES, 1000, 5.0, 450.0, 30, 3, True),
    (512, 6.0, LOGSCALES, 1000, 5.0, 450.0, 30, 1, False),
    (513, 2.0, LINFREQS, 1000, 5.0, 450.0, 30, 8, True),
    (1000, 16.0, LINFREQS, 1000, 1.0, 20.0, 200, 1, True),
    (1024, 2.0, LOGSCALES, 1000, 2.0, 490.0, 64, 8, True),
    (1500, 0.5, LOGSCALES, 1000, 2.0, 490.0, 50, 1, False),
    (4096, 4.0, LINSCALES, 1000, 2.0, 490.0, 50, 2, True),
    (6000, 2.0, LOGSCALES, 1000, 2.0, 490.0, 40, 1, True),
    (10000, 2.0, LINFREQS, 1000, 1.0, 101.0, 300, 1, True),
    (16384, 2.0, LOGSCALES, 1000, 2.0, 200.0, 128, 8, True),
    (16385, 2.0, LOGSCALES, 1000, 2.0, 200.0, 40, 8, True),
    (40000, 1.0, LOGSCALES, 1000, 1.0, 450.0, 40, 4, False),
    (65536, 6.0, LINFREQS, 30000, 1.0, 5000.0, 64, 8, True),
    (100000, 2.0, LINFREQS, 1000, 1.0, 101.0, 96, 1, True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}_fb{c[1]}_st{c[2]}_T{c[7]}")
def test_cwt_vs_fp64_oracle(fcwt, oracle, case):
    n, fb, st, fs, f0, f1, fn, T, norm = case
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 0.05)).astype(np.float32)
    sc = oracle.scales(st, fs, f0, f1, fn)
    out = _run(fcwt, x, sc, fb, T, norm)
    ref = oracle.cwt_fp64(x, sc, fb, T, norm)
    assert rel_l2(out, ref) < TOL
    exact = _run(fcwt, x, sc, fb, T, norm, exact=True)
    assert rel_l2(exact, ref) < TOL


@pytest.mark.parametrize("n", [1000, 4096, 8000, 30000])
def test_ccwt_complex_input(fcwt, oracle, n):
    rng = np.random.default_rng(11)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    sc = oracle.scales(LOGSCALES, 1000, 2.0, 450.0, 48)
    out = _run(fcwt, x, sc, 4.0, 8, True, complex_input=True)
    assert rel_l2(out, oracle.cwt_fp64(x, sc, 4.0, 8, True)) < TOL


def test_device_mother_table_matches_reference(fcwt, golden):
    total = mism = 0
    for k, (fb, N) in enumerate(golden["mother_cases"]):
        m = fcwt.Morlet(float(fb))
        m.generate(int(N))
        g = golden[f"mother_{k}"]
        total += g.size
        diff = m.mother.view(np.int32).astype(np.int64) - g.view(np.int32).astype(np.int64)
        # float64 exp rounded to float vs glibc expf (not always correctly rounded)
        assert np.abs(diff).max() <= 1, k
        mism += int(np.count_nonzero(diff))
    assert mism <= total // 1000


def test_odd_length_rows_are_unshifted(fcwt, oracle):
    n = 1001
    rng = np.random.default_rng(2)
    x = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 20.0, 64)
    out = _run(fcwt, x, sc, 16.0, 1, True)
    assert rel_l2(out, oracle.cwt_fp64(x, sc, 16.0, 1, True)) < TOL


@pytest.mark.parametrize("kind", ["descending", "custom"])
def test_scale_orders_and_stale_sources(fcwt, oracle, kind):
    """Descending grids (f0 > f1: no stale bins) and a non-monotone custom grid
    (stale bins from several earlier rows) follow the reference's reuse of O1."""
    n = 8192
    rng = np.random.default_rng(9)
    x = rng.standard_normal(n).astype(np.float32)
    if kind == "descending":
        sc = oracle.scales(LOGSCALES, 1000, 300.0, 3.0, 40)
    else:
        sc = np.concatenate([oracle.scales(LOGSCALES, 1000, 3.0, 300.0, 20),
                             oracle.scales(LOGSCALES, 1000, 2.0, 100.0, 15)[::-1],
                             rng.uniform(3.0, 200.0, 10).astype(np.float32)]).astype(np.float32)
    for fb in (0.5, 2.0):
        out = _run(fcwt, x, sc, fb, 4, True)
        assert rel_l2(out, oracle.cwt_fp64(x, sc, fb, 4, True)) < TOL


def test_torch_device_path_equals_host_path(fcwt, oracle):
    import torch

    n = 20000
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 100)
    host = _run(fcwt, x, sc, 2.0, 1, True)
    xd = torch.from_numpy(x).cuda()
    outd = torch.empty((sc.size, n), dtype=torch.complex64, device="cuda")
    fcwt.FCWT(fcwt.Morlet(2.0), 1, False, True).cwt(xd, sc, outd)
    torch.cuda.synchronize()
    assert np.array_equal(outd.cpu().numpy(), host)
    freqs, outb = fcwt.cwt_device(xd, 1000, 1.0, 101.0, 100)
    torch.cuda.synchronize()
    assert np.array_equal(outb.cpu().numpy(), host)


def test_repeated_calls_are_deterministic(fcwt, oracle):
    n = 50000
    x = np.random.default_rng(4).standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 64)
    a = _run(fcwt, x, sc, 2.0, 1, True)
    b = _run(fcwt, x, sc, 2.0, 1, True)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("out_type", ["bf16", "f16"])
def test_16bit_outputs(fcwt, oracle, out_type):
    import torch

    n = 30000
    x = np.random.default_rng(6).standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 50)
    ref = oracle.cwt_fp64(x, sc, 2.0, 1, True)
    dt = torch.bfloat16 if out_type == "bf16" else torch.float16
    _, out = fcwt.cwt_device(torch.from_numpy(x).cuda(), 1000, 1.0, 101.0, 50, out_dtype=dt)
    o = out.float().cpu().numpy()
    got = o[..., 0] + 1j * o[..., 1]
    assert rel_l2(got, ref) < 3e-3


def test_row_shard_plan_matches_full(fcwt, oracle):
    n = 40000
    x = np.random.default_rng(8).standard_normal(n).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 1.0, 450.0, 64)
    full = _run(fcwt, x, sc, 0.5, 2, True)
    for rb, re_ in [(0, 10), (10, 37), (37, 64)]:
        p = fcwt.Plan(n, sc, fb=0.5, threads=2, norm=True, rows=(rb, re_))
        out = np.zeros((re_ - rb, n), np.complex64)
        p.execute(x, out)
        p.close()
        assert np.array_equal(out, full[rb:re_])


def test_large_config_rows_and_linearity(fcwt, oracle):
    """100k x 3000 (LINFREQS 1-101 Hz at 1 kHz, σ=2): sampled rows against the
    float64 oracle and linearity of the full output."""
    import torch

    n, fn = 100000, 3000
    rng = np.random.default_rng(12)
    x = rng.standard_normal(n).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, fn)
    plan = fcwt.Plan(n, sc, fb=2.0, threads=1, norm=True)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    ox = torch.empty((fn, n), dtype=torch.complex64, device="cuda")
    oy = torch.empty_like(ox)
    oz = torch.empty_like(ox)
    plan.execute(xd, ox)
    plan.execute(yd, oy)
    plan.execute(2.0 * xd - 0.5 * yd, oz)
    torch.cuda.synchronize()
    fcwt.synchronize()
    lin = torch.linalg.vector_norm(oz - (2.0 * ox - 0.5 * oy)) / torch.linalg.vector_norm(oz)
    assert float(lin) < 1e-5
    rows = [0, 1, 777, 1500, 2998, 2999]
    ref = oracle.cwt_fp64(x, sc, 2.0, 1, True, rows=rows)
    got = ox[rows].cpu().numpy()
    assert rel_l2(got, ref) < TOL
    plan.close()


class _IndexTable:
    """A wavelet whose frequency-domain table is mother[w] = w: a row's
    daughter weight at bin q is then the mother-table index the row uses
    there (or, for bins past its truncation, the index an earlier row left in
    the reused O1 buffer)."""

    def __init__(self):
        self.width = 0
        self.four_wavelen = 1.0
        self.imag_frequency = False
        self.doublesided = False
        self.mother = None

    def generate(self, size):
        self.mother = np.arange(size, dtype=np.float32)


@pytest.mark.parametrize("mode", ["auto", "cuda_cores"])
def test_device_weights_equal_reference_daughter_product(fcwt, golden, mode):
    """The device path's truncation lengths, mother-table indices and reused
    bins, bit for bit against the reference's own daughter product
    (src/fcwt/fcwt.cpp:197-311 applied row after row, fcwt.cpp:514-518).
    A unit impulse has spectrum 1, so row i of the transform (n = N, norm on)
    is IFFT(W_i) and its float64 FFT returns W_i[q] = idx; rounding recovers
    the integer index exactly (the float32 transform error is < 0.05 here)."""
    import torch

    from fcwt_b200 import _lib

    c = _lib.context(0)
    c.set_engine(_lib.FCWT_ENGINE_AUTO if mode == "auto" else _lib.FCWT_ENGINE_CUDA_CORES)
    try:
        for k, (n, si, T) in enumerate(golden["dw_cases"]):
            n = int(n)
            sc = golden[f"scales_{si}"]
            rows = golden[f"dw_rows_{k}"]
            x = torch.zeros(n, dtype=torch.float32, device="cuda")
            x[0] = 1.0
            out = torch.empty((sc.size, n), dtype=torch.complex64, device="cuda")
            fcwt.FCWT(_IndexTable(), int(T), False, True).cwt(x, sc, out)
            y = out[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
            W = np.fft.fft(y, axis=1)
            half = n // 2
            err = np.max(np.abs(W[:, :half] - np.round(W[:, :half].real)))
            assert err < 0.05, (k, err)
            assert np.max(np.abs(W[:, half:])) < 0.05, k
            assert np.array_equal(np.round(W[:, :half].real).astype(np.int32), golden[f"dw_{k}"]), (k, mode)
    finally:
        c.set_engine(_lib.FCWT_ENGINE_AUTO)


@pytest.mark.parametrize("n", [1001, 9999, 40001])
@pytest.mark.parametrize("norm", [True, False])
def test_compat_align_shift_reproduces_reference_rows(fcwt, oracle, reference, n, norm):
    """With compat_align_shift the odd-n output equals the reference's own
    output row for row, including the rows its std::align writes one sample to
    the right and their element 0 (the previous row's sample n, normalised
    twice): src/fcwt/fcwt.cpp:418-445."""
    import torch

    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + np.sin(np.arange(n) * 0.02)).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 2.0, 400.0, 9)
    want = reference.cwt(x, sc, 2.0, 1000, 2, norm)
    assert want.ctypes.data % 16 == 0
    got = np.zeros_like(want)
    fcwt.FCWT(fcwt.Morlet(2.0), 2, False, norm, compat_align_shift=True).cwt(x, sc, got)
    for i in range(sc.size):
        assert rel_l2(got[i], want[i]) < 1e-5, i
        assert abs(got[i, 0] - want[i, 0]) <= 1e-5 * np.abs(want[i]).max() + 1e-30, i
    # device buffers: same
    dev = torch.empty((sc.size, n), dtype=torch.complex64, device="cuda")
    fcwt.FCWT(fcwt.Morlet(2.0), 2, False, norm, compat_align_shift=True).cwt(torch.from_numpy(x).cuda(), sc, dev)
    torch.cuda.synchronize()
    assert rel_l2(dev.cpu().numpy(), want) < 1e-5
    # without the mode, rows are clean (unshifted)
    clean = np.zeros_like(want)
    fcwt.FCWT(fcwt.Morlet(2.0), 2, False, norm).cwt(x, sc, clean)
    ref64 = oracle.cwt_fp64(x, sc, 2.0, 2, norm)
    assert rel_l2(clean, ref64) < 1e-5


def test_split_work_units_equal_whole_rows(fcwt, oracle):
    """The tensor-core queue splits the last rows of a launch into 2, 4 or 8
    column-group parts. A 7-row shard of the 100k x 3000 grid runs every row
    as parts; inside the full 3000-row plan rows 0-6 and 1500-1506 are whole
    units, and its last 74 rows are halves. Every split computes each column
    group the same way, so the rows are bit-equal."""
    import torch

    n = 100000
    x = torch.from_numpy(np.random.default_rng(11).standard_normal(n).astype(np.float32)).cuda()
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, 3000)
    full = torch.empty((3000, n), dtype=torch.complex64, device="cuda")
    p = fcwt.Plan(n, sc, fb=2.0, threads=8, norm=True)
    assert p.stats()["tensor_core_rows"] == 3000
    p.execute(x, full)
    p.close()
    for rb, re_ in [(0, 7), (1500, 1507), (2993, 3000)]:
        ps = fcwt.Plan(n, sc, fb=2.0, threads=8, norm=True, rows=(rb, re_))
        part = torch.full((re_ - rb, n), float("nan"), dtype=torch.complex64, device="cuda")
        ps.execute(x, part)
        ps.close()
        torch.cuda.synchronize()
        assert torch.equal(part, full[rb:re_]), (rb, re_)
    del full
    torch.cuda.empty_cache()
