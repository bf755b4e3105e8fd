"""GPU tests of the host-buffer path's row-block pipeline: outputs larger
than one 256 MB block are computed block by block into two device staging
slots and copied to the host while the next block is computed. The host
result must be bit-identical to the device-resident transform (same kernels,
same rows), for complex64 and BF16, even and odd lengths, and through the
reference-facing FCWT.cwt call (src/fcwt/fcwt.cpp:532-543)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,fn", [(100000, 700), (99999, 400)])
def test_pipelined_host_output_equals_device_output(fcwt, oracle, n, fn):
    import torch

    rng = np.random.default_rng(n)
    x = (np.sin(np.arange(n) * 0.01) + 0.2 * rng.standard_normal(n)).astype(np.float32)
    sc = oracle.scales(LINFREQS, 1000, 1.0, 101.0, fn)
    p = fcwt.Plan(n, sc, fb=2.0, threads=4, norm=True)
    assert p.stats()["tensor_core_rows"] == fn  # every row on the tensor-core engine: pipelined path
    assert fn * n * 8 > 256 << 20
    host = np.zeros((fn, n), np.complex64)
    p.execute(x, host)
    dev = torch.empty((fn, n), dtype=torch.complex64, device="cuda")
    p.execute(torch.from_numpy(x).cuda(), dev)
    torch.cuda.synchronize()
    assert np.array_equal(host, dev.cpu().numpy())
    ref = oracle.cwt_fp64(x, sc, 2.0, 4, True, rows=[0, fn // 2, fn - 1])
    assert rel_l2(host[[0, fn // 2, fn - 1]], ref) < 1e-5
    # the reference-facing call on numpy buffers
    out = np.zeros((fn, n), np.complex64)
    fcwt.FCWT(fcwt.Morlet(2.0), 4, False, True).cwt(x, sc, out)
    assert np.array_equal(out, host)
    if n % 4 == 0:
        h16 = np.zeros((fn, n, 2), np.uint16)
        p.execute(x, h16.view(np.uint32).reshape(fn, n), out_type=fcwt.FCWT_OUT_BF16)
        d16 = torch.empty((fn, n, 2), dtype=torch.bfloat16, device="cuda")
        p.execute(torch.from_numpy(x).cuda(), d16, out_type=fcwt.FCWT_OUT_BF16)
        torch.cuda.synchronize()
        assert np.array_equal(h16, d16.view(torch.int16).cpu().numpy().view(np.uint16))
