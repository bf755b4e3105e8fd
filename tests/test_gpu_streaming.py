"""GPU tests of the streaming transform: every frame of a sliding window
equals the transform of that window by a plan (same kernels), for pushes of
arbitrary block sizes, with and without CUDA-graph replay, and for the hop
and window emit modes."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [True, False])
def test_frames_equal_windowed_transforms(fcwt, oracle, graph):
    import torch

    from fcwt_b200.streaming import StreamingCWT

    W, H = 16384, 4096
    rng = np.random.default_rng(1)
    L = W + 5 * H + 100
    x = (rng.standard_normal(L) + np.sin(np.arange(L) * 0.01)).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 1.0, 400.0, 40)
    s = StreamingCWT(W, H, sc, fb=2.0, graph=graph)
    frames = []
    for a in range(0, L, 3000):                       # blocks unrelated to the hop
        frames += [f.clone() for f in s.push(x[a:a + 3000])]
    assert len(frames) == 6
    p = fcwt.Plan(W, sc, fb=2.0, threads=1, norm=True)
    for k, f in enumerate(frames):
        seg = torch.from_numpy(x[k * H:k * H + W]).cuda()
        ref = torch.empty((40, W), dtype=torch.complex64, device="cuda")
        p.execute(seg, ref)
        torch.cuda.synchronize()
        assert torch.equal(f, ref)
    assert rel_l2(frames[-1].cpu().numpy(), oracle.cwt_fp64(x[5 * H:5 * H + W], sc, 2.0, 1, True)) < 1e-5
    p.close()
    s.close()


def test_hop_emit_and_power_output(fcwt, oracle):
    import torch

    from fcwt_b200.streaming import StreamingCWT

    W, H = 16384, 8192
    rng = np.random.default_rng(2)
    x = rng.standard_normal(W + 2 * H).astype(np.float32)
    sc = oracle.scales(LOGSCALES, 1000, 1.0, 400.0, 24)
    s = StreamingCWT(W, H, sc, fb=2.0, emit="hop", out_type=fcwt.FCWT_OUT_POWER)
    frames = s.push(torch.from_numpy(x).cuda())
    assert len(frames) == 3 and frames[0].shape == (24, H)
    ref = np.abs(oracle.cwt_fp64(x[2 * H:2 * H + W], sc, 2.0, 1, True)) ** 2
    got = frames[-1].cpu().numpy()
    assert np.linalg.norm(got - ref[:, W - H:]) / np.linalg.norm(ref[:, W - H:]) < 2e-5
    s.close()
