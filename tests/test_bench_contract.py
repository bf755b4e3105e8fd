"""The parts of bench.py that fix the numbers it reports, checked on the CPU:
the algorithmic bytes of the default workload (the roofline numerator), the
output-type table behind `--out` and the per-type DRAM traffic constants."""
from __future__ import annotations

import bench


def test_algorithmic_bytes_of_default_workload():
    # fn*n*bytes_out + 4n (real input) + 8(N/2 + 1) (spectrum read)
    n, fn, N = bench.N_SAMPLES, bench.FN, 131072
    assert bench.algorithmic_bytes(n, fn, N) == fn * n * 8 + 4 * n + 8 * (N // 2 + 1) == 2400924296
    assert bench.algorithmic_bytes(n, fn, N, 4) == fn * n * 4 + 4 * n + 8 * (N // 2 + 1)


def test_output_types_map_to_library_constants():
    import fcwt_b200 as fcwt

    codes = {name: getattr(fcwt, spec[0]) for name, spec in bench.OUT_TYPES.items()}
    assert codes == {"complex64": fcwt.FCWT_OUT_C64, "bf16": fcwt.FCWT_OUT_BF16, "f16": fcwt.FCWT_OUT_F16,
                     "power": fcwt.FCWT_OUT_POWER, "db": fcwt.FCWT_OUT_DB}
    for name, (_, shape, dtype, nbytes) in bench.OUT_TYPES.items():
        # bytes per output point: complex64 8, 16-bit pairs 2 x 2, float32 scalograms 4
        assert nbytes == {"complex64": 8, "bfloat16": 4, "float16": 4, "float32": 4}[dtype]
        assert shape == ((2,) if dtype in ("bfloat16", "float16") else ())


def test_traffic_constants_are_per_launch_and_near_algorithmic():
    """Measured DRAM bytes of one full-size launch per output type: at least
    the output written, and within 1.25x of the algorithmic bytes."""
    N = 131072
    for name, traffic in bench.TRAFFIC_PER_LAUNCH.items():
        assert name in bench.OUT_TYPES
        algo = bench.algorithmic_bytes(bench.N_SAMPLES, bench.FN, N, bench.OUT_TYPES[name][3])
        assert 0.9 * algo < traffic < 1.25 * algo


def test_both_arms_print_the_same_config():
    """The reference arm and the GPU arm describe one workload: same keys and
    values, including the `threads` argument that sets the truncation length."""
    cfg = bench.plain_config()
    assert cfg == bench.plain_config(bench.FN, "complex64", bench.THREADS)
    assert cfg["threads_param"] == bench.THREADS and cfg["fn"] == 3000 and cfg["N"] == 131072


def test_reference_arm_loads_no_product_code():
    """`--impl reference` runs the reference build only: its code path names
    no fcwt_b200 module."""
    import inspect

    src = inspect.getsource(bench.run_reference_arm)
    assert "fcwt_b200" not in src and "_lib" not in src


def _shard_worker(rank, world, port, result_path):
    import os

    import numpy as np
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = bench.sharded_transform(compute=lambda x, b, e: None)
        if rank == 0:
            np.save(result_path, np.array(sh.blocks))
        assert sh.rows == sh.blocks[rank]
    finally:
        dist.destroy_process_group()


def test_sharded_bench_blocks_cover_all_rows(tmp_path):
    """bench.py --gpus N builds one ShardedCWT over the 100k x 3000 transform:
    the ranks' contiguous row blocks cover the 3000 rows exactly once."""
    import socket

    import numpy as np
    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    res = str(tmp_path / "blocks.npy")
    mp.start_processes(_shard_worker, args=(2, port, res), nprocs=2, join=True, start_method="spawn")
    blocks = np.load(res)
    assert blocks[0][0] == 0 and blocks[0][1] == blocks[1][0] and blocks[1][1] == bench.FN
    assert 0 < blocks[0][1] < bench.FN
