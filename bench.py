"""Benchmark of the fCWT transform path on B200.

Workload (the 100k x 3000 configuration): one real float32 signal of
n = 100,000 samples at fs = 1 kHz (sum of 3 seeded chirps plus white noise,
unit RMS), padded to N = 131,072; Morlet sigma = 2.0; 3000 linearly spaced
frequencies 1-101 Hz (LINFREQS); normalisation on; complex64 output
[3000 x 100000] (2.4 GB); float32 arithmetic. One step = one full transform
(forward FFT of the signal + all 3000 rows) through a reusable plan.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0). Metric: output points/s = n * fn / t.
`value` times the transform with input and output resident in HBM (CUDA
events on the launching stream, max over ranks); `e2e` times the
reference-facing call FCWT.cwt(numpy in, numpy out) with pinned host buffers,
host<->device copies included. `--impl reference` times the reference's own
CPU path (FFTW + OpenMP, built from its sources into oracle/_ref) on the host
cores on the same workload.

Multi-GPU (torchrun): every rank runs its own full 100k x 3000 job on its GPU
(independent signals, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SAMPLES = 100_000
FS = 1000
F0, F1, FN = 1.0, 101.0, 3000
SIGMA = 2.0
WORKLOAD = "cwt_100k_x_3000: real f32 n=100000 (N=131072) fs=1000, Morlet sigma=2, LINFREQS 1-101 Hz fn=3000, complex64 out"


def make_signal(seed: int) -> np.ndarray:
    """Sum of 3 seeded linear chirps (random 1-100 Hz ranges and phases) plus
    white noise, scaled to unit RMS."""
    rng = np.random.default_rng(seed)
    t = np.arange(N_SAMPLES) / FS
    T = N_SAMPLES / FS
    x = np.zeros(N_SAMPLES)
    for _ in range(3):
        fa, fb = rng.uniform(1, 100, 2)
        ph = rng.uniform(0, 2 * np.pi)
        x += np.sin(2 * np.pi * (fa * t + 0.5 * (fb - fa) / T * t * t) + ph)
    x += rng.normal(0, 0.5, N_SAMPLES)
    x /= np.sqrt(np.mean(x * x))
    return x.astype(np.float32)


def algorithmic_bytes(n: int, fn: int, N: int, out_bytes: int = 8) -> int:
    # output + real input + spectrum read (bins < N/2 + 1)
    return fn * n * out_bytes + 4 * n + 8 * (N // 2 + 1)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_time(x: np.ndarray, scales: np.ndarray, threads: int, runs: int):
    """Times the reference's CPU path (oracle/_ref) on the full workload:
    median wall time of `runs` calls after one warm-up."""
    from oracle.oracle import Reference

    ref = Reference()
    out = np.zeros((scales.size, x.size), np.complex64)
    ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
    ts = []
    for _ in range(runs):
        t0 = time.perf_counter()
        ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts), ts


def run_reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    from oracle.oracle import Reference

    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/libfcwt_ref.so missing"}))
        return
    import fcwt_b200.api as api

    x = make_signal(1234)
    scales = np.zeros(FN, np.float32)
    from fcwt_b200 import _lib  # host-only helper for the grid (bit-exact with the reference)

    _lib.call("fcwt_scales", api.FCWT_LINFREQS, FS, api.ctypes.c_float(F0), api.ctypes.c_float(F1), FN,
              api._ptr(scales))
    threads = os.cpu_count() or 1
    ref = Reference()
    out = np.zeros((FN, N_SAMPLES), np.complex64)
    for _ in range(max(args.warmup, 0)):
        ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
        ts.append(time.perf_counter() - t0)
    tot = sum(ts)
    v = N_SAMPLES * FN * args.steps / tot
    line = {
        "impl": "reference", "metric": "scalogram points/s", "value": v, "unit": "points/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": N_SAMPLES, "fn": FN, "N": 131072},
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": threads, "kind": "reference",
                         "sample": f"full workload, {args.steps} timed calls of FCWT::cwt (FFTW+OpenMP, {threads} threads)"},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-runs", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fn", type=int, default=FN,
                    help="number of rows; values other than 3000 are for profiling captures only")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import fcwt_b200 as fcwt
    from fcwt_b200 import _lib

    dev = local_rank
    x = make_signal(1234 + rank)
    morl = fcwt.Morlet(SIGMA)
    fn = args.fn
    sc = fcwt.Scales(morl, fcwt.FCWT_LINFREQS, FS, F0, F1, fn)
    plan = fcwt.Plan(N_SAMPLES, sc, fb=SIGMA, threads=1, norm=True, device=dev)
    N = 1 << _lib.load().fcwt_find2power(N_SAMPLES)
    xd = torch.from_numpy(x).to(f"cuda:{dev}")
    out = torch.empty((fn, N_SAMPLES), dtype=torch.complex64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    ctx = plan.ctx

    # warm-up
    for _ in range(args.warmup):
        plan.execute(xd, out, stream=stream)
    torch.cuda.synchronize(dev)
    ctx.synchronize()

    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ctx.profile_enable(True)
    ctx.profile_read()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.execute(xd, out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    eng_ms, eng_n, kernels = ctx.profile_read()
    ctx.profile_enable(False)
    ctx.synchronize()
    clocks = sampler.stop() if sampler else None
    if dist:
        t = torch.tensor([ms_total, eng_ms / max(eng_n, 1)], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total, eng_avg = float(t[0]), float(t[1])
    else:
        eng_avg = eng_ms / max(eng_n, 1)
    ms_step = ms_total / args.steps
    points = N_SAMPLES * fn
    value = world * points * args.steps / (ms_total / 1e3)

    # ---- e2e: reference-facing call with host buffers (pinned)
    e2e = None
    if args.e2e_steps > 0:
        xin = torch.from_numpy(x).pin_memory()
        hout = torch.empty((fn, N_SAMPLES), dtype=torch.complex64, pin_memory=True)
        xin_np, hout_np = xin.numpy(), hout.numpy()
        f = fcwt.FCWT(morl, 1, False, True, device=dev)
        f.cwt(xin_np, sc, hout_np)  # warm
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            f.cwt(xin_np, sc, hout_np)
        te = time.perf_counter() - t0
        if dist:
            tt = torch.tensor([te], device=f"cuda:{dev}", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt[0])
        e2e = {"value": world * points * args.e2e_steps / te, "unit": "points/s",
               "h2d_bytes_per_step": 4 * N_SAMPLES, "d2h_bytes_per_step": 8 * points,
               "ms_per_step": 1e3 * te / args.e2e_steps, "host_buffers": "pinned"}
        del xin, hout

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import Reference

        if Reference.available():
            threads = os.cpu_count() or 1
            tmed, ts = cpu_reference_time(x, sc.scales, threads, args.cpu_runs)
            cpu = {"value": points / tmed, "unit": "points/s", "cores": threads, "kind": "reference",
                   "sample": f"full workload, median of {len(ts)} calls of the reference FCWT::cwt "
                             f"(FFTW 3.3.10 + OpenMP, threads={threads}, norm on)"}
        else:
            cpu = {"value": None, "unit": "points/s", "cores": 0, "kind": "reference",
                   "sample": "reference build missing"}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = load_peaks()
    algo = algorithmic_bytes(N_SAMPLES, fn, N)
    achieved = algo / (eng_avg / 1e3) / 1e9
    line = {
        "metric": "scalogram points/s", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD if fn == FN else WORKLOAD.replace("fn=3000", f"fn={fn}"),
                   "n": N_SAMPLES, "N": N, "fn": fn, "fs": FS, "f0": F0, "f1": F1,
                   "sigma": SIGMA, "scaling": "LINFREQS", "threads_param": 1, "out": "complex64",
                   "l2": "each step writes a 2.4 GB output (> 126 MB L2); no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "k_row_engine", "kernel_ms": eng_avg, "algorithmic_bytes": algo},
        "hbm_gbs_step": algo / (ms_step / 1e3) / 1e9,
        "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": kernels,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
