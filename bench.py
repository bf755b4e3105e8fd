"""Benchmark of the fCWT transform path on B200.

Workload (the 100k x 3000 configuration): one real float32 signal of
n = 100,000 samples at fs = 1 kHz (sum of 3 seeded chirps plus white noise,
unit RMS), padded to N = 131,072; Morlet sigma = 2.0; 3000 linearly spaced
frequencies 1-101 Hz (LINFREQS); normalisation on; complex64 output
[3000 x 100000] (2.4 GB); float32 arithmetic. One step = one full transform
(forward FFT of the signal + all 3000 rows) through a reusable plan. Both
arms pass threads = os.cpu_count() (the reference's `threads` argument also
sets the per-scale truncation length, src/fcwt/fcwt.cpp:213-214, so the two
arms compute the same transform).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0). Metric: output points/s = n * fn / t.
`value` times the transform with input and output resident in HBM (CUDA
events on the launching stream, max over ranks); `e2e` times the
reference-facing call FCWT.cwt(numpy in, numpy out) with pinned host buffers,
host<->device copies included. `--impl reference` times the reference's own
CPU path (FFTW + OpenMP, built from its sources into oracle/_ref) on the host
cores on the same workload; it loads nothing of fcwt_b200.

At N = 1 the line also carries the other forms of the transform, each timed
on its own workload and checked against the float64 oracle on sampled rows
outside the timed region (`forms`): BF16 and |W|^2 outputs of this workload,
384 uneven channels in one persistent launch, the complex 2^20 x 1024 signal
with BF16 output, and the differentiable 64 x 16384 x 128 step.

Multi-GPU (torchrun, N > 1): one 100k x 3000 transform is split by scale rows
across the ranks (fcwt_b200.distributed.ShardedCWT, cost-balanced contiguous
row blocks): each step broadcasts the signal from rank 0 over NCCL and runs
the rank's row block; the shards stay on their GPUs (no gather in the timed
region; the gather is timed separately). Strong scaling.
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
N_PADDED = 131_072
FS = 1000
F0, F1, FN = 1.0, 101.0, 3000
SIGMA = 2.0
LINFREQS, LOGSCALES = 2, 1
THREADS = os.cpu_count() or 1
# DRAM bytes (read + write) of one k_row_tc launch of this workload, per
# output type, from one-pass ncu captures of the full-size launch
# (dram__bytes_read.sum + dram__bytes_write.sum; the capture summaries are
# kept under profiles/, named for the kernel and the workload)
TRAFFIC_PER_LAUNCH = {"complex64": 147.96e6 + 2.34565e9, "bf16": 156.01e6 + 1.14550e9}

# --out choices: (constant in fcwt_b200, trailing shape, torch dtype, bytes per point)
OUT_TYPES = {
    "complex64": ("FCWT_OUT_C64", (), "complex64", 8),
    "bf16": ("FCWT_OUT_BF16", (2,), "bfloat16", 4),
    "f16": ("FCWT_OUT_F16", (2,), "float16", 4),
    "power": ("FCWT_OUT_POWER", (), "float32", 4),
    "db": ("FCWT_OUT_DB", (), "float32", 4),
}
WORKLOAD = "cwt_100k_x_3000: real f32 n=100000 (N=131072) fs=1000, Morlet sigma=2, LINFREQS 1-101 Hz fn=3000, complex64 out"


def plain_config(fn: int = FN, out: str = "complex64", threads: int = THREADS) -> dict:
    """The `config` object of the 100k x 3000 workload; both arms print it."""
    return {"workload": WORKLOAD.replace("fn=3000", f"fn={fn}").replace("complex64 out", f"{out} out"),
            "n": N_SAMPLES, "N": N_PADDED, "fn": fn, "fs": FS, "f0": F0, "f1": F1, "sigma": SIGMA,
            "scaling": "LINFREQS", "threads_param": threads, "out": out, "norm": True,
            "l2": "each step writes a 2.4 GB output (> 126 MB L2); no flush"}


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


def algorithmic_bytes(n: int, fn: int, N: int, out_bytes: int = 8, in_bytes: int = 4) -> int:
    # output + input + spectrum read (bins < N/2 + 1)
    return fn * n * out_bytes + in_bytes * n + 8 * (N // 2 + 1)


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


def rel_l2(got, ref) -> float:
    """||got - ref|| / ||ref|| over all given rows (numpy or torch, float64)."""
    g = np.asarray(got).astype(np.complex128).ravel()
    r = np.asarray(ref).astype(np.complex128).ravel()
    d = np.linalg.norm(r)
    return float(np.linalg.norm(g - r) / (d if d > 0 else 1.0))


def cpu_reference_time(x: np.ndarray, scales: np.ndarray, threads: int, runs: int):
    """Times the reference's CPU path (oracle/_ref) on the full workload:
    median wall time of `runs` calls after one warm-up. Returns the median,
    the times and the reference's output."""
    from oracle.oracle import Reference

    ref = Reference()
    out = np.zeros((scales.size, x.size), np.complex64)
    ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
    ts = []
    for _ in range(runs):
        t0 = time.perf_counter()
        ref.cwt(x, scales, SIGMA, FS, threads, True, out=out)
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts), ts, out


def run_reference_arm(args, rank: int) -> None:
    """The reference's own CPU implementation (oracle/_ref: src/fcwt/fcwt.cpp
    with its FFTW build) on the host cores, same workload and config as the
    GPU arm. Loads only the reference build."""
    if rank != 0:
        return
    from oracle.oracle import Reference

    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/libfcwt_ref.so missing"}))
        return
    ref = Reference()
    x = make_signal(1234)
    scales = ref.scales(LINFREQS, FS, F0, F1, FN, fb=SIGMA)  # Scales(Morlet, LINFREQS, ...) of the reference
    threads = THREADS
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
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": plain_config(),
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": threads, "kind": "reference",
                         "sample": f"full workload, {args.steps} timed calls of FCWT::cwt (FFTW 3.3.10 + OpenMP, "
                                   f"{threads} threads, norm on)"},
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
    ap.add_argument("--cpu-runs", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fn", type=int, default=FN,
                    help="number of rows; values other than 3000 are for profiling captures only")
    ap.add_argument("--no-forms", action="store_true", help="skip the other forms (BF16, power, batched, long, grad)")
    ap.add_argument("--out", default="complex64", choices=list(OUT_TYPES),
                    help="output type of the timed transform; values other than complex64 are for profiling "
                         "captures of the other epilogues (no forms then)")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "grad", "long"],
                    help="plain: the 100k x 3000 transform with all forms (default); batched / grad / long: "
                         "only that form, as its own JSON line")
    ap.add_argument("--skip-loop", action="store_true",
                    help="--workload batched: time only the batched plan, not the per-channel loop beside it "
                         "(profiling captures)")
    args = ap.parse_args()
    if args.skip_loop and args.workload != "batched":
        ap.error("--skip-loop applies to --workload batched")
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload != "plain":
        run_form(args)
        return
    if world > 1:
        run_sharded(args, world, rank, local_rank)
        return

    import torch

    torch.cuda.set_device(local_rank)
    import fcwt_b200 as fcwt
    from fcwt_b200 import _lib

    dev = local_rank
    x = make_signal(1234)
    morl = fcwt.Morlet(SIGMA)
    fn = args.fn
    sc = fcwt.Scales(morl, fcwt.FCWT_LINFREQS, FS, F0, F1, fn)
    plan = fcwt.Plan(N_SAMPLES, sc, fb=SIGMA, threads=THREADS, norm=True, device=dev)
    N = 1 << _lib.load().fcwt_find2power(N_SAMPLES)
    xd = torch.from_numpy(x).to(f"cuda:{dev}")
    out = torch.empty((fn, N_SAMPLES), dtype=torch.complex64, device=f"cuda:{dev}")
    out_code, out_shape, out_dtype, out_bytes = OUT_TYPES[args.out]
    out_t = out if args.out == "complex64" else torch.empty((fn, N_SAMPLES) + out_shape, dtype=getattr(torch, out_dtype),
                                                            device=f"cuda:{dev}")
    out_type = getattr(fcwt, out_code)
    stream = torch.cuda.current_stream(dev)
    ctx = plan.ctx

    # warm-up
    for _ in range(args.warmup):
        plan.execute(xd, out_t, out_type=out_type, stream=stream)
    torch.cuda.synchronize(dev)
    ctx.synchronize()

    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.3)
    ctx.profile_enable(True)
    ctx.profile_read()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.execute(xd, out_t, out_type=out_type, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_total = e0.elapsed_time(e1)
    eng_ms, eng_n, kernels = ctx.profile_read()
    ctx.profile_enable(False)
    ctx.synchronize()
    clocks = sampler.stop()
    eng_avg = eng_ms / max(eng_n, 1)
    ms_step = ms_total / args.steps
    points = N_SAMPLES * fn
    value = points * args.steps / (ms_total / 1e3)

    # ---- e2e: reference-facing call with host buffers (pinned)
    e2e = None
    if args.e2e_steps > 0:
        xin = torch.from_numpy(x).pin_memory()
        hout = torch.empty((fn, N_SAMPLES), dtype=torch.complex64, pin_memory=True)
        xin_np, hout_np = xin.numpy(), hout.numpy()
        f = fcwt.FCWT(morl, THREADS, False, True, device=dev)
        f.cwt(xin_np, sc, hout_np)  # warm
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            f.cwt(xin_np, sc, hout_np)
        te = time.perf_counter() - t0
        e2e = {"value": points * args.e2e_steps / te, "unit": "points/s",
               "h2d_bytes_per_step": 4 * N_SAMPLES, "d2h_bytes_per_step": 8 * points,
               "ms_per_step": 1e3 * te / args.e2e_steps, "host_buffers": "pinned"}
        del xin, hout

    # complex64 result of the timed plan, for the checks below
    if args.out != "complex64":
        plan.execute(xd, out, stream=stream)
    torch.cuda.synchronize(dev)
    sel = np.arange(0, fn, max(1, fn // 30))
    out_rows = out[torch.from_numpy(sel).to(out.device)].cpu().numpy()

    forms = None
    if not args.no_forms and args.out == "complex64":
        forms = plain_forms(plan, xd, out, sel, out_rows, ms_step, fn, N, stream, args)
        del out
        torch.cuda.empty_cache()
        forms.update(other_forms(args, stream))

    cpu = None
    if not args.no_cpu_baseline:
        from oracle.oracle import Reference

        if Reference.available():
            tmed, ts, ref_out = cpu_reference_time(x, sc.scales, THREADS, args.cpu_runs)
            cpu = {"value": points / tmed, "unit": "points/s", "cores": THREADS, "kind": "reference",
                   "sample": f"full workload, median of {len(ts)} calls of the reference FCWT::cwt "
                             f"(FFTW 3.3.10 + OpenMP, threads={THREADS}, norm on)",
                   "rel_l2_vs_reference": rel_l2(out_rows, ref_out[sel]), "rel_l2_rows": int(sel.size)}
            del ref_out
        else:
            cpu = {"value": None, "unit": "points/s", "cores": 0, "kind": "reference",
                   "sample": "reference build missing"}

    peak, peak_kind = load_peaks()
    st = plan.stats()
    kname = ("k_row_tc" if st["tensor_core_rows"] == st["rows"] else
             "k_row_engine" if st["tensor_core_rows"] == 0 else "k_row_tc + k_row_engine")
    # DRAM bytes of one launch of the row kernel (read + write), from the ncu
    # capture summarised in profiles/ (same workload); per launch like `achieved`
    traffic = TRAFFIC_PER_LAUNCH.get(args.out) if (fn == FN and kname == "k_row_tc") else None
    algo = algorithmic_bytes(N_SAMPLES, fn, N, out_bytes)
    achieved = algo / (eng_avg / 1e3) / 1e9
    line = {
        "metric": "scalogram points/s", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": plain_config(fn, args.out),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": kname, "kernel_ms": eng_avg, "algorithmic_bytes": algo},
        "forms": forms,
        "hbm_gbs_step": algo / (ms_step / 1e3) / 1e9,
        "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": kernels,
    }
    print(json.dumps(line))


def plain_forms(plan, xd, out, sel, out_rows, ms_step, fn, N, stream, args) -> dict:
    """BF16 and |W|^2 outputs of the 100k x 3000 workload (same plan), and the
    complex64 result's error against the float64 oracle on sampled rows."""
    import torch

    import fcwt_b200 as fcwt
    from oracle.oracle import Restatement

    points = N_SAMPLES * fn
    dev = out.device
    tsel = torch.from_numpy(sel).to(dev)
    x = xd.cpu().numpy()
    fp64 = Restatement().cwt_fp64(x, plan.scales, SIGMA, THREADS, True, rows=sel)
    forms = {"complex64_out": {"rel_l2_vs_fp64": rel_l2(out_rows, fp64), "error_rows": int(sel.size)}}

    outb = torch.empty((fn, N_SAMPLES, 2), dtype=torch.bfloat16, device=dev)
    ms_b = _timed(lambda: plan.execute(xd, outb, out_type=fcwt.FCWT_OUT_BF16, stream=stream), args.steps,
                  args.warmup, stream)
    got = torch.complex(outb[tsel, :, 0].double(), outb[tsel, :, 1].double()).cpu().numpy()
    forms["bf16_out"] = {"value": points / (ms_b / 1e3), "unit": "points/s", "ms_per_step": ms_b,
                         "speedup_vs_complex64": ms_step / ms_b, "rel_l2_vs_fp64": rel_l2(got, fp64),
                         "rel_l2_vs_complex64": rel_l2(got, out_rows),
                         "algorithmic_bytes": algorithmic_bytes(N_SAMPLES, fn, N, 4), "error_rows": int(sel.size)}
    del outb
    # fused |W|^2 epilogue (float32 scalogram)
    outp = torch.empty((fn, N_SAMPLES), dtype=torch.float32, device=dev)
    ms_p = _timed(lambda: plan.execute(xd, outp, out_type=fcwt.FCWT_OUT_POWER, stream=stream), args.steps,
                  args.warmup, stream)
    pw = outp[tsel].double().cpu().numpy()
    forms["power_out"] = {"value": points / (ms_p / 1e3), "unit": "points/s", "ms_per_step": ms_p,
                          "speedup_vs_complex64": ms_step / ms_p,
                          "rel_l2_vs_fp64_abs2": rel_l2(pw, np.abs(fp64) ** 2)}
    del outp
    # fused decimation: every 16th sample of every row (the transform skips the other columns)
    D = 16
    pd = fcwt.Plan(N_SAMPLES, plan.scales, fb=SIGMA, threads=THREADS, norm=True, time_stride=D)
    outd = torch.empty(pd.out_shape, dtype=torch.complex64, device=dev)
    ms_d = _timed(lambda: pd.execute(xd, outd, stream=stream), args.steps, args.warmup, stream)
    gd = outd[tsel].cpu().numpy()
    forms["decimated_t16"] = {"value": fn * pd.out_shape[1] / (ms_d / 1e3), "unit": "output points/s",
                              "ms_per_step": ms_d, "speedup_vs_complex64": ms_step / ms_d,
                              "output_shape": list(pd.out_shape),
                              "rel_l2_vs_full_transform": rel_l2(gd, out_rows[:, ::D]),
                              "rel_l2_vs_fp64": rel_l2(gd, fp64[:, ::D])}
    del outd
    pd.close()
    return forms


# ----------------------------------------------------------------- other forms
# Single-GPU workloads of the batched, differentiable and reduced-precision
# forms. The default run puts each into `forms`; --workload prints one alone.

def _timed(fn_step, steps: int, warmup: int, stream) -> float:
    import torch

    for _ in range(warmup):
        fn_step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn_step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _pink_bursts(rng, n: int, fs: float) -> np.ndarray:
    """Pink (1/f) noise shaped in the frequency domain plus bursts of 5-200 Hz
    sinusoids at random onsets and durations; unit RMS."""
    w = rng.standard_normal(n)
    W = np.fft.rfft(w)
    f = np.fft.rfftfreq(n, 1.0 / fs)
    W[1:] /= np.sqrt(f[1:])
    W[0] = 0
    x = np.fft.irfft(W, n)
    x /= np.std(x) + 1e-30
    t = np.arange(n) / fs
    for _ in range(int(rng.integers(2, 8))):
        f0 = rng.uniform(5, 200)
        a = int(rng.integers(0, n))
        d = int(rng.integers(n // 50 + 1, n // 5 + 2))
        x[a:a + d] += 2.0 * np.sin(2 * np.pi * f0 * t[a:a + d] + rng.uniform(0, 2 * np.pi))
    return (x / np.sqrt(np.mean(x * x))).astype(np.float32)


def batched_workload():
    """384 real channels, lengths U[20000, 200000] at 30 kHz (pink noise plus
    bursts), Morlet sigma 6, per-channel LOGSCALES grids of U[64, 256]
    frequencies in 1-5000 Hz. Returns (signals, lengths, row counts)."""
    rng = np.random.default_rng(2024)
    C = 384
    ns = [int(v) for v in rng.integers(20000, 200001, C)]
    fns = [int(v) for v in rng.integers(64, 257, C)]
    xs = [_pink_bursts(rng, n, 30000.0) for n in ns]
    return xs, ns, fns


def long_workload() -> np.ndarray:
    """Complex 2^20 signal: independent AR(1) (phi = 0.95) real and imaginary parts."""
    from scipy.signal import lfilter

    rng = np.random.default_rng(5)
    n = 1 << 20
    e = rng.standard_normal((2, n))
    ar = lfilter([1.0], [1.0, -0.95], e, axis=1)
    return (ar[0] + 1j * ar[1]).astype(np.complex64)


def grad_workload():
    """64 x 16384 Gaussian-windowed chirps plus noise at 1 kHz, 128 log-spaced
    centre frequencies 2-200 Hz, seeded target scalogram."""
    rng = np.random.default_rng(7)
    B, n, F = 64, 16384, 128
    t = np.arange(n) / 1000.0
    env = np.exp(-0.5 * ((t - t.mean()) / (0.25 * t.max())) ** 2)
    xs = np.stack([env * np.sin(2 * np.pi * (rng.uniform(2, 50) + rng.uniform(10, 100) * t) * t)
                   + 0.1 * rng.standard_normal(n) for _ in range(B)]).astype(np.float32)
    target = rng.uniform(0, 1e-3, (B, F, n)).astype(np.float32)
    return xs, np.geomspace(2.0, 200.0, F), target


# channels of the batched workload checked against the float64 oracle: the
# shortest, the longest, an odd-length one and three more spread over the list
def _batched_check_channels(ns) -> list[int]:
    order = np.argsort(ns)
    odd = [i for i in range(len(ns)) if ns[i] % 2 == 1][:1]
    picks = [int(order[0]), int(order[-1])] + odd + [len(ns) // 3, len(ns) // 2, (5 * len(ns)) // 6]
    return sorted(set(picks))


def form_batched(steps: int, warmup: int, stream, check: bool = True, loop_baseline: bool = True) -> dict:
    import torch

    import fcwt_b200 as fcwt

    xs_np, ns, fns = batched_workload()
    C = len(ns)
    morl = fcwt.Morlet(6.0)
    grids = [fcwt.Scales(morl, fcwt.FCWT_LOGSCALES, 30000, 1.0, 5000.0, k).scales for k in fns]
    xs = [torch.from_numpy(x).cuda() for x in xs_np]
    outs = [torch.empty((k, n), dtype=torch.complex64, device="cuda") for k, n in zip(fns, ns)]
    points = sum(k * n for k, n in zip(fns, ns))
    plans = [fcwt.Plan(n, g, fb=6.0, threads=1, norm=True) for n, g in zip(ns, grids)]
    bp = fcwt.BatchPlan(ns, grids, fb=6.0, threads=1, norm=True)

    def loop():
        for p, x, o in zip(plans, xs, outs):
            p.execute(x, o, stream=stream)

    def batched():
        bp.execute(xs, outs, graph=True, stream=stream)

    ms_loop = _timed(loop, steps, warmup, stream) if loop_baseline else None
    for p in plans:
        p.close()
    ms_b = _timed(batched, steps, warmup, stream)
    st = bp.stats()
    res = {"metric": "scalogram points/s", "value": points / (ms_b / 1e3), "unit": "points/s",
           "ms_per_step": ms_b,
           "config": {"workload": "batched_384ch: real f32 channels n~U[20000,200000] fs=30000, "
                                  "Morlet sigma=6, LOGSCALES 1-5000 Hz fn~U[64,256], complex64 out, one "
                                  "persistent launch per kernel in a CUDA graph",
                      "channels": C, "points": points, "output_bytes": 8 * points,
                      "rows": st["rows"], "tensor_core_rows": st["tensor_core_rows"]},
           "plain_loop": {"value": points / (ms_loop / 1e3), "ms_per_step": ms_loop,
                          "what": "one plan per channel executed in a loop on one stream"} if ms_loop else None,
           "speedup_vs_plain_loop": ms_loop / ms_b if ms_loop else None,
           "hbm_gbs": 8 * points / (ms_b / 1e3) / 1e9}
    if check:
        from oracle.oracle import Restatement

        o = Restatement()
        num = den = 0.0
        nrows = 0
        chans = _batched_check_channels(ns)
        for c in chans:
            rows = sorted({0, fns[c] // 2, fns[c] - 1})
            ref = o.cwt_fp64(xs_np[c], grids[c], 6.0, 1, True, rows=rows)
            got = outs[c][torch.tensor(rows, device="cuda")].cpu().numpy().astype(np.complex128)
            num += float(np.sum(np.abs(got - ref) ** 2))
            den += float(np.sum(np.abs(ref) ** 2))
            nrows += len(rows)
        res["rel_l2_vs_fp64"] = (num / den) ** 0.5
        res["error_rows"] = f"{nrows} rows of channels {chans}"
    bp.close()
    return res


def form_long(steps: int, warmup: int, stream, check: bool = True) -> dict:
    import torch

    import fcwt_b200 as fcwt

    x = long_workload()
    n, F = x.size, 1024
    sc = fcwt.Scales(fcwt.Morlet(4.0), fcwt.FCWT_LOGSCALES, 200000, 10.0, 80000.0, F)
    plan = fcwt.Plan(n, sc, fb=4.0, threads=1, norm=True, complex_input=True)
    xd = torch.from_numpy(x).cuda()
    out64 = torch.empty((F, n), dtype=torch.complex64, device="cuda")
    ms64 = _timed(lambda: plan.execute(xd, out64, stream=stream), steps, warmup, stream)
    out16 = torch.empty((F, n, 2), dtype=torch.bfloat16, device="cuda")
    ms16 = _timed(lambda: plan.execute(xd, out16, out_type=fcwt.FCWT_OUT_BF16, stream=stream), steps, warmup,
                  stream)
    st = plan.stats()
    points = n * F
    res = {"metric": "scalogram points/s (BF16 output)", "value": points / (ms16 / 1e3), "unit": "points/s",
           "ms_per_step": ms16,
           "config": {"workload": "long_complex_2^20_x_1024: complex f32 AR(1) n=2^20 fs=200000, Morlet "
                                  "sigma=4, LOGSCALES 10 Hz-80 kHz fn=1024, BF16 complex out",
                      "rows": st["rows"], "tensor_core_rows": st["tensor_core_rows"]},
           "complex64_out": {"value": points / (ms64 / 1e3), "ms_per_step": ms64},
           "speedup_vs_complex64": ms64 / ms16,
           "hbm_gbs_bf16": 4 * points / (ms16 / 1e3) / 1e9}
    sel = np.arange(0, F, 64)
    tsel = torch.from_numpy(sel).cuda()
    r64 = out64[tsel].cpu().numpy()
    r16 = torch.complex(out16[tsel, :, 0].double(), out16[tsel, :, 1].double()).cpu().numpy()
    res["rel_l2_bf16_vs_complex64"] = rel_l2(r16, r64)
    if check:
        from oracle.oracle import Restatement

        ref = Restatement().cwt_fp64(x, sc.scales, 4.0, 1, True, rows=sel)
        res["rel_l2_vs_fp64"] = rel_l2(r16, ref)
        res["complex64_out"]["rel_l2_vs_fp64"] = rel_l2(r64, ref)
        res["error_rows"] = int(sel.size)
    del out64, out16
    plan.close()
    return res


def form_grad(steps: int, warmup: int, stream, check: bool = True) -> dict:
    import torch

    from fcwt_b200.autograd import LearnableMorletCWT

    xs, freqs, target_np = grad_workload()
    B, n = xs.shape
    F = freqs.size
    x = torch.from_numpy(xs).cuda().requires_grad_(True)
    layer = LearnableMorletCWT(freqs, 1000.0, sigma=2.0)
    target = torch.from_numpy(target_np).cuda()

    def step():
        x.grad = None
        layer.zero_grad()
        y = layer(x)
        loss = ((y.real ** 2 + y.imag ** 2 - target) ** 2).mean()
        loss.backward()

    def fwd():
        with torch.no_grad():
            layer(x)

    ms_f = _timed(fwd, steps, warmup, stream)
    ms = _timed(step, steps, warmup, stream)
    # the hand-written adjoint alone: backward of a kept forward with a fixed incoming gradient
    y_keep = layer(x)
    g_in = torch.randn(y_keep.shape, dtype=torch.complex64, device="cuda")

    def adj():
        x.grad = None
        layer.zero_grad()
        y_keep.backward(g_in, retain_graph=True)

    ms_adj = _timed(adj, steps, warmup, stream)
    del y_keep, g_in
    # the same loss through the power layer: |W|^2 from the row kernels' power
    # epilogue, backward = recomputed W times 2 dL/dP into the same adjoint
    layer_p = LearnableMorletCWT(freqs, 1000.0, sigma=2.0, power=True)

    def step_power():
        x.grad = None
        layer_p.zero_grad()
        P = layer_p(x)
        loss = ((P - target) ** 2).mean()
        loss.backward()

    ms_p = _timed(step_power, steps, warmup, stream)
    points = B * F * n
    res = {"metric": "scalogram points/s (forward + backward)", "value": points / (ms / 1e3),
           "unit": "points/s", "ms_per_step": ms,
           "config": {"workload": "grad_64x16384x128: batch 64 real f32 n=16384 fs=1000, learnable "
                                  "sigma (2.0) and 128 centre frequencies 2-200 Hz, loss MSE(|W|^2, target)",
                      "batch": B, "n": n, "fn": F},
           "forward_ms": ms_f, "adjoint_ms": ms_adj,
           "note": "step = forward transform + loss + hand-written adjoint (signal, sigma, frequencies); "
                   "adjoint_ms = the backward of a kept forward alone",
           "power_layer": {"value": points / (ms_p / 1e3), "ms_per_step": ms_p, "speedup": ms / ms_p,
                           "what": "the same loss on LearnableMorletCWT(power=True): |W|^2 written by the "
                                   "row kernels, backward recomputes W"}}
    if check:
        from oracle.grad_ref import power_mse, ref_forward

        step()
        torch.cuda.synchronize()
        with torch.no_grad():
            y = layer(x).detach()
        xr = x.detach().double().clone().requires_grad_(True)
        sr = torch.tensor(2.0, dtype=torch.float64, device="cuda", requires_grad=True)
        fr = torch.tensor(freqs, dtype=torch.float64, device="cuda", requires_grad=True)
        yr = ref_forward(xr, sr, fr, 1000.0, True)
        Lr = power_mse(yr, target.double())
        Lr.backward()

        def rel(a, b):
            return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

        res["rel_l2_vs_fp64"] = rel(y.to(torch.complex128), yr.detach())
        res["grad_rel_vs_fp64"] = {"signal": rel(x.grad.double(), xr.grad),
                                   "sigma": abs(float(layer.sigma.grad) - float(sr.grad)) / abs(float(sr.grad)),
                                   "freqs_max": float(torch.max(torch.abs(layer.freqs.grad.cuda() - fr.grad))
                                                      / torch.max(torch.abs(fr.grad)))}
        step_power()
        torch.cuda.synchronize()
        with torch.no_grad():
            P = layer_p(x).detach()
        res["power_layer"]["rel_l2_vs_fp64"] = rel(P.double(), (yr.detach().abs() ** 2))
        res["power_layer"]["grad_rel_vs_fp64"] = {
            "signal": rel(x.grad.double(), xr.grad),
            "sigma": abs(float(layer_p.sigma.grad) - float(sr.grad)) / abs(float(sr.grad)),
            "freqs_max": float(torch.max(torch.abs(layer_p.freqs.grad.cuda() - fr.grad)) / torch.max(torch.abs(fr.grad)))}
        del yr, Lr, xr, y, P
    return res


def other_forms(args, stream) -> dict:
    """The batched, long-signal and differentiable forms, each on its own workload."""
    import torch

    forms = {}
    for name, fn in (("batched_384ch", form_batched), ("long_2e20_bf16", form_long),
                     ("grad_64x16384x128", form_grad)):
        forms[name] = fn(args.steps, args.warmup, stream)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return forms


def run_form(args) -> None:
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    steps, warmup = args.steps, max(args.warmup, 3)
    sampler = ClockSampler(dev)
    fn = {"batched": form_batched, "grad": form_grad, "long": form_long}[args.workload]
    sampler.start()
    res = fn(steps, warmup, stream, loop_baseline=False) if args.skip_loop else fn(steps, warmup, stream)
    clocks = sampler.stop()
    line = {"n_gpus": 1, "steps": steps, "warmup": warmup, "data": "synthetic", "scaling": "weak",
            "vs_baseline": None, "higher_is_better": True, "dtype": "f32"}
    line.update(res)
    line["clocks"] = clocks
    print(json.dumps(line))


# ------------------------------------------------------------- multi-GPU (N > 1)

def sharded_transform(compute=None, device=None):
    """The row-sharded 100k x 3000 transform of this process's rank in the
    current torch.distributed group (cost-balanced contiguous row blocks)."""
    import fcwt_b200 as fcwt
    from fcwt_b200.distributed import ShardedCWT

    sc = fcwt.Scales(fcwt.Morlet(SIGMA), fcwt.FCWT_LINFREQS, FS, F0, F1, FN)
    return ShardedCWT(N_SAMPLES, sc.scales, fb=SIGMA, threads=THREADS, norm=True, compute=compute, device=device)


def run_sharded(args, world: int, rank: int, local_rank: int) -> None:
    """One 100k x 3000 transform split by rows over `world` GPUs."""
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device(f"cuda:{local_rank}"))
    dev = local_rank
    sh = sharded_transform(device=dev)
    rb, re_ = sh.rows
    x_src = torch.from_numpy(make_signal(1234)).cuda(dev)
    xd = torch.empty(N_SAMPLES, dtype=torch.float32, device=f"cuda:{dev}")
    out = torch.empty((re_ - rb, N_SAMPLES), dtype=torch.complex64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)

    def step():
        if rank == 0:
            xd.copy_(x_src)
        sh.broadcast_signal(xd, src=0)
        if re_ > rb:
            sh.plan.execute(xd, out, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ctx = sh.plan.ctx
    ctx.profile_enable(True)
    ctx.profile_read()
    dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dist.barrier()
    ms_total = e0.elapsed_time(e1)
    eng_ms, eng_n, kernels = ctx.profile_read()
    ctx.profile_enable(False)
    clocks = sampler.stop() if sampler else None
    t = torch.tensor([ms_total, eng_ms / max(eng_n, 1), float(kernels)], device=f"cuda:{dev}", dtype=torch.float64)
    per_rank = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(per_rank, t)
    ms_total = max(float(p[0]) for p in per_rank)

    # gather of the shards to rank 0 (outside the timed region)
    torch.cuda.synchronize(dev)
    dist.barrier()
    g0 = time.perf_counter()
    full = sh.gather(out, dst=0)
    torch.cuda.synchronize(dev)
    dist.barrier()
    gather_ms = 1e3 * (time.perf_counter() - g0)
    del full

    # e2e: host signal in (pinned) on rank 0, broadcast, row block, block to pinned host memory per rank
    hx = torch.from_numpy(make_signal(1234)).pin_memory()
    hout = torch.empty((re_ - rb, N_SAMPLES), dtype=torch.complex64, pin_memory=True)

    def e2e_step():
        if rank == 0:
            xd.copy_(hx, non_blocking=True)
        sh.broadcast_signal(xd, src=0)
        if re_ > rb:
            sh.plan.execute(xd, out, stream=stream)
            hout.copy_(out, non_blocking=True)
        torch.cuda.synchronize(dev)

    e2e_step()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(max(args.e2e_steps, 1)):
        e2e_step()
    te = time.perf_counter() - t0
    tt = torch.tensor([te], device=f"cuda:{dev}", dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    te = float(tt[0])
    e2e_steps = max(args.e2e_steps, 1)
    sh.close()
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return
    points = N_SAMPLES * FN
    peak, peak_kind = load_peaks()
    k0 = float(per_rank[0][1])
    algo0 = algorithmic_bytes(N_SAMPLES, re_ - rb, N_PADDED)
    line = {
        "metric": "scalogram points/s", "value": points * args.steps / (ms_total / 1e3), "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(plain_config(), parallelism=f"row shards x{world}",
                       row_blocks=[list(b) for b in sh.blocks]),
        "ranks": [{"rank": r, "rows": list(sh.blocks[r]), "ms_per_step": float(per_rank[r][0]) / args.steps,
                   "kernel_ms": float(per_rank[r][1])} for r in range(world)],
        "roofline": {"bound": "hbm", "achieved": algo0 / (k0 / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": algo0 / (k0 / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "k_row_tc (rank 0 block)", "kernel_ms": k0, "algorithmic_bytes": algo0},
        "gather": {"ms": gather_ms, "bytes": 8 * points, "what": "row blocks sent point to point (NCCL) "
                                                                  "into their rows of one [fn, n] tensor on rank 0"},
        "e2e": {"value": points * e2e_steps / te, "unit": "points/s", "h2d_bytes_per_step": 4 * N_SAMPLES,
                "d2h_bytes_per_step": 8 * points, "ms_per_step": 1e3 * te / e2e_steps,
                "host_buffers": "pinned; each rank copies its row block to host"},
        "clocks": clocks, "gpu_launches": int(sum(float(p[2]) for p in per_rank)),
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
