"""Benchmark of the batched ComplexF32 transform hot path on B200.

Workload: batched ComplexF32 forward FFTs of length N=4096, 16384 columns per
GPU (the target configuration named for FFTA's batched path; configuration 2
shapes, inputs i.i.d. complex normal from a seed).  One step is one forward
transform of the whole batch.  Inputs (512 MiB) and outputs (512 MiB) are each
larger than the 126 MB L2, so no flush is needed between steps.

  value     GFLOP/s (5 N log2 N per transform) over all ranks, inputs resident in HBM
  e2e       the same metric through the C ABI's host-array entry point
            (fb_execute_host) from pinned host memory: H2D + transform + D2H
  roofline  achieved HBM GB/s of the line kernel (2 N B sizeof(C) algorithmic
            bytes per launch / CUDA-event launch time) against the measured
            copy bandwidth in MEASURED_PEAKS.json
  cpu_baseline  the oracle (C++ restatement of FFTA's algorithm) on the host's
            cores over a bounded sample of the same workload

`--impl reference` times FFTA's algorithm on the host cores (the oracle, as
FFTA itself -- Julia -- is not installed) on the same metric.
Multi-GPU: one process per GPU (torchrun), each transforming its own 16384
columns (weak scaling, no collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ffta.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N = 4096
BATCH = 16384
ES = 8  # bytes per ComplexF32
# Other configurations, timed after the headline and reported under "extra":
# (label, dtype, transform dims (Julia order), batch, region)
EXTRA = [
    ("c64_n1024_b1", "c64", (1024,), 1),
    ("c32_n4096_b4096", "c32", (4096,), 4096),
    ("c64_n4096_b4096", "c64", (4096,), 4096),
    ("c32_n19683_b852", "c32", (19683,), 852),
    ("c64_n19683_b852", "c64", (19683,), 852),
    ("c32_n27648_b606", "c32", (27648,), 606),
    ("c64_n27648_b606", "c64", (27648,), 606),
    ("c32_n1048576_b16", "c32", (2 ** 20,), 16),
    ("c64_n1048576_b16", "c64", (2 ** 20,), 16),
    ("c32_n1009_b64", "c32", (1009,), 64),
    ("c32_n65537_b16", "c32", (65537,), 16),
    ("c32_n1000003_b1", "c32", (1000003,), 1),
    ("c32_n1049344_b4", "c32", (2 ** 8 * 4099,), 4),
    ("c32_2d_4096x4096", "c32", (4096, 4096), 1),
    ("c32_2d_2187x2048", "c32", (2187, 2048), 1),
    ("c32_2d_1000x1000", "c32", (1000, 1000), 1),
]
# Workloads timed only on request (--workload), for profiling captures of
# kernels the configurations above do not reach: the generic line kernel (a
# length without a specialised kernel), the half-length real kernel, and the
# opt-in tensor-copy tile feed.  (label, kind, dims, batch, plan flags name)
PROFILE_ONLY = [
    ("c32_n7168_b4096", "c32", (7168,), 4096, None),
    ("f32_rfft_n4096_b8192", "r32", (4096,), 8192, None),
    ("c32_n1048576_b16_tma", "c32", (2 ** 20,), 16, "FB_FLAG_TMA"),
]


SPEC_HBM_GBS = 8000.0  # B200 HBM3e specification, GB/s

# DRAM traffic of one launch of the headline kernel (fast_direct_kernel, C32
# N=4096): dram__bytes_read.sum + dram__bytes_write.sum from an ncu capture of
# three back-to-back launches at batch 4096 (inputs and outputs of 134 MB,
# each larger than L2) with --cache-control none, taken from the third
# launch, so that the write-back of an earlier launch's output still held in
# L2 is counted like the steady state of the timed loop.  Traffic grows with
# the columns, so the bench scales it by its batch / 4096.
HEADLINE_TRAFFIC = (4096, 132.317952e6 + 132.321536e6,
                    "ncu dram__bytes_read.sum + dram__bytes_write.sum, third of three "
                    "back-to-back batch-4096 launches (--cache-control none)")


def flops(n, b):
    return 5.0 * n * np.log2(n) * b


def spot_rel_l2(x, y, dims, max_cols=3):
    """rel-L2 of a device result against the FP64 oracle: up to `max_cols`
    transforms of the batch (first, middle, last).  x, y: torch tensors shaped
    (batch, reversed dims), i.e. Julia's column-major (dims..., batch)."""
    import oracle
    b = x.shape[0]
    cols = sorted({0, b // 2, b - 1})[:max_cols]
    xs = x[cols].cpu().numpy().astype(np.complex128)
    ys = y[cols].cpu().numpy().astype(np.complex128)
    nthr = os.cpu_count() or 1
    if len(dims) == 1:
        ref = oracle.fft_batched(xs, -1, nthreads=nthr)
    else:
        ref = np.stack([oracle.fft(np.asfortranarray(v.T), nthreads=nthr).T for v in xs])
    return float(np.linalg.norm(ys - ref) / np.linalg.norm(ref))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def cpu_baseline(n, sample_cols, nthreads, direction=-1):
    """Time the oracle (FFTA's algorithm restated in C++) on host cores."""
    import oracle
    rng = np.random.default_rng(7)
    x = (rng.standard_normal((sample_cols, n)) + 1j * rng.standard_normal((sample_cols, n))
         ).astype(np.complex64)
    oracle.fft_batched(x[:min(8, sample_cols)], direction, nthreads=1)  # warm
    t0 = time.perf_counter()
    oracle.fft_batched(x, direction, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return flops(n, sample_cols) / dt / 1e9, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    sample = 1024  # columns per step: a bounded sample of the 16384-column batch
    for _ in range(args.warmup):
        cpu_baseline(N, sample, nthreads)
    times = []
    for _ in range(args.steps):
        _, dt = cpu_baseline(N, sample, nthreads)
        times.append(dt)
    tot = float(np.sum(times))
    value = flops(N, sample) * args.steps / tot / 1e9
    line = {
        "impl": "reference", "metric": "batched FFT GFLOP/s (5 N log2 N), C32 N=4096 x 16384",
        "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched C32 forward FFT N={N}, {sample}-column sample per "
                               f"step of the {BATCH}-column batch", "n": N, "batch": sample},
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": nthreads, "kind": "port",
                         "sample": f"{sample} transforms of N={N} per step, batch split over "
                                   f"{nthreads} threads (FFTA itself is single-threaded)"},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": julia_probe(),
    }
    print(json.dumps(line))
    return 0


def julia_probe():
    """Whether FFTA.jl itself could be timed on this host: a `julia` binary on
    PATH and FFTA's sources.  The sources of the reference are not shipped with
    this repository, so the reference arm times the C++ restatement of FFTA's
    algorithm (oracle/ffta_oracle.cpp) either way; the probe's answer is
    recorded in the line."""
    import shutil
    jl = shutil.which("julia")
    if jl is None:
        return ("julia: not found on PATH on this host, so FFTA.jl cannot run here; the "
                "reference arm times the C++ restatement of FFTA's algorithm "
                "(oracle/ffta_oracle.cpp)")
    try:
        ver = subprocess.run([jl, "--version"], capture_output=True, text=True,
                             timeout=60).stdout.strip()
    except (OSError, subprocess.TimeoutExpired) as e:
        ver = f"unusable ({e})"
    return (f"julia found at {jl} ({ver}), but FFTA.jl's sources are not present on this "
            "host; the reference arm times the C++ restatement of FFTA's algorithm "
            "(oracle/ffta_oracle.cpp)")


def launch_command(gpus, argv, port=None, script=None):
    """torchrun command that re-runs this script (or `script`) with one
    process per GPU, rendezvous on 127.0.0.1."""
    port = port or 29500 + (os.getpid() % 1000)
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr", "127.0.0.1",
            "--master-port", str(port), script or os.path.abspath(__file__)] + list(argv)


def maybe_launch(gpus, argv):
    """`bench.py --gpus N` started without torchrun (no WORLD_SIZE in the
    environment) starts its N ranks itself; returns their exit code, or None
    when this process is already a rank (or N is 1)."""
    if gpus <= 1 or "WORLD_SIZE" in os.environ:
        return None
    return subprocess.run(["timeout", "-k", "60", "1800"] + launch_command(gpus, argv)).returncode


def reference_benchmark_sizes():
    """The size categories of FFTA's own benchmark suite
    (benchmark/common_defs.jl): odd powers of two 2^1..2^19, even powers
    2^2..2^20, powers of three 3^1..3^9, the cumulative products of
    3, 4, 5, 5, 7, 11, and the primes nearest to 20 log-spaced points between
    2 and 20000 (duplicates dropped).  Returns {n: category}."""
    def is_prime(v):
        if v < 2:
            return False
        f = 2
        while f * f <= v:
            if v % f == 0:
                return False
            f += 1
        return True
    cats = {}
    for i in range(1, 20, 2):
        cats[2 ** i] = "odd_power_of_2"
    for i in range(2, 21, 2):
        cats[2 ** i] = "even_power_of_2"
    for i in range(1, 10):
        cats[3 ** i] = "power_of_3"
    c = 1
    for f in (3, 4, 5, 5, 7, 11):
        c *= f
        cats[c] = "composite"
    primes = [v for v in range(2, 20001) if is_prime(v)]
    chosen = []
    for k in range(20):
        target = np.exp(np.log(2.0) + (np.log(20000.0) - np.log(2.0)) * k / 19)
        best = min(primes, key=lambda q: abs(q - target))
        if best not in chosen:
            chosen.append(best)
    for q in chosen:
        cats[q] = "prime"
    return dict(sorted(cats.items()))


def run_profile_case(case, args, dev):
    """One PROFILE_ONLY workload: warm-up, then `steps` timed steps (CUDA
    events), a rel-L2 spot check against the FP64 oracle, one JSON line."""
    import torch
    import ffta_b200 as F
    import oracle
    label, kind, dims, batch, flag = case
    flags = getattr(F, flag) if flag else 0
    n = dims[0]
    g = torch.Generator(device=dev).manual_seed(7)
    if kind == "r32":
        x = torch.randn(batch, n, device=dev, generator=g)
        p = F.plan_rfft(x.T, 1)
        alg = batch * (4.0 * n + 8.0 * (n // 2 + 1))
        fl = flops(n, batch) / 2
    else:
        x = torch.randn(batch, n, dtype=torch.complex64, device=dev, generator=g)
        p = F.plan_fft(x.T, 1, _flags=flags)
        alg = 2.0 * n * batch * 8
        fl = flops(n, batch)
    y = p * x.T
    for _ in range(args.warmup):
        y = p * x.T
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        y = p * x.T
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    cols = [0, batch - 1]
    xc = x[cols].cpu().numpy().astype(np.complex128)
    ref = oracle.fft_batched(xc, -1, nthreads=os.cpu_count() or 1)
    if kind == "r32":
        ref = ref[:, : n // 2 + 1]
    got = y.T[cols].cpu().numpy()
    print(json.dumps({"workload": label, "ms": ms, "GB/s": alg / (ms * 1e-3) / 1e9,
                      "GFLOP/s": fl / (ms * 1e-3) / 1e9,
                      "rel_l2_vs_fp64_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                      "schedule": p.describe((n, batch)) if kind == "r32" else p.describe(x.T)}))
    return 0


def run_size_sweep(dev, stream):
    """FFTA's own benchmark (benchmark/bench_ffta.jl): one ComplexF64 fft and
    one Float64 rfft of each size category, median time per call; here per
    call through the Python mirror on device-resident data (CUDA events
    around each call, so the host's call overhead counts when it exceeds the
    kernel), with the oracle's single-threaded CPU time of the same complex
    transform beside it and rel-L2 against the FP64 oracle."""
    import oracle
    import torch

    import ffta_b200 as F
    sweep_out = []
    gsw = torch.Generator(device=dev).manual_seed(9)
    for n, cat in reference_benchmark_sizes().items():
        xc = torch.randn(n, dtype=torch.complex128, device=dev, generator=gsw)
        pc = F.plan_fft(xc, 1)
        yc = pc * xc
        ts = []
        for it in range(23):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            F.mul_(yc, pc, xc)
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= 3:
                ts.append(e0.elapsed_time(e1))
        xh = xc.cpu().numpy()[None, :]
        ref = oracle.fft_batched(xh, -1)[0]
        frel = float(np.linalg.norm(yc.cpu().numpy() - ref) / np.linalg.norm(ref))
        cpu_ts, t_end = [], time.perf_counter() + 0.2
        while time.perf_counter() < t_end or not cpu_ts:
            t0 = time.perf_counter()
            oracle.fft_batched(xh, -1)
            cpu_ts.append(time.perf_counter() - t0)
        xr = torch.randn(n, dtype=torch.float64, device=dev, generator=gsw)
        pr = F.plan_rfft(xr, 1)
        yr = pr * xr
        rts = []
        for it in range(23):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            yr = pr * xr
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= 3:
                rts.append(e0.elapsed_time(e1))
        rref = oracle.fft_batched(xr.cpu().numpy().astype(np.complex128)[None, :], -1)[0]
        rref = rref[: n // 2 + 1]
        rrel = float(np.linalg.norm(yr.cpu().numpy() - rref) / np.linalg.norm(rref))
        fms = float(np.median(ts))
        sweep_out.append({
            "size": n, "category": cat,
            "fft_c64_median_ms": fms, "fft_ns_per_element": fms * 1e6 / n,
            "fft_rel_l2_vs_fp64_oracle": frel,
            "cpu_oracle_1thread_median_ms": float(np.median(cpu_ts)) * 1e3,
            "rfft_f64_median_ms": float(np.median(rts)),
            "rfft_rel_l2_vs_fp64_oracle": rrel})
        del xc, yc, pc, xr, yr, pr
    return sweep_out


def main():
    global BATCH
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extra", action="store_true", help="skip the other batched sizes")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--batch", type=int, default=BATCH,
                    help="columns per GPU (smaller for profiling captures)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving comparison")
    ap.add_argument("--no-serving-config5", action="store_true",
                    help="skip configuration 5 at its stated scale (100k requests, batch "
                         "1..512, lengths 64..2^20, 100 GB budget; about five minutes)")
    ap.add_argument("--tensor-stage", action="store_true",
                    help="time the main workload with the split-BF16 tensor-core radix-16 "
                         "stage (ComplexF32 programs that start with 16)")
    ap.add_argument("--workload", default=None,
                    help="time one of the `extra` configurations instead of the headline "
                         "(for profiling captures): " +
                         ", ".join(e[0] for e in EXTRA + PROFILE_ONLY))
    args = ap.parse_args()
    rc = maybe_launch(args.gpus, sys.argv[1:])
    if rc is not None:
        return rc
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(args.warmup, 3)
    BATCH = args.batch

    import torch
    import torch.distributed as dist
    import ffta_b200 as F

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    from ffta_b200 import sharding

    def max_over_ranks(v):
        return sharding.max_over_ranks(v, dev)

    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    label, kind, dims, batch = "headline", "c32", (N,), BATCH
    if args.workload:
        prof = [e for e in PROFILE_ONLY if e[0] == args.workload]
        if prof:
            return run_profile_case(prof[0], args, dev)
        sel = [e for e in EXTRA if e[0] == args.workload]
        if not sel:
            raise SystemExit(f"unknown workload {args.workload}")
        label, kind, dims, batch = sel[0]
    es = 8 if kind == "c32" else 16
    rdt = torch.float32 if kind == "c32" else torch.float64
    # Julia's column-major (dims..., batch) array = torch row-major (batch, reversed dims)
    shape = (batch,) + tuple(reversed(dims))
    x = torch.complex(torch.randn(shape, device=dev, generator=g, dtype=rdt),
                      torch.randn(shape, device=dev, generator=g, dtype=rdt))
    y = torch.empty_like(x)
    perm = tuple(range(x.ndim - 1, -1, -1))
    xt, yt = x.permute(perm), y.permute(perm)
    flags = F.FB_FLAG_TENSOR_STAGE if args.tensor_stage else 0
    p = F.plan_fft(xt, tuple(range(1, len(dims) + 1)), _flags=flags)
    n_tot = int(np.prod(dims))
    stream = torch.cuda.current_stream(dev)

    def step():
        F.mul_(yt, p, xt)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches_per_step = p.describe(xt).count("(")  # one line-kernel launch per pass
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # keep the GPU busy with the same step for ~1 s so that the 100 ms clock
        # samples cover the load, then time exactly K steps inside the same window
        t_soak = time.perf_counter()
        while time.perf_counter() - t_soak < 1.0:
            for _ in range(20):
                step()
            torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(ms)
    total_flops = flops(n_tot, batch) * world
    value = total_flops / (ms_max * 1e-3) / 1e9
    alg_bytes = 2.0 * n_tot * batch * es
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    peak, peak_kind = peaks()

    # accuracy spot check of this run against the FP64 oracle on a few columns
    rel = spot_rel_l2(x, y, dims)

    # e2e: through the C ABI with host buffers (pinned), copies inside the timed region
    hx = x.cpu().pin_memory()
    hy = torch.empty_like(hx).pin_memory()
    hxn, hyn = hx.numpy(), hy.numpy()
    ph = F.plan_fft(hxn.T, tuple(range(1, len(dims) + 1)), _flags=flags)

    def e2e_step():
        F.mul_(hyn.T, ph, hxn.T)

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(e2e_steps):
        e2e_step()
    e2e_dt = (time.perf_counter() - t0) / e2e_steps
    e2e_dt = max_over_ranks(e2e_dt)
    e2e_value = total_flops / e2e_dt / 1e9

    extra = {}
    if not args.no_extra and rank == 0 and not args.workload:
        for (elabel, ekind, edims, b2) in EXTRA:
            label_, kind_, dims_ = elabel, ekind, edims
            ees = 8 if kind_ == "c32" else 16
            erdt = torch.float32 if kind_ == "c32" else torch.float64
            # row-major torch (b, dims reversed) = Julia column-major (dims..., b)
            eshape = (b2,) + tuple(reversed(dims_))
            xe = torch.complex(torch.randn(eshape, device=dev, dtype=erdt),
                               torch.randn(eshape, device=dev, dtype=erdt))
            ye = torch.empty_like(xe)
            perm = tuple(range(xe.ndim - 1, -1, -1))
            xj, yj = xe.permute(perm), ye.permute(perm)
            pe = F.plan_fft(xj, tuple(range(1, len(dims_) + 1)))
            for _ in range(3):
                F.mul_(yj, pe, xj)
            reps = 10
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                F.mul_(yj, pe, xj)
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / reps
            en = int(np.prod(dims_))
            fl = 5.0 * en * np.log2(en) * b2
            gbs = 2.0 * en * b2 * ees / (t * 1e-3) / 1e9
            extra[label_] = {
                "ms": t, "GFLOP/s": fl / (t * 1e-3) / 1e9, "GB/s": gbs,
                "frac_of_hbm": gbs / peaks()[0], "frac_of_spec_8tbs": gbs / SPEC_HBM_GBS,
                "rel_l2_vs_fp64_oracle": spot_rel_l2(xe, ye, dims_),
                "schedule": pe.describe(xj)}
            del xe, ye, pe, xj, yj

    # configuration 4: 2-D ComplexF32 with the plain FP32 path and with the
    # split-BF16 tensor-core radix-16 stage, rel-L2 vs the FP64 oracle for each
    precision = {}
    if not args.no_extra and rank == 0 and not args.workload:
        import oracle
        for plabel, pdims in (("c32_2d_4096x4096", (4096, 4096)), ("c32_2d_2187x2048", (2187, 2048)),
                              ("c32_2d_1000x1000", (1000, 1000))):
            gen = torch.Generator(device=dev).manual_seed(4)
            xr = torch.complex(torch.randn(tuple(reversed(pdims)), device=dev, generator=gen),
                               torch.randn(tuple(reversed(pdims)), device=dev, generator=gen))
            xj = xr.permute(1, 0)
            yj = torch.empty_like(xr).permute(1, 0)
            ref = oracle.fft_nd(xj.cpu().numpy().astype(np.complex128), [1, 2], -1, prec="f64",
                                nthreads=os.cpu_count() or 1)
            row = {}
            for name, fl in (("fp32", 0), ("tensor_stage", F.FB_FLAG_TENSOR_STAGE)):
                pp = F.plan_fft(xj, (1, 2), _flags=fl)
                for _ in range(3):
                    F.mul_(yj, pp, xj)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(10):
                    F.mul_(yj, pp, xj)
                e1.record(stream)
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / 10
                y4 = yj.cpu().numpy()
                en = int(np.prod(pdims))
                row[name] = {"ms": t, "GB/s": 2.0 * en * 8 / (t * 1e-3) / 1e9,
                             "rel_l2_vs_fp64_oracle": float(np.linalg.norm(y4 - ref) /
                                                            np.linalg.norm(ref)),
                             "tensor_core_passes": pp.describe(xj).count("<tc>"),
                             "schedule": pp.describe(xj)}
            precision[plabel] = row
            del xr, xj, yj

    # real transforms: rfft of Float32 N=4096 x 16384 (FFTA's half-length
    # algorithm, one kernel); bytes charged: the real input (4 N) and the
    # n/2+1 complex outputs (8 (N/2+1)) per transform
    real_out = {}
    if not args.no_extra and rank == 0 and not args.workload:
        for rlabel, rn, rb in (("f32_rfft_n4096_b16384", 4096, 16384),
                               ("f32_rfft_n2048_b4096", 2048, 4096)):
            gen = torch.Generator(device=dev).manual_seed(6)
            xr = torch.randn(rb, rn, device=dev, generator=gen)
            pr = F.plan_rfft(xr.T, 1)
            yr = pr * xr.T
            for _ in range(3):
                yr = pr * xr.T
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(10):
                yr = pr * xr.T
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 10
            rbytes = rb * (4.0 * rn + 8.0 * (rn // 2 + 1))
            gbs = rbytes / (t * 1e-3) / 1e9
            import oracle
            cols = [0, rb // 2, rb - 1]
            ref = oracle.fft_batched(xr[cols].cpu().numpy().astype(np.complex128), -1,
                                     nthreads=os.cpu_count() or 1)[:, : rn // 2 + 1]
            got = yr.T[cols].cpu().numpy()
            real_out[rlabel] = {
                "ms": t, "GB/s": gbs, "frac_of_hbm": gbs / peaks()[0],
                "frac_of_spec_8tbs": gbs / SPEC_HBM_GBS,
                "GFLOP/s": flops(rn, rb) / 2 / (t * 1e-3) / 1e9,
                "rel_l2_vs_fp64_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                "schedule": pr.describe((rn, rb))}
            del xr, yr, pr

    sweep_out = []
    if not args.no_extra and rank == 0 and not args.workload:
        sweep_out = run_size_sweep(dev, stream)

    serving_out = None
    if rank == 0 and world == 1 and not args.no_serving and not args.workload:
        from ffta_b200 import serving as S
        serving_out = {}
        for name, kw in (("config5_bounded", dict(count=300, rates=(1e3, 1e4, 1e5, 0.0),
                                                   n_max=2 ** 20, batch_max=512,
                                                   max_elems=1 << 21)),
                         ("small_requests", dict(count=3000, rates=(5e4, 2e5, 1e6, 0.0),
                                                 n_max=4096, batch_max=16,
                                                 max_elems=1 << 16))):
            res = S.compare(**kw)
            sat = res["sweep"][-1]
            serving_out[name] = {
                "saturated_throughput_ratio": sat["throughput_ratio"],
                "saturated_p99_ms": {"batched": sat["batched"]["p99_ms"],
                                     "one_launch_per_request":
                                         sat["one_launch_per_request"]["p99_ms"]},
                **res}
        serving_out["recurring_multipass_graphs"] = S.compare_graphs()
        if not args.no_serving_config5:
            import oracle
            print("bench: serving configuration 5 (100k requests, both paths)",
                  file=sys.stderr, flush=True)
            c5 = S.compare_config5(count=100000, prefix=10000, prefix_rates=(1000.0, 3000.0),
                                   sample=240, reference=oracle.fft_batched)
            sat = c5["sweep"][0]
            serving_out["config5"] = {
                "saturated_throughput_ratio": sat["throughput_ratio"],
                "saturated_p50_p99_ms": {
                    k: [sat[k]["p50_ms"], sat[k]["p99_ms"]]
                    for k in ("batched", "one_launch_per_request")},
                **c5}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        sample = BATCH  # the whole batch: about 10-30 CPU-seconds on a host of 8-32 cores
        v, dt = cpu_baseline(N, sample, nthreads)
        v1, dt1 = cpu_baseline(N, 256, 1)
        cpu = {"value": v, "unit": "GFLOP/s", "cores": nthreads, "kind": "port",
               "sample": f"{sample} transforms of C32 N={N} (the whole {BATCH}-column batch), "
                         f"split over {nthreads} threads: {dt:.2f} s wall, "
                         f"{dt * nthreads:.0f} thread-seconds",
               "single_thread": {"value": v1, "unit": "GFLOP/s", "cores": 1,
                                 "sample": f"256 transforms of N={N} on one thread "
                                           f"(FFTA itself is single-threaded), {dt1:.2f} s"}}

    # DRAM bytes per launch of the headline kernel, measured by ncu (see
    # HEADLINE_TRAFFIC) and scaled from its batch to this launch's batch
    traffic, traffic_note = None, None
    if label == "headline" and not args.tensor_stage:
        tb, tbytes, tnote = HEADLINE_TRAFFIC
        traffic = tbytes * batch / tb
        traffic_note = tnote + f"; scaled by {batch}/{tb} columns"
    if rank == 0:
        wl = (f"batched C32 forward FFT, N={N}, {BATCH} contiguous columns per GPU"
              if label == "headline" else f"{label} forward FFT")
        line = {
            "metric": "batched FFT GFLOP/s (5 N log2 N), C32 N=4096 x 16384",
            "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl, "n": list(dims), "batch_per_gpu": batch,
                       "parallelism": f"batch-sharded x{world} (no collective)",
                       "l2": "inputs and outputs (512 MiB each) larger than L2; no flush",
                       "schedule": p.describe(xt)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "frac_of_spec_8tbs": achieved / SPEC_HBM_GBS,
                         "alg_bytes_per_launch": alg_bytes, "traffic": traffic,
                         "traffic_source": traffic_note},
            "hbm_gbs": achieved,
            "rel_l2_vs_fp64_oracle": rel,
            "e2e": {"value": e2e_value, "unit": "GFLOP/s",
                    "h2d_bytes_per_step": int(n_tot * batch * es),
                    "d2h_bytes_per_step": int(n_tot * batch * es),
                    "path": "fb_execute_host from pinned host memory"},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "extra": extra,
            "serving": serving_out,
            "config4_precision": precision or None,
            "real_transforms": real_out or None,
            "reference_size_sweep": sweep_out or None,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
