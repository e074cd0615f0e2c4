"""Benchmark of the FFT hot path on B200.

Workload (the configuration the headline metric is quoted on): 1D real
transforms in FP32 — R2C FORWARD then C2R INVERSE — at N=3000 (2^3*3*5^3) and
N=4096, batch 4096 each.  Input: seeded Gaussian noise (sigma=1) plus three
sinusoids at random bins with amplitudes in [0.1, 10].  One step = the four
launches R2C(3000), C2R(3000), R2C(4096), C2R(4096) over the full batches.

Metric: FFT GFLOP/s with 5*N*log2(N) flops per transform (also for R2C/C2R),
whole job (all ranks).  `value` is timed with inputs resident in HBM and L2
flushed (256 MiB write) between steps; `e2e` goes through the C ABI's aclTensor
entry points with pinned host buffers, H2D of the inputs and D2H of the
round-trip results inside the timed region, streamed in 1024-row chunks so that
the two copy directions and the transforms overlap.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun every rank runs an independent replica (the transforms shard
with no exchange); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZES = (3000, 4096)
BATCH = 4096
E2E_CHUNK = 1024  # rows per chunk of the streamed end-to-end step (256: 981, 512: 1178, 1024: 1211, 4096: 992 GFLOP/s measured)
METRIC = "FFT GFLOP/s (5N*log2N per transform), R2C+C2R round trip"
WORKLOAD = "1D R2C FORWARD + C2R INVERSE, FP32, N=3000 and N=4096, batch 4096 each"


def flops_per_transform(n: int) -> float:
    return 5.0 * n * math.log2(n)


def step_flops() -> float:
    return sum(2 * BATCH * flops_per_transform(n) for n in SIZES)


def algorithmic_bytes(n: int) -> int:
    """One read of the input and one write of the output, per launch (R2C and C2R alike)."""
    return BATCH * (4 * n + 8 * (n // 2 + 1))


def make_signal(n: int, rows: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((rows, n))
    t = np.arange(n)
    for _ in range(3):
        k = rng.integers(1, n // 2, size=(rows, 1))
        a = rng.uniform(0.1, 10.0, size=(rows, 1))
        ph = rng.uniform(0, 2 * np.pi, size=(rows, 1))
        x += a * np.cos(2 * np.pi * k * t / n + ph)
    return x.astype(np.float32)


# ----------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic() -> dict | None:
    path = os.path.join(ROOT, "profiles", "r2c_c2r_roundtrip_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ----------------------------------------------------------------------------------- CPU baseline
def cpu_baseline(budget_s: float = 10.0) -> dict:
    """FP64 host FFT (the oracle port: scipy pocketfft) on a bounded sample of the workload."""
    import scipy.fft as sfft

    cores = os.cpu_count() or 1
    rows = 256
    xs = {n: make_signal(n, rows, 100 + n).astype(np.float64) for n in SIZES}
    t0 = time.perf_counter()
    reps = 0
    while True:
        for n in SIZES:
            X = sfft.rfft(xs[n], axis=-1, workers=cores)
            sfft.irfft(X, n=n, axis=-1, workers=cores)
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or reps >= 2000:
            break
    fl = reps * sum(2 * rows * flops_per_transform(n) for n in SIZES)
    return {"value": fl / el / 1e9, "unit": "GFLOP/s", "cores": cores, "kind": "port",
            "sample": f"{reps} x (rfft+irfft of {rows} rows at N=3000 and N=4096), complex128/float64 "
                      f"scipy.fft workers={cores}, {el:.1f} s"}


# ----------------------------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    # NCCL reduces device tensors; the gloo backend (CPU tests of this plumbing) host tensors
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------------- reference arm
def run_reference(args, world, rank):
    if rank != 0:
        return
    import scipy.fft as sfft

    cores = os.cpu_count() or 1
    rows = 256
    xs = {n: make_signal(n, rows, 100 + n).astype(np.float64) for n in SIZES}

    def one():
        for n in SIZES:
            X = sfft.rfft(xs[n], axis=-1, workers=cores)
            sfft.irfft(X, n=n, axis=-1, workers=cores)

    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    el = time.perf_counter() - t0
    fl = args.steps * sum(2 * rows * flops_per_transform(n) for n in SIZES)
    v = fl / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian + 3 sinusoids)",
        "config": {"workload": WORKLOAD + f"; each step a bounded sample of {rows} rows per length",
                   "batch": rows, "sizes": list(SIZES)},
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": cores, "kind": "port",
                         "sample": f"{rows} rows per length per step; the reference's FFT runs only on an "
                                   f"Ascend NPU, so its CPU stand-in is the FP64 host FFT (scipy pocketfft)"},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------- multi-axis configs
MULTIAXIS = (("2d_2048x2048_b8", [2048, 2048], 8), ("3d_256x256x256_b1", [256, 256, 256], 1))
FORM_NAMES = ("fp32", "fp16x3", "bf16x3")


def multiaxis_measure(sizes, batch: int, form: str, reps: int, flush_l2) -> dict:
    """One C2C plan (FORWARD) over device-resident data: median CUDA-event time of
    `reps` executions with the L2 flushed before each, GFLOP/s, algorithmic-byte
    roofline, and the error of the first transform of the batch against FP64."""
    import torch

    from sip_b200 import fft

    prec = {"fp32": fft.PRECISION_FP32, "fp16x3": fft.PRECISION_FP16X3, "bf16x3": fft.PRECISION_BF16X3}[form]
    g = torch.Generator(device="cuda").manual_seed(31)
    shape = [batch] + list(sizes)
    x = torch.complex(torch.rand(shape, device="cuda", generator=g) * 2 - 1,
                      torch.rand(shape, device="cuda", generator=g) * 2 - 1)
    y = torch.empty_like(x)
    plan = fft.FftPlan(sizes, fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_FORWARD, batch, precision=prec)
    plan(x, y)
    for _ in range(2):
        plan.exec_raw(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        flush_l2(plan.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(plan.stream)
        plan.exec_raw(x.data_ptr(), y.data_ptr())
        e1.record(plan.stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    from oracle import oracle as _oracle  # checker only

    xs = x[:1].cpu().numpy()
    ref = _oracle.c2c(xs, True, ndim=len(sizes))
    ys = y[:1].cpu().numpy()
    n_total = int(np.prod(sizes))
    med = statistics.median(ms)
    peak, _ = measured_peak_hbm()
    nbytes = 16 * n_total * batch
    out = {"ms": med, "GFLOPps": 5.0 * n_total * math.log2(n_total) * batch / (med / 1e3) / 1e9,
           "GBps": nbytes / (med / 1e3) / 1e9, "frac_of_hbm": nbytes / (med / 1e3) / 1e9 / peak,
           "rel_l2": _oracle.rel_l2(ys, ref), "max_abs": _oracle.max_abs(ys, ref),
           "bound": _oracle.tolerance(n_total), "launches": plan.launches(),
           "tensor_core": "tensor-core" in plan.describe()}
    plan.close()
    return out


def config_extras(args, flush_l2) -> dict:
    """The other workload configurations, a few seconds each, for the bench line:
    C3 multi-axis transforms per arithmetic form (with the tensor-core / plain
    ratio), C4 uneven batch, C5 serving at four offered loads per form."""
    ex = {}
    c3 = {}
    for name, sizes, batch in MULTIAXIS:
        per = {}
        for form in FORM_NAMES:
            per[form] = multiaxis_measure(sizes, batch, form, args.extra_reps, flush_l2)
        for form in FORM_NAMES[1:]:
            per[f"{form}_over_fp32"] = per["fp32"]["ms"] / per[form]["ms"]
        c3[name] = per
    ex["c3_multiaxis"] = {"workload": "C2C complex64 FORWARD, uniform[-1,1] inputs; L2 flushed before each of "
                                      f"{args.extra_reps} timed executions; error of the first transform vs FP64",
                          "results": c3}
    ex["c4_uneven"] = dict(uneven_measure(20000, max(3, args.extra_reps // 2), 3), workload="20000 " + UNEVEN_WORKLOAD)
    c5 = {}
    for form in ("fp32", "fp16x3"):
        c5[form] = serving_points(form, True, [1000.0, 5000.0, 20000.0, 50000.0], 0.25, 2000, 4)
    ex["c5_serving"] = {"workload": SERVE_WORKLOAD + "; device-resident request buffers; 4 lanes",
                        "points": c5}
    return ex


# ----------------------------------------------------------------------------------- our arm
def run_ours(args, world, rank, local):
    import ctypes

    import torch

    from sip_b200 import fft

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    fft.load_library()
    stream = torch.cuda.Stream(device=dev)
    R2C, C2R, FWD, INV = fft.ASCEND_FFT_R2C, fft.ASCEND_FFT_C2R, fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE

    plans, bufs = [], []
    host_in, host_out = {}, {}
    for n in SIZES:
        x = make_signal(n, BATCH, seed=1000 * rank + n)
        xd = torch.from_numpy(x).to(dev)
        X = torch.empty((BATCH, n // 2 + 1), dtype=torch.complex64, device=dev)
        y = torch.empty_like(xd)
        f = fft.FftPlan([n], R2C, FWD, BATCH, stream=stream)
        g = fft.FftPlan([n], C2R, INV, BATCH, stream=stream)
        plans.append((n, f, g))
        bufs.append((xd, X, y))
        host_in[n] = torch.from_numpy(x).pin_memory()
        host_out[n] = torch.empty_like(host_in[n]).pin_memory()

    # Tensor descriptors are built once, as a caller of the C ABI would.
    descs = []
    for (n, f, g), (xd, X, y) in zip(plans, bufs):
        descs.append((fft.AclTensor.from_torch(xd), fft.AclTensor.from_torch(X), fft.AclTensor.from_torch(y)))
    lib = fft.load_library()

    def launch_step(events=None):
        i = 0
        for (n, f, g), (ax, aX, ay) in zip(plans, descs):
            if events is not None:
                events[i].record(stream)
            st = lib.asdFftExecR2C(f.handle, ax.ptr, aX.ptr)
            if events is not None:
                events[i + 1].record(stream)
            st2 = lib.asdFftExecC2R(g.handle, aX.ptr, ay.ptr)
            if st or st2:
                raise RuntimeError(f"exec failed: {st} {st2}")
            i += 2
        if events is not None:
            events[i].record(stream)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    flush_read = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush_l2(sync=True, on=None):
        # write a buffer larger than L2, then read another one: the dirty lines
        # of the write are written back here, outside the timed region.  The
        # flush runs on the benchmark stream, so a step's first event is recorded
        # after it completes; without the synchronize the host enqueues the step
        # while the flush still runs, and no launch gap enters the timed region.
        st = on if on is not None else stream
        with torch.cuda.stream(st):
            flush.fill_(1.0)
            flush_read.sum()
        if sync:
            st.synchronize()

    # ---------------- accuracy of the round trip on this data
    with torch.cuda.stream(stream):
        launch_step()
    stream.synchronize()
    acc = {}
    from oracle import oracle as _oracle  # checker only

    for (n, f, g), (xd, X, y) in zip(plans, bufs):
        xr = xd[:256].double().cpu().numpy()
        yr = y[:256].double().cpu().numpy() / n
        acc[str(n)] = {"round_trip_rel_l2": _oracle.rel_l2(yr, xr),
                       "r2c_rel_l2_vs_fp64": _oracle.rel_l2(X[:64].cpu().numpy(), _oracle.r2c(xr[:64], True)),
                       "bound": _oracle.tolerance(n)}

    # ---------------- device-resident timing
    for _ in range(max(3, args.warmup)):
        flush_l2()
        with torch.cuda.stream(stream):
            launch_step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    nlaunch = 2 * len(SIZES)
    step_ms, launch_ms = [], [[] for _ in range(nlaunch)]
    sampler = ClockSampler(local)  # every rank samples its own GPU
    sampler.start()
    time.sleep(0.3)
    # The timed steps carry one event before and one after the four launches:
    # an event recorded between two launches costs about 2-3 us of device time
    # (measured), so the per-launch durations come from a second pass of the
    # same steps with an event between launches.
    for _ in range(args.steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        flush_l2(sync=False)  # L2 flush between timed steps, before the first event
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            launch_step()
            ev[1].record(stream)
        stream.synchronize()
        step_ms.append(ev[0].elapsed_time(ev[1]))
    for _ in range(args.steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(nlaunch + 1)]
        flush_l2(sync=False)
        with torch.cuda.stream(stream):
            launch_step(ev)
        stream.synchronize()
        for i in range(nlaunch):
            launch_ms[i].append(ev[i].elapsed_time(ev[i + 1]))
    clocks = sampler.stop()
    torch.cuda.synchronize()
    total_s = sum(step_ms) / 1e3
    total_s = max_over_ranks(total_s, world)
    flops = step_flops() * args.steps * world
    value = flops / total_s / 1e9

    # roofline of the dominant kernel: the four launches of a step are all the
    # TMA-pipelined row kernel, so its achieved bandwidth is the step's
    # algorithmic bytes over the timed step (inter-launch gaps included)
    peak, peak_kind = measured_peak_hbm()
    alg_bytes = sum(algorithmic_bytes(n) for n in SIZES) * 2  # R2C + C2R per length
    achieved = alg_bytes / (sum(step_ms) / 1e3 / args.steps) / 1e9
    per_launch = {}
    for i, (n, _, _) in enumerate(plans):
        for j, kind in enumerate(("r2c", "c2r")):
            ms = statistics.median(launch_ms[2 * i + j])
            per_launch[f"{kind}_{n}"] = {"ms": ms, "GBps": algorithmic_bytes(n) / (ms / 1e3) / 1e9}
    traffic = profiled_traffic()

    # ---------------- end to end through the C ABI with host buffers
    # A host-resident batch is streamed through the device in chunks of
    # E2E_CHUNK rows: the H2D copy of chunk c+1, the R2C + C2R of chunk c and
    # the D2H copy of chunk c-1 run on three streams (two copy engines and the
    # SMs), so the PCIe transfers in both directions overlap each other and the
    # transforms.  Every input byte goes up and every output byte comes back
    # inside the timed region.
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    nchunk = max(1, BATCH // args.e2e_chunk)
    rows = BATCH // nchunk
    chunks = []  # (n, c0, c1, plan_f, plan_g, descriptors, device buffers)
    chunk_plans = []
    for (n, f, g), (xd, X, y) in zip(plans, bufs):
        fc = fft.FftPlan([n], R2C, FWD, rows, stream=stream)
        gc = fft.FftPlan([n], C2R, INV, rows, stream=stream)
        chunk_plans.append((fc, gc))
        for c in range(nchunk):
            c0, c1 = c * rows, (c + 1) * rows
            d = (fft.AclTensor.from_torch(xd[c0:c1]), fft.AclTensor.from_torch(X[c0:c1]),
                 fft.AclTensor.from_torch(y[c0:c1]))
            chunks.append((n, c0, c1, fc, gc, d, (xd, X, y)))
    e2e_ms = []
    h2d = sum(host_in[n].numel() * 4 for n in SIZES)
    d2h = sum(host_out[n].numel() * 4 for n in SIZES)
    for it in range(args.warmup + args.steps):
        flush_l2()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        for n, c0, c1, fc, gc, (ax, aX, ay), (xd, X, y) in chunks:
            with torch.cuda.stream(s_in):
                xd[c0:c1].copy_(host_in[n][c0:c1], non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(s_in)
            stream.wait_event(ready)
            st = lib.asdFftExecR2C(fc.handle, ax.ptr, aX.ptr)
            st2 = lib.asdFftExecC2R(gc.handle, aX.ptr, ay.ptr)
            if st or st2:
                raise RuntimeError(f"exec failed: {st} {st2}")
            done = torch.cuda.Event()
            done.record(stream)
            s_out.wait_event(done)
            with torch.cuda.stream(s_out):
                host_out[n][c0:c1].copy_(y[c0:c1], non_blocking=True)
        e1.record(s_out)
        s_out.synchronize()
        if it >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    for n in SIZES:  # the streamed round trip returns its input (times n: C2R is unnormalised)
        ref = host_in[n][:8]
        if not torch.allclose(host_out[n][:8] / n, ref, rtol=0, atol=1e-4 * float(ref.abs().max())):
            raise RuntimeError(f"end-to-end round trip of N={n} does not return its input")
    e2e_launches = sum(fc.launches() + gc.launches() for fc, gc in chunk_plans) * nchunk
    for fc, gc in chunk_plans:
        fc.close()
        gc.close()
    e2e_s = max_over_ranks(sum(e2e_ms) / 1e3, world)
    e2e_value = step_flops() * args.steps * world / e2e_s / 1e9

    launches_per_step = sum(f.launches() + g.launches() for _, f, g in plans)
    extras = None
    if world == 1 and not args.no_extras:
        extras = config_extras(args, lambda st: flush_l2(sync=False, on=st))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Gaussian noise + 3 sinusoids, amplitudes U[0.1,10])",
            "config": {"workload": WORKLOAD, "batch": BATCH, "sizes": list(SIZES),
                       "parallelism": f"replicas x{world}", "l2": "flushed between steps (256 MiB write + 256 MiB read)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": (traffic or {}).get("traffic_bytes_per_step"),
                         "traffic_note": (traffic or {}).get("note"),
                         "algorithmic_bytes_per_step": alg_bytes,
                         "kernel": "sipfft::pipelined_rows_kernel<StaticEngine> (R2C and C2R, 4 launches per step; "
                                   "achieved = algorithmic bytes of the step / timed step; per_launch: CUDA events "
                                   "between the launches of a second pass of the same steps, each event adding "
                                   "about 2-3 us)",
                         "per_launch": per_launch},
            "e2e": {"value": e2e_value, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_s / args.steps * 1e3,
                    "pipeline": f"{nchunk} chunks of {rows} rows per length; H2D, R2C + C2R and D2H on three streams",
                    "gpu_launches_per_step": e2e_launches},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "accuracy": acc,
        }
        if extras is not None:
            line.update(extras)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    for d in descs:
        for t in d:
            t.close()
    for _, f, g in plans:
        f.close()
        g.close()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------------------- uneven batch
UNEVEN_WORKLOAD = ("1D C2C complex64 transforms, lengths log-uniform in [64, 65536] snapped to 7-smooth, "
                   "Zipf(1.2) batch per length capped at 512; one persistent launch replayed from a CUDA graph")


def uneven_measure(total: int, steps: int, warmup: int, autotune: bool = False) -> dict:
    """The uneven batch in one persistent, graph-captured launch: per-step time
    (CUDA events on the launching stream), GFLOP/s and algorithmic-byte roofline."""
    import torch

    from sip_b200 import fft, workloads

    groups = workloads.uneven_batch_set(total=total, seed=2024)
    fl, alg_bytes = workloads.uneven_flops_bytes(groups)
    cache = os.path.join(ROOT, "sip_b200", "tune", "b200_c2c_fp32.jsonl")
    if autotune:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        fft.autotune(groups, fft.ASCEND_FFT_FORWARD, cache)
    plan = fft.BatchPlan(groups, fft.ASCEND_FFT_FORWARD, cache if os.path.exists(cache) else None)
    x = torch.randn(plan.total, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(max(3, warmup)):
            plan(x, y, stream=stream)
    stream.synchronize()
    ms = []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            plan(x, y, stream=stream)
            ev[1].record(stream)
        stream.synchronize()
        ms.append(ev[0].elapsed_time(ev[1]))
    plan.close()
    peak, kind = measured_peak_hbm()
    t = sum(ms) / 1e3 / steps
    return {"ms_per_step": t * 1e3, "GFLOPps": fl / t / 1e9, "groups": len(groups), "transforms": total,
            "bytes_in": alg_bytes // 2, "tuned": os.path.exists(cache),
            "roofline": {"bound": "hbm", "achieved": alg_bytes / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg_bytes / t / 1e9 / peak, "peak_source": kind,
                         "algorithmic_bytes_per_step": alg_bytes},
            "launches_per_step": 1, "l2": f"inputs ({alg_bytes // 2 / 1e9:.2f} GB) larger than L2"}


def run_uneven(args, world, rank, local):
    """20 000 1D C2C transforms of uneven lengths in one persistent, graph-captured launch."""
    import torch

    torch.cuda.set_device(local)
    r = uneven_measure(args.uneven_total, args.steps, args.warmup, args.autotune)
    t = max_over_ranks(r["ms_per_step"] / 1e3 * args.steps, world)
    if rank == 0:
        print(json.dumps({
            "metric": "FFT GFLOP/s (5N*log2N per transform), uneven batch", "value": r["GFLOPps"] * world,
            "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "dtype": "f32",
            "data": "synthetic (seeded lengths/batches, randn values)",
            "config": {"workload": f"{args.uneven_total} {UNEVEN_WORKLOAD}", "groups": r["groups"],
                       "transforms": args.uneven_total, "bytes_in": r["bytes_in"], "tuned": r["tuned"]},
            "roofline": r["roofline"], "gpu_launches": args.steps,
        }), flush=True)


# ----------------------------------------------------------------------------------- serving
SERVE_SIZES = (4096, 8192, 16384, 65536)


def serving_points(precision_name: str, device_io: bool, rates, seconds: float, max_requests: int,
                   lanes: int) -> list[dict]:
    """Poisson arrivals into the C++ continuous-batching server at each offered
    load; p50/p99 latency, achieved request rate and throughput per load."""
    import torch

    from sip_b200 import fft, workloads

    classes = [(t, n) for n in SERVE_SIZES for t in (fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_R2C)]
    rows_min, rows_max = 64, 1024
    rng = np.random.default_rng(5)
    pin, pout, keep = [], [], []
    for i, (t, n) in enumerate(classes):
        x = workloads.chirp_noise(n, rows_max, snr_db=float(rng.uniform(0, 20)), seed=500 + i)
        if t == fft.ASCEND_FFT_R2C:
            x = np.ascontiguousarray(x.real.astype(np.float32))
        xt = torch.from_numpy(x)
        ot = torch.empty((rows_max, n if t == fft.ASCEND_FFT_C2C else n // 2 + 1), dtype=torch.complex64)
        if device_io:
            xt, ot = xt.cuda(), ot.cuda()
        else:
            xt, ot = xt.pin_memory(), ot.pin_memory()
        keep += [xt, ot]
        pin.append(xt.data_ptr())
        pout.append(ot.data_ptr())
    precision = {"fp32": fft.PRECISION_FP32, "fp16x3": fft.PRECISION_FP16X3,
                 "bf16x3": fft.PRECISION_BF16X3}[precision_name]
    srv = fft.Server(budget_bytes=32 << 30, lanes=lanes, max_rows=rows_max, device_io=device_io,
                     precision=precision)
    for t, n in classes:
        srv.warm(t, fft.ASCEND_FFT_FORWARD, n)
    # warm-up traffic: allocates each lane's staging buffers
    srv.run_poisson(1e6, 4 * lanes * len(classes), 1, classes, pin, pout, rows_max, rows_max)
    points = []
    for rate in rates:
        count = int(min(max_requests, max(10, rate * seconds)))
        b0 = srv.batches()
        wall, lat, rows, cls = srv.run_poisson(rate, count, 11, classes, pin, pout, rows_min, rows_max)
        ok = lat[lat > 0]
        by = 0
        fl = 0.0
        for r, c in zip(rows, cls):
            t, n = classes[c]
            fl += r * 5.0 * n * math.log2(n)
            by += r * (16 * n if t == fft.ASCEND_FFT_C2C else 4 * n + 8 * (n // 2 + 1))
        points.append({"offered_rps": rate, "requests": count, "completed": int(ok.size),
                       "p50_ms": float(np.percentile(ok, 50) * 1e3), "p99_ms": float(np.percentile(ok, 99) * 1e3),
                       "achieved_rps": count / wall, "GBps": by / wall / 1e9, "GFLOPps": fl / wall / 1e9,
                       "batches": srv.batches() - b0})
    srv.close()
    return points


SERVE_WORKLOAD = ("Poisson arrivals; R2C or C2C FP32, N in {4096, 8192, 16384, 65536}, rows uniform in "
                  "[64, 1024], chirp + noise at SNR U[0,20] dB; 32 GiB admission budget")


def run_serving(args, world, rank, local):
    """Poisson arrivals over a swept offered load into the C++ continuous-batching server."""
    import torch

    torch.cuda.set_device(local)
    points = serving_points(args.precision, args.device_io, [float(r) for r in args.rates.split(",")],
                            args.seconds, args.max_requests, args.lanes)
    if rank == 0:
        print(json.dumps({
            "metric": "serving p50/p99 latency (ms) and throughput vs offered load", "unit": "ms",
            "form": {"fp32": "plain FP32", "fp16x3": "split FP16 hi/lo x3 (tensor-core stages where available)",
                     "bf16x3": "split BF16 hi/lo x3 (tensor-core stages where available)"}[args.precision],
            "io": "device-resident buffers" if args.device_io else "pinned host buffers",
            "config": {"workload": SERVE_WORKLOAD, "lanes": args.lanes, "max_rows": 1024},
            "points": points}), flush=True)


# ----------------------------------------------------------------------------------- one plan
def run_kernel(args, world, rank, local):
    """Times one plan (kind, sizes, batch, direction) on device-resident data: the
    small-case driver of the profiles and the per-config measurements (the
    N=1024 C2C case, the 2D / 3D multi-axis transforms)."""
    import torch

    from sip_b200 import fft

    torch.cuda.set_device(local)
    kind = {"c2c": fft.ASCEND_FFT_C2C, "r2c": fft.ASCEND_FFT_R2C, "c2r": fft.ASCEND_FFT_C2R}[args.kind]
    direction = fft.ASCEND_FFT_INVERSE if args.inverse else fft.ASCEND_FFT_FORWARD
    sizes = [int(v) for v in args.sizes.split(",")]
    b = args.batch
    n_total = int(np.prod(sizes))
    last_h = sizes[-1] // 2 + 1
    half = [b] + sizes[:-1] + [last_h]
    full = [b] + sizes
    g = torch.Generator(device="cuda").manual_seed(7)
    if kind == fft.ASCEND_FFT_C2C:
        x = torch.randn(full, dtype=torch.complex64, device="cuda", generator=g)
        y = torch.empty_like(x)
        nbytes = 16 * n_total * b
    elif kind == fft.ASCEND_FFT_R2C:
        x = torch.randn(full, dtype=torch.float32, device="cuda", generator=g)
        y = torch.empty(half, dtype=torch.complex64, device="cuda")
        nbytes = (4 * n_total + 8 * n_total // sizes[-1] * last_h) * b
    else:
        x = torch.randn(half, dtype=torch.complex64, device="cuda", generator=g)
        y = torch.empty(full, dtype=torch.float32, device="cuda")
        nbytes = (4 * n_total + 8 * n_total // sizes[-1] * last_h) * b
    precision = {"fp32": fft.PRECISION_FP32, "fp16x3": fft.PRECISION_FP16X3,
                 "bf16x3": fft.PRECISION_BF16X3}[args.precision]
    plan = fft.FftPlan(sizes, kind, direction, b, precision=precision)
    plan(x, y)  # through the aclTensor entry point once (shape checks)
    # then back-to-back raw-pointer executions, so host overhead does not
    # open gaps between launches inside the timed region
    reps = max(1, int(args.reps))
    for _ in range(max(1, args.warmup)):
        plan.exec_raw(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(plan.stream)
        for _ in range(reps):
            plan.exec_raw(x.data_ptr(), y.data_ptr())
        e1.record(plan.stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1) / reps)
    med = statistics.median(ms)
    peak, pk = measured_peak_hbm()
    acc = None
    if args.check:
        from oracle import oracle as _oracle  # checker only

        nd = len(sizes)
        xs, ys = x[:1].cpu().numpy(), y[:1].cpu().numpy()
        f = direction == fft.ASCEND_FFT_FORWARD
        ref = (_oracle.c2c(xs, f, ndim=nd) if kind == fft.ASCEND_FFT_C2C else
               _oracle.r2c(xs, f, ndim=nd) if kind == fft.ASCEND_FFT_R2C else
               _oracle.c2r(xs, sizes[-1], f, ndim=nd))
        acc = {"rel_l2": _oracle.rel_l2(ys, ref), "bound": _oracle.tolerance(n_total)}
    if rank == 0:
        print(json.dumps({
            "workload": f"{args.kind} sizes={sizes} batch={b} {'inverse' if args.inverse else 'forward'}",
            "precision": args.precision,
            "ms_median": med, "ms_min": min(ms), "GBps": nbytes / (med / 1e3) / 1e9,
            "frac_of_hbm": nbytes / (med / 1e3) / 1e9 / peak, "peak_source": pk,
            "GFLOPps": 5.0 * n_total * math.log2(max(2, n_total)) * b / (med / 1e3) / 1e9,
            "launches": plan.launches(), "plan": plan.describe(), "accuracy": acc}), flush=True)
    plan.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the C3 multi-axis, C4 uneven and C5 serving keys of the bench line")
    ap.add_argument("--extra-reps", type=int, default=10, help="timed executions per C3 form")
    ap.add_argument("--e2e-chunk", type=int, default=E2E_CHUNK, help="rows per chunk of the streamed end-to-end step")
    ap.add_argument("--workload", default="roundtrip", choices=["roundtrip", "uneven", "serving", "kernel"])
    ap.add_argument("--kind", default="c2c", choices=["c2c", "r2c", "c2r"], help="(kernel) transform type")
    ap.add_argument("--sizes", default="4096", help="(kernel) comma-separated transform sizes (1D/2D/3D)")
    ap.add_argument("--batch", type=int, default=4096, help="(kernel) batch")
    ap.add_argument("--inverse", action="store_true", help="(kernel) INVERSE direction")
    ap.add_argument("--check", action="store_true", help="(kernel) check one transform against the oracle")
    ap.add_argument("--reps", type=int, default=20, help="(kernel) executions per timed sample")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16x3", "bf16x3"],
                    help="(kernel, serving) stage arithmetic: FP32 kernels or tensor-core hi/lo split forms")
    ap.add_argument("--device-io", action="store_true", help="(serving) request buffers in HBM instead of pinned host")
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--rates", default="1,10,100,1000,10000,50000")
    ap.add_argument("--seconds", type=float, default=1.0)
    ap.add_argument("--max-requests", type=int, default=2000)
    ap.add_argument("--autotune", action="store_true", help="(uneven) run the autotuner and refresh its cache")
    ap.add_argument("--uneven-total", type=int, default=20000, help="(uneven) transforms in the drawn set")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.workload == "uneven":
        run_uneven(args, world, rank, local)
        return
    if args.workload == "serving":
        run_serving(args, world, rank, local)
        return
    if args.workload == "kernel":
        run_kernel(args, world, rank, local)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
