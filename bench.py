#!/usr/bin/env python
"""Benchmark of SHAFFT's C2C hot path on B200.

Workload (one "step"): FFTND 512x512x512 complex64, forward transform then
backward transform, each followed by normalize (fused into the transform's
last pass through shafftExecuteNormalized / the kernel ABI's scale).
Metric: GB/s of compulsory HBM traffic, 2 transforms x (read + write of the
8-byte-element tensor) = 2*2*8*512^3 bytes per step, divided by the step
time; "% HBM peak" is that figure over the measured copy bandwidth.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms:
  ours       value: device-resident tensor, kernels launched through the
             kernel library's C ABI on one stream, CUDA events around every
             launch; e2e: the public SHAFFT C ABI (libshafft.so) with pinned
             host buffers, H2D + execute + execute + D2H inside the timed
             region.
  reference  the reference's CPU path as restated by the oracle
             (oracle/oracle_fft.c, FP64, all host threads); FFTW and MPI are
             not installed, so the reference's own FFTW backend cannot be
             built.  Each step is a bounded sample (256^3 fwd+bwd).
Multi-GPU (torchrun): every rank transforms its own 512^3 tensor (replicas,
weak scaling); time = max over ranks of the CUDA-event time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D C2C fwd+bwd GB/s (% HBM peak) at 512^3 c64"
UNIT = "GB/s"
DIMS = (512, 512, 512)
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", default=None, help="override the 512^3 workload (debug only)")
    ap.add_argument("--tensor-core", action="store_true",
                    help="plan with the tensor-core form (complex64; debug / profiling of that form)")
    ap.add_argument("--plan-flags", type=int, default=0,
                    help="SHAFFT_SM100_PLAN_* flags of the plan (debug / profiling; 2 = tensor cores "
                         "on prime-factor axes)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-lanes", type=int, default=2,
                    help="plans / host threads of the e2e arm (overlapping steps)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--suite", default="headline", choices=["headline", "batched", "serve", "configs", "tc"],
                    help="headline (default, the contract line) or one of the side workloads")
    ap.add_argument("--count", type=int, default=4096, help="transforms of the batched suite")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def step_bytes(dims, esize=8):
    n = math.prod(dims)
    return 2 * 2 * esize * n


# ---------------------------------------------------------------------------
# clocks (nvidia-smi sampled during the timed region)
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# ncu traffic summary committed under profiles/
# ---------------------------------------------------------------------------

def committed_traffic(dims, prec, step):
    """bytes per launch of `step` from profiles/ncu_traffic.txt (lines of
    key=value pairs: dims=512x512x512 prec=c64 step=i bytes_per_launch=B)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    want = {"dims": "x".join(str(d) for d in dims), "prec": prec, "step": str(step)}
    for line in open(path):
        if line.startswith("#") or "=" not in line:
            continue
        kv = dict(p.split("=", 1) for p in line.split() if "=" in p)
        if all(kv.get(k) == v for k, v in want.items()) and "bytes_per_launch" in kv:
            return float(kv["bytes_per_launch"])
    return None


# ---------------------------------------------------------------------------
# CPU baseline (oracle port, all host threads)
# ---------------------------------------------------------------------------

def cpu_sample(threads=None, dims=(256, 256, 256)):
    import numpy as np

    from oracle import oracle as o
    threads = threads or os.cpu_count() or 1
    x = o.uniform_input(dims, seed=42, dtype=np.complex128)
    n = x.size
    f = o.nd_norm_factor(n, 1)
    t0 = time.perf_counter()
    y = o.fftn(x, sign=-1, nthreads=threads) * f
    z = o.fftn(y, sign=1, nthreads=threads) * f
    t = time.perf_counter() - t0
    err = o.rel_l2(z, x)
    return step_bytes(dims) / t / 1e9, t, threads, err


def cpu_model():
    """Host CPU model name (Linux /proc/cpuinfo), recorded beside the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dims = (256, 256, 256)
    threads = os.cpu_count() or 1
    for _ in range(max(0, args.warmup)):
        cpu_sample(threads, dims)
    times = []
    for _ in range(max(1, args.steps)):
        _, t, _, err = cpu_sample(threads, dims)
        times.append(t)
    tot = sum(times)
    value = step_bytes(dims) * len(times) / tot / 1e9
    sample = (f"{'x'.join(map(str, dims))} complex64 forward+normalize+backward+normalize per step, "
              f"FP64 Stockham restatement of the FFTW path (oracle/oracle_fft.c), {threads} threads; "
              f"FFTW/MPI not installed so the reference's FFTW backend cannot be built")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "FFTND complex C2C fwd+bwd with normalize, bounded CPU sample",
                   "dims": list(dims), "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "roundtrip_rel_l2": err,
    }
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# replicas: one process per GPU, no data-path collective
# ---------------------------------------------------------------------------

def dist_init(backend="nccl"):
    """(rank, world, local_rank, process group or None) from the torchrun
    environment; the group exists only for N > 1 and carries timing
    reductions, never data."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return rank, world, local, dist


def _reduce(x, dist, device, op):
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op(dist))
    return float(t.item())


def max_over_ranks(x, dist, device="cuda"):
    return _reduce(x, dist, device, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(x, dist, device="cuda"):
    return _reduce(x, dist, device, lambda d: d.ReduceOp.SUM)


def shard(seq, rank, world):
    """Contiguous block of `seq` owned by `rank` (block sizes differ by at
    most one; the blocks of all ranks partition `seq` in order)."""
    n = len(seq)
    return list(seq[rank * n // world:(rank + 1) * n // world])


def kernel_name(st):
    """Kernel that runs a plan step (from the plan's JSON description)."""
    if st.get("tc"):
        return "k_fft_tc"
    if st.get("fast"):
        if not st.get("in_row") and st.get("L") in (256, 512) and os.environ.get("SHAFFT_SM100_TMA", "0") != "0":
            return "k_fft_fast_tma"  # column tile fed by bulk tensor copies (when its view qualifies)
        return f"k_fft_fast<IN_ROW={st.get('in_row', 0)}>"
    if st["kind"] == "plane":
        return "k_fft_plane_flow"
    return "k_fft_pass" if st["kind"] == "pass" else f"k_bs/{st['kind']}"


def ours(args):
    import torch

    import shafft_b200 as S
    from shafft_b200 import _sm100

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rank, world, local, dist = dist_init("nccl")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    dims = tuple(int(v) for v in args.dims.split("x")) if args.dims else DIMS
    n = math.prod(dims)
    plan = _sm100.Plan(dims, 0, (_sm100.PLAN_TENSOR_CORE if args.tensor_core else 0) | args.plan_flags)
    nst = plan.launches
    scale = float(1.0 / math.sqrt(n))
    # a dedicated stream: the kernels and the events that time them share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    gen = torch.Generator(device="cuda").manual_seed(42 + rank)
    a = (torch.rand(2 * n, device="cuda", generator=gen) * 2 - 1).view(torch.complex64)
    b = torch.empty_like(a)
    ap, bp = a.data_ptr(), b.data_ptr()

    def one_step(events=None):
        for direction, (src, dst) in ((0, (ap, bp)), (1, (bp, ap))):
            for i in range(nst):
                if events is not None:
                    ev = torch.cuda.Event(enable_timing=True)
                    ev.record(stream)
                    events.append((direction, i, ev))
                plan.execute_step(i, src, dst, direction, scale, sh)

    for _ in range(max(3, args.warmup)):
        one_step()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.2)
    barrier()
    events = []
    t0 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        one_step(events)
    t1 = torch.cuda.Event(enable_timing=True)
    t1.record(stream)
    barrier()
    clocks.stop()
    total_ms = t0.elapsed_time(t1)
    # per-kernel durations
    per = {}
    bounds = [e for (_, _, e) in events] + [t1]
    for j, (direction, i, ev) in enumerate(events):
        per.setdefault(i, []).append(ev.elapsed_time(bounds[j + 1]))
    tmax = max_over_ranks(total_ms, dist)
    ms_per_step = tmax / args.steps
    value = world * step_bytes(dims) * args.steps / (tmax / 1e3) / 1e9

    peak, peak_kind = peaks()
    desc = plan.describe()
    kern = []
    for i in range(nst):
        d = per.get(i, [0.0])
        kern.append({"step": i, "kind": desc["steps"][i]["kind"], "L": desc["steps"][i].get("L"),
                     "avg_ms": sum(d) / len(d), "alg_bytes": plan.step_bytes(i)})
    dom = max(kern, key=lambda k: k["avg_ms"])
    achieved = dom["alg_bytes"] / (dom["avg_ms"] / 1e3) / 1e9
    traffic = committed_traffic(dims, "c64", dom["step"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": f"{kernel_name(desc['steps'][dom['step']])} step {dom['step']} (L={dom['L']})",
                "alg_bytes_per_launch": dom["alg_bytes"]}
    plan_bytes_per_step = 2 * sum(k["alg_bytes"] for k in kern)

    e2e = None
    if not args.no_e2e and world >= 1:
        e2e = e2e_arm(S, dims, n, args, stream, barrier, dist)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, t, thr, err = cpu_sample()
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"256x256x256 complex64 fwd+normalize+bwd+normalize, FP64 oracle "
                         f"(oracle/oracle_fft.c), {thr} threads, {t:.2f} s",
               "cpu_model": cpu_model()}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": "FFTND 512x512x512 complex64 C2C: forward+normalize then "
                        "backward+normalize (normalize fused into the last pass)"
            if dims == DIMS else f"FFTND {'x'.join(map(str, dims))} complex64 fwd+bwd",
            "dims": list(dims), "precision": "complex64", "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (1 GiB tensor vs 126 MB L2), no flush",
            "bytes_per_step": step_bytes(dims),
            "plan_hbm_bytes_per_step": plan_bytes_per_step,
            "passes_per_transform": nst,
            "pct_hbm_peak": 100.0 * value / world / peak,
            "plan_hbm_gbs": world * plan_bytes_per_step * args.steps / (tmax / 1e3) / 1e9,
            "kernels": kern,
        },
        "e2e": e2e,
        "gpu_launches": args.steps * 2 * nst,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def e2e_arm(S, dims, n, args, stream, barrier, dist):
    """Public SHAFFT C ABI with host buffers: per step, copy the input from
    pinned host memory, forward+normalize, backward+normalize, copy the
    result back.  Two plan instances are driven from two host threads (each
    thread's NULL-stream work goes to its own stream), so one step's
    device->host copy overlaps the next step's host->device copy on the
    full-duplex PCIe link; every step still moves its own input and result."""
    import threading

    import torch
    lanes = max(1, args.e2e_lanes)
    lib = S.load()
    nbytes = 8 * n
    plans, bufs, hosts = [], [], []
    for _ in range(lanes):
        plan = S.FFTND()
        S.check(plan.init([1] * len(dims), list(dims), S.C2C), "init")
        S.check(plan.plan(), "plan")
        da = S.DeviceBuffer(n, S.C2C)
        db = S.DeviceBuffer(n, S.C2C)
        S.check(plan.set_buffers(da.ptr, db.ptr), "setBuffers")
        host_in = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
        host_in.uniform_(-1, 1)
        host_out = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
        plans.append(plan)
        bufs.append((da, db))
        hosts.append((host_in, host_out))

    def step(i):
        plan, (host_in, host_out) = plans[i], hosts[i]
        _, d, _ = plan.get_buffers()
        S.check(lib.shafftCopyToBufferF(ctypes.c_void_p(d), ctypes.c_void_p(host_in.data_ptr()), n),
                "copyToBuffer")
        S.check(plan.execute_normalized(S.FORWARD), "execute")
        S.check(plan.execute_normalized(S.BACKWARD), "execute")
        _, d, _ = plan.get_buffers()
        S.check(lib.shafftCopyFromBufferF(ctypes.c_void_p(host_out.data_ptr()), ctypes.c_void_p(d), n),
                "copyFromBuffer")

    errors = []
    dev = torch.cuda.current_device()  # new threads start on device 0

    def lane(i, count):
        try:
            torch.cuda.set_device(dev)
            for _ in range(count):
                step(i)
        except Exception as e:  # surfaced after join
            errors.append(e)

    def run(count_per_lane):
        th = [threading.Thread(target=lane, args=(i, count_per_lane)) for i in range(lanes)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errors:
            raise errors[0]

    run(max(1, min(args.warmup, 2)))
    k = lanes * max(2, min(args.steps, 10) // lanes)
    barrier()
    w0 = time.perf_counter()
    run(k // lanes)
    barrier()
    wall = time.perf_counter() - w0
    tmax = max_over_ranks(1e3 * wall, dist)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    for plan in plans:
        plan.release()
    return {"value": world * step_bytes(dims) * k / (tmax / 1e3) / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": k,
            "ms_per_step": tmax / k,
            "path": "libshafft.so C ABI: shafftCopyToBufferF, shafftExecuteNormalized x2, "
                    f"shafftCopyFromBufferF, pinned host buffers; {lanes} plans on {lanes} host "
                    "threads (steps overlap), host wall clock between barriers"}


# ---------------------------------------------------------------------------
# side workloads (not the contract line)
# ---------------------------------------------------------------------------

def _is_smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def _is_prime(n):
    return n > 1 and all(n % d for d in range(2, int(n ** 0.5) + 1))


def batched_shapes(count=4096, seed=42):
    """Seeded uneven 2-D/3-D shapes: extents log-uniform in [16, 256] over the
    7-smooth numbers, 5% drawn from the primes in [16, 256]."""
    import numpy as np
    rng = np.random.Generator(np.random.MT19937(seed))
    smooth = [n for n in range(16, 257) if _is_smooth7(n)]
    lsm = np.log(np.array(smooth, dtype=np.float64))
    primes = [p for p in range(16, 257) if _is_prime(p)]
    shapes = []
    for _ in range(count):
        nd = 2 if rng.uniform() < 0.5 else 3
        dims = []
        for _ in range(nd):
            if rng.uniform() < 0.05:
                dims.append(int(primes[int(rng.integers(0, len(primes)))]))
            else:
                v = rng.uniform(np.log(16), np.log(256))
                dims.append(int(smooth[int(np.argmin(np.abs(lsm - v)))]))
        shapes.append(tuple(dims))
    return shapes


def suite_batched(args):
    import numpy as np
    import torch

    import shafft_b200 as S  # noqa: F401
    from oracle import oracle as o
    from shafft_b200 import _sm100
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank, world, _, dist = dist_init("nccl")
    # replicas: each rank owns a contiguous block of the transform list
    shapes = shard(batched_shapes(args.count), rank, world)
    sizes = [math.prod(s) for s in shapes]
    offs, tot = [], 0
    for n in sizes:
        offs.append(tot)
        tot += (n + 63) // 64 * 64
    gen = torch.Generator(device="cuda").manual_seed(42)
    src = (torch.rand(2 * tot, device="cuda", generator=gen) * 2 - 1).view(torch.complex64)
    dst = torch.empty_like(src)
    scr = torch.empty_like(src)
    sp = [src.data_ptr() + 8 * off for off in offs]
    dp = [dst.data_ptr() + 8 * off for off in offs]
    cp = [scr.data_ptr() + 8 * off for off in offs]
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    batch = _sm100.Batch(shapes, 0, autotune=True)
    t_create = time.perf_counter() - t0
    for _ in range(2):
        batch.execute(sp, dp, 0, 1.0, stream.cuda_stream)
    torch.cuda.synchronize()
    k = max(3, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        batch.execute(sp, dp, 0, 1.0, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    batch.status()
    t_batch = e0.elapsed_time(e1) / k
    # sampled parity against the oracle
    rng = np.random.Generator(np.random.MT19937(7))
    small = [i for i, n in enumerate(sizes) if n <= (1 << 20)]
    sample = sorted(set(rng.choice(small, size=min(24, len(small)), replace=False).tolist()
                        + [i for i in small if any(_is_prime(d) for d in shapes[i])][:8]))
    errs = []
    for i in sample:
        x = src[offs[i]:offs[i] + sizes[i]].cpu().numpy().reshape(shapes[i])
        y = dst[offs[i]:offs[i] + sizes[i]].cpu().numpy().reshape(shapes[i])
        errs.append(o.rel_l2(y, o.fftn(x.astype(np.complex128))))
    # the plain path: one plan per transform, launched one by one
    t0 = time.perf_counter()
    plans = {}
    for s in shapes:
        if s not in plans:
            plans[s] = _sm100.Plan(s, 0)
    t_plans = time.perf_counter() - t0
    launches = sum(plans[s].launches for s in shapes)

    def plain():
        for i, s in enumerate(shapes):
            plans[s].execute(cp[i], dp[i], 0, 1.0, stream.cuda_stream)
    scr.copy_(src)
    # two untimed passes: a plan replays a launch sequence it has seen twice
    # (graph replay of executes), so the timed passes run at steady state
    for _ in range(2):
        plain()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(2):
        plain()
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 2
    comp = sum(2 * 8 * n for n in sizes)
    # whole job: bytes of all ranks over the slowest rank's time
    comp_all = sum_over_ranks(comp, dist)
    t_batch = max_over_ranks(t_batch, dist)
    t_plain = max_over_ranks(t_plain, dist)
    if rank != 0:
        dist.destroy_process_group()
        return 0
    out = {
        "metric": "batched uneven 2-D/3-D c64 forward transforms: compulsory GB/s", "unit": "GB/s",
        "value": comp_all / (t_batch / 1e3) / 1e9, "plain_value": comp_all / (t_plain / 1e3) / 1e9,
        "speedup_vs_plain": t_plain / t_batch, "ms_batched": t_batch, "ms_plain": t_plain,
        "n_gpus": world, "transforms_per_rank": len(shapes), "elements_rank0": sum(sizes),
        "plan_hbm_gbs_batched": batch.alg_bytes / (t_batch / 1e3) / 1e9,
        "launches_batched_per_execute": 1, "launches_plain_per_execute": launches,
        "create_s": {"batch_with_autotune": t_create, "plain_plans": t_plans},
        "batch": batch.describe(), "max_rel_l2_sample": max(errs), "sample": len(errs),
        "tol_c64": "1e-6*log2(N)", "data": "synthetic",
    }
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


SERVE_1D = [1 << e for e in range(10, 23)]
SERVE_2D = [64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048]
SERVE_3D = [32, 48, 64, 96, 128, 192, 256, 384]
SERVE_PRIMES = {1: [1031, 16411, 262147, 1048583], 2: [97, 211, 509, 1021], 3: [37, 97, 131, 257]}


def serve_requests(count, seed=42):
    """Seeded request mix: equal shares of 1-D (2^10..2^22), 2-D (64^2..2048^2)
    and 3-D (32^3..384^3) sizes drawn log-uniformly from a fixed ladder (so
    shapes repeat and plans stay resident), 30% complex128, 10% with a prime
    length, forward/backward 50/50."""
    import numpy as np
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for _ in range(count):
        cls = int(rng.integers(1, 4))
        ladder = {1: SERVE_1D, 2: SERVE_2D, 3: SERVE_3D}[cls]
        n = ladder[int(rng.integers(0, len(ladder)))]
        dims = [n] * cls
        if rng.uniform() < 0.10:
            dims[int(rng.integers(0, cls))] = int(rng.choice(SERVE_PRIMES[cls]))
        prec = 1 if rng.uniform() < 0.30 else 0
        out.append((tuple(dims), prec, int(rng.integers(0, 2))))
    return out


def suite_serve(args):
    import numpy as np
    import torch

    from shafft_b200 import _sm100
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank, world, _, dist = dist_init("nccl")
    # replicas: each rank serves a contiguous block of the request stream
    reqs = shard(serve_requests(max(40, min(args.count, 400)) * world), rank, world)
    maxb = max(math.prod(d) * (16 if p else 8) for d, p, _ in reqs)
    hin = torch.empty(maxb // 4, dtype=torch.float32, pin_memory=True).uniform_(-1, 1)
    hout = torch.empty(maxb // 4, dtype=torch.float32, pin_memory=True)
    # serial baseline: one request at a time through a resident plan
    plans = {}
    dev = torch.empty(maxb // 4, dtype=torch.float32, device="cuda")
    dev2 = torch.empty_like(dev)
    lib = _sm100.load()

    def serial_one(dims, prec, direction):
        key = (dims, prec)
        if key not in plans:
            plans[key] = _sm100.Plan(dims, prec)
        nb = math.prod(dims) * (16 if prec else 8)
        t0 = time.perf_counter()
        lib.shafft_sm100_memcpy(ctypes.c_void_p(dev.data_ptr()), ctypes.c_void_p(hin.data_ptr()), nb, 1, None)
        plans[key].execute(dev.data_ptr(), dev2.data_ptr(), direction, 1.0, 0)
        lib.shafft_sm100_memcpy(ctypes.c_void_p(hout.data_ptr()), ctypes.c_void_p(dev2.data_ptr()), nb, 2, None)
        return (time.perf_counter() - t0) * 1e3
    for d, p, r in reqs:  # warm plans
        serial_one(d, p, r)
    t0 = time.perf_counter()
    lat = [serial_one(d, p, r) for d, p, r in reqs]
    serial_s = time.perf_counter() - t0
    serial_tput = len(reqs) / serial_s
    lat.sort()
    serial = {"throughput_per_s": serial_tput, "p50_ms": lat[len(lat) // 2],
              "p99_ms": lat[min(len(lat) - 1, int(0.99 * (len(lat) - 1) + 0.5))]}
    del plans, dev, dev2
    torch.cuda.empty_cache()
    srv = _sm100.Server(budget_bytes=40 << 30, streams=8)
    # warm the server's plan cache with one pass over the mix
    ids = [srv.submit(d, p, r, 1.0, hin.data_ptr(), hout.data_ptr()) for d, p, r in reqs]
    for i in ids:
        srv.wait(i)
    rng = np.random.Generator(np.random.MT19937(5))
    sweep = []
    for mult in (0.5, 1.0, 2.0, 4.0, 8.0):
        rate = mult * serial_tput
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        srv.reset_stats()
        start = time.perf_counter()
        due = start
        ids = []
        for (d, p, r), gap in zip(reqs, gaps):
            due += gap
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            ids.append(srv.submit(d, p, r, 1.0, hin.data_ptr(), hout.data_ptr()))
        for i in ids:
            srv.wait(i)
        wall = time.perf_counter() - start
        st = srv.stats()
        st["offered_per_s"] = rate
        st["achieved_per_s"] = len(reqs) / wall
        sweep.append(st)
    srv.destroy()
    best = max(s["achieved_per_s"] for s in sweep)
    # whole job: request rates add over the replicas; latency is the worst rank's
    best_all = sum_over_ranks(best, dist)
    serial_all = sum_over_ranks(serial_tput, dist)
    p99_best = max_over_ranks(max(sweep, key=lambda s: s["achieved_per_s"])["p99_ms"], dist)
    if rank != 0:
        dist.destroy_process_group()
        return 0
    out = {"metric": "served mixed C2C requests: throughput and p50/p99 latency", "unit": "requests/s",
           "value": best_all, "serial_plain": serial, "speedup_vs_serial": best_all / serial_all,
           "n_gpus": world, "p99_ms_at_best_worst_rank": p99_best,
           "requests_per_rank": len(reqs), "budget_bytes": 40 << 30, "streams": 8,
           "sweep_rank0": sweep,
           "host_buffers": "pinned, shared by all requests (timing only)", "data": "synthetic"}
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def suite_configs(args):
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.current_stream()
    peak, _ = peaks()
    res = []

    def run(dims, prec, reps, check):
        n = math.prod(dims)
        dt = torch.complex128 if prec else torch.complex64
        es = 16 if prec else 8
        x = o.uniform_input(dims, seed=42, dtype=np.complex128 if prec else np.complex64) if check else None
        a = torch.from_numpy(x.ravel()).cuda() if check else torch.randn(n, dtype=dt, device="cuda")
        a0 = a.clone()
        b = torch.empty_like(a)
        p = _sm100.Plan(dims, prec)
        err = None
        if check:
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            y = b.cpu().numpy()
            err = o.rel_l2(y, o.fftn(x.astype(np.complex128), precise=bool(prec)).ravel())
        for _ in range(3):
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        comp = 2 * 2 * es * n
        res.append({"dims": list(dims), "precision": "c128" if prec else "c64", "ms_fwd_bwd": ms,
                    "compulsory_gbs": comp / (ms / 1e3) / 1e9,
                    "plan_gbs": 2 * sum(p.step_bytes(i) for i in range(p.launches)) / (ms / 1e3) / 1e9,
                    "pct_hbm_plan": 100 * 2 * sum(p.step_bytes(i) for i in range(p.launches)) / (ms / 1e3) / 1e9 / peak,
                    "launches_per_transform": p.launches,
                    "rel_l2_vs_oracle": err,
                    "tol": (1e-6 if prec == 0 else 1e-14) * math.log2(n)})
        del a, a0, b
        p.destroy()
    run((256, 256, 256), 1, 20, False)
    run((64, 64, 32), 0, 50, True)
    for n in (1 << 24, 1488375, 1000003):
        for prec in (0, 1):
            run((n,), prec, 10, True)
    print(json.dumps({"metric": "other configurations (512^3 aside): fwd+bwd time and error", "configs": res}), flush=True)
    return 0


def suite_tc(args):
    """Tensor-core form (tcgen05 split-FP16 DFT stages) against the plain
    kernels on the same GPU: fwd+bwd time, per-pass kernel times and the
    forward error of both forms against the FP64 oracle."""
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.current_stream()
    peak, _ = peaks()
    res = []

    def run(dims, flags, reps, ref):
        n = math.prod(dims)
        x = o.uniform_input(dims, seed=42, dtype=np.complex64)
        a = torch.from_numpy(x.ravel()).cuda()
        b = torch.empty_like(a)
        p = _sm100.Plan(dims, 0, flags)
        p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
        p.status()
        err = o.rel_l2(b.cpu().numpy(), ref.ravel())
        a.copy_(torch.from_numpy(x.ravel()))
        for _ in range(3):
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        # per-launch times of one forward (steps run in order on one stream)
        steps = p.describe()["steps"]
        per = []
        for i in range(p.launches):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for _ in range(2):
                p.execute_step(i, a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            s0.record(stream)
            for _ in range(5):
                p.execute_step(i, a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            s1.record(stream)
            torch.cuda.synchronize()
            t = s0.elapsed_time(s1) / 5
            st = steps[i]
            d = {"kind": st["kind"], "L": st.get("L"), "tc": st.get("tc", 0), "ms": t,
                 "gbs": p.step_bytes(i) / (t / 1e3) / 1e9}
            if st.get("tc"):
                lp = (st["L"] + 15) // 16 * 16
                rows = n // st["L"]
                groups = -(-rows // 128)
                # 3 products x Lp/16 K-steps x 4 MMAs of 128 x Lp x 16 per group
                d["mma_tflops"] = groups * 3072 * lp * lp / (t / 1e3) / 1e12
            per.append(d)
        plan_bytes = sum(p.step_bytes(i) for i in range(p.launches))
        out = {"ms_fwd_bwd": ms, "compulsory_gbs": 2 * 2 * 8 * n / (ms / 1e3) / 1e9,
               "plan_gbs": 2 * plan_bytes / (ms / 1e3) / 1e9,
               "pct_hbm_plan": 100 * 2 * plan_bytes / (ms / 1e3) / 1e9 / peak,
               "launches": p.launches, "rel_l2_fwd_vs_fp64_oracle": err, "steps": per}
        del a, b
        p.destroy()
        return out

    # the FFT1D sizes of the tensor-core configuration and the headline, then
    # axes with a prime factor above 13, where the plain path runs O(L^2)
    # direct DFTs and the hybrid plan (tensor cores on those axes only) applies
    for dims in ((1 << 24,), (1488375,), (1000003,), (64, 64, 32), (512, 512, 512),
                 (65536, 61), (65536, 47), (65536, 31), (65536, 17), (4096, 61, 16), (61, 61, 61),
                 (53, 59, 61)):
        n = math.prod(dims)
        x = o.uniform_input(dims, seed=42, dtype=np.complex64)
        ref = o.fftn(x.astype(np.complex128))
        plain = run(dims, 0, 10, ref)
        tc = run(dims, _sm100.PLAN_TENSOR_CORE, 10, ref)
        row = {"dims": list(dims), "tol": 1e-6 * math.log2(n), "plain": plain, "tensor_core": tc,
               "speedup_tc_vs_plain": plain["ms_fwd_bwd"] / tc["ms_fwd_bwd"]}
        if any(s.get("tc") for s in _sm100.plan_query(dims, 0, _sm100.PLAN_TC_PRIME_AXES)["steps"]):
            hy = run(dims, _sm100.PLAN_TC_PRIME_AXES, 10, ref)
            row["tc_prime_axes"] = hy
            row["speedup_hybrid_vs_plain"] = plain["ms_fwd_bwd"] / hy["ms_fwd_bwd"]
        res.append(row)
    print(json.dumps({"metric": "tensor-core split-FP16 form vs plain FP32 kernels, complex64 fwd+bwd",
                      "configs": res, "data": "synthetic, iid uniform[-1,1) seed 42"}), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.suite == "batched":
        return suite_batched(args)
    if args.suite == "serve":
        return suite_serve(args)
    if args.suite == "configs":
        return suite_configs(args)
    if args.suite == "tc":
        return suite_tc(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
