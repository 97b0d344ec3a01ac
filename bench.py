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
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
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
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "roundtrip_rel_l2": err,
    }
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def ours(args):
    import torch

    import shafft_b200 as S
    from shafft_b200 import _sm100

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    dims = tuple(int(v) for v in args.dims.split("x")) if args.dims else DIMS
    n = math.prod(dims)
    plan = _sm100.Plan(dims, 0)
    nst = plan.launches
    scale = float(1.0 / math.sqrt(n))
    stream = torch.cuda.current_stream()
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
    tmax = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tmax = float(tmax.item())
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
                "kernel": f"k_fft_pass step {dom['step']} (L={dom['L']})",
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
                         f"(oracle/oracle_fft.c), {thr} threads, {t:.2f} s"}
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
    result back."""
    import torch
    plan = S.FFTND()
    S.check(plan.init([1] * len(dims), list(dims), S.C2C), "init")
    S.check(plan.plan(), "plan")
    da = S.DeviceBuffer(n, S.C2C)
    db = S.DeviceBuffer(n, S.C2C)
    S.check(plan.set_buffers(da.ptr, db.ptr), "setBuffers")
    host_in = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
    host_in.uniform_(-1, 1)
    host_out = torch.empty(2 * n, dtype=torch.float32, pin_memory=True)
    lib = S.load()
    nbytes = 8 * n

    def step():
        _, d, _ = plan.get_buffers()
        S.check(lib.shafftCopyToBufferF(ctypes.c_void_p(d), ctypes.c_void_p(host_in.data_ptr()), n),
                "copyToBuffer")
        S.check(plan.execute_normalized(S.FORWARD), "execute")
        S.check(plan.execute_normalized(S.BACKWARD), "execute")
        _, d, _ = plan.get_buffers()
        S.check(lib.shafftCopyFromBufferF(ctypes.c_void_p(host_out.data_ptr()), ctypes.c_void_p(d), n),
                "copyFromBuffer")

    for _ in range(max(2, min(args.warmup, 3))):
        step()
    k = max(3, min(args.steps, 10))
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(torch.cuda.default_stream())
    w0 = time.perf_counter()
    for _ in range(k):
        step()
    t1.record(torch.cuda.default_stream())
    barrier()
    wall = time.perf_counter() - w0
    ms = t0.elapsed_time(t1)
    tt = torch.tensor([max(ms, 1e3 * wall)], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    tmax = float(tt.item())
    world = int(os.environ.get("WORLD_SIZE", "1"))
    plan.release()
    return {"value": world * step_bytes(dims) * k / (tmax / 1e3) / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": k,
            "ms_per_step": tmax / k,
            "path": "libshafft.so C ABI: shafftCopyToBufferF, shafftExecuteNormalized x2, "
                    "shafftCopyFromBufferF, pinned host buffers"}


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
