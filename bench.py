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
             launch; after the timed region the buffers it transformed are
             checked (K+W normalised round trips must return the input).
             e2e: the public SHAFFT C ABI (libshafft.so) with pinned host
             buffers, H2D + execute + execute + D2H inside the timed region.
             api_sequence: the reference's own call sequence through the C
             ABI (execute, normalize, execute, normalize; device-resident).
             At N = 1 the line also carries `configs` (the other transform
             sizes) and `forms` (tensor-core, batched and served forms
             against the plain kernels), each timing with its own clock
             record and its error against the CPU oracle.
  reference  the reference's CPU path as restated by the oracle
             (oracle/oracle_fft.c, FP64, all host threads) on the same
             512^3 workload; FFTW and MPI are not installed, so the
             reference's own FFTW backend cannot be built.
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
    ap.add_argument("--no-forms", action="store_true",
                    help="leave the configs / forms objects out of the default line")
    ap.add_argument("--suite", default="headline", choices=["headline", "batched", "serve", "configs", "tc", "exchange"],
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
    y = o.fftn(x, sign=-1, nthreads=threads)
    y *= f
    z = o.fftn(y, sign=1, nthreads=threads)
    z *= f
    t = time.perf_counter() - t0
    del y
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


WORKLOAD = ("FFTND 512x512x512 complex64 C2C: forward+normalize then backward+normalize "
            "(iid U[-1,1) input)")


def headline_config(dims, world):
    """`config` of both arms (identical for the same workload)."""
    return {"workload": WORKLOAD if dims == DIMS else
            f"FFTND {'x'.join(map(str, dims))} complex64 C2C: forward+normalize then backward+normalize",
            "dims": list(dims), "precision": "complex64", "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (1 GiB tensor vs 126 MB L2), no flush"}


def reference_arm(args):
    """The reference's CPU path (its FFTW backend, restated by the oracle:
    one full C2C per execute, then a separate normalize,
    src/cpp/fft/fftw_method/fftnd_method.cpp:236-276 and
    src/cpp/shafft_internal.cpp:129-188) on the same 512^3 workload as our
    arm, all host threads.  Only rank 0 runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dims = tuple(int(v) for v in args.dims.split("x")) if args.dims else DIMS
    threads = os.cpu_count() or 1
    for _ in range(max(0, args.warmup)):
        cpu_sample(threads, dims)
    times = []
    err = None
    for _ in range(max(1, args.steps)):
        _, t, _, err = cpu_sample(threads, dims)
        times.append(t)
    tot = sum(times)
    value = step_bytes(dims) * len(times) / tot / 1e9
    v256, t256, _, _ = cpu_sample(threads, (256, 256, 256))
    sample = (f"{'x'.join(map(str, dims))} complex64 forward+normalize+backward+normalize per step "
              f"(the full workload), FP64 Stockham restatement of the FFTW path (oracle/oracle_fft.c), "
              f"{threads} threads; FFTW/MPI not installed so the reference's FFTW backend cannot be built")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": headline_config(dims, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "roundtrip_rel_l2": err,
        "extra_256cube": {"value": v256, "unit": UNIT, "ms_per_step": 1e3 * t256,
                          "dims": [256, 256, 256]},
    }
    print(json.dumps(out), flush=True)
    return 0


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
        if st.get("prefetch") and not st.get("bs") and not st.get("map"):
            return f"k_fft_fast_pf<IN_ROW={st.get('in_row', 0)}>"  # with the L2 prefetch of a later tile
        return f"k_fft_fast<IN_ROW={st.get('in_row', 0)}>"
    if st["kind"] == "plane":
        return "k_fft_plane_cluster" if st.get("cluster") else "k_fft_plane_flow"
    return "k_fft_pass" if st["kind"] == "pass" else f"k_bs/{st['kind']}"


def nd_norm_factor_c64(n):
    """The ND normalisation factor as libshafft applies it to complex64: long
    double 1/sqrt(N) rounded to float (src/cpp/shafft_internal.cpp:136, 153)."""
    import numpy as np
    f = np.longdouble(1) / np.sqrt(np.longdouble(n))
    return float(np.float32(f))


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
    scale = nd_norm_factor_c64(n)
    # a dedicated stream: the kernels and the events that time them share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    gen = torch.Generator(device="cuda").manual_seed(42 + rank)
    a = (torch.rand(2 * n, device="cuda", generator=gen) * 2 - 1).view(torch.complex64)
    a0 = a.clone()  # the input, to check the transformed buffers after the timed region
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
    # every step is a normalised forward+backward pair, so the buffer the
    # timed region ended on holds the input after max(3, W) + K round trips
    roundtrip = float((torch.linalg.vector_norm(a - a0) / torch.linalg.vector_norm(a0)).item())
    round_trips = max(3, args.warmup) + args.steps
    del a0
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
                     "kernel": kernel_name(desc["steps"][i]),
                     "avg_ms": sum(d) / len(d), "alg_bytes": plan.step_bytes(i)})
    dom = max(kern, key=lambda k: k["avg_ms"])
    achieved = dom["alg_bytes"] / (dom["avg_ms"] / 1e3) / 1e9
    traffic = committed_traffic(dims, "c64", dom["step"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": f"{dom['kernel']} step {dom['step']} (L={dom['L']})",
                "alg_bytes_per_launch": dom["alg_bytes"]}
    plan_bytes_per_step = 2 * sum(k["alg_bytes"] for k in kern)
    plan.destroy()
    del a, b
    torch.cuda.empty_cache()

    e2e = None
    api = None
    if not args.no_e2e:
        e2e = e2e_arm(S, dims, n, args, stream, barrier, dist)
        api = api_sequence(S, dims, n, args, barrier, dist)

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
        "config": headline_config(dims, world),
        "detail": {
            "normalize": "fused into the last pass (shafftExecuteNormalized semantics); "
                         "the reference's separate-normalize sequence is `api_sequence`",
            "bytes_per_step": step_bytes(dims),
            "plan_hbm_bytes_per_step": plan_bytes_per_step,
            "passes_per_transform": nst,
            "pct_hbm_peak": 100.0 * value / world / peak,
            "plan_hbm_gbs": world * plan_bytes_per_step * args.steps / (tmax / 1e3) / 1e9,
            "pct_hbm_peak_plan": 100.0 * plan_bytes_per_step * args.steps / (tmax / 1e3) / 1e9 / peak,
            "kernels": kern,
        },
        "check": {"roundtrip_rel_l2": roundtrip, "round_trips": round_trips,
                  "what": "the timed buffers after every normalised forward+backward pair of the "
                          "warm-up and timed steps, against the input",
                  "tol": 1e-6 * math.log2(n)},
        "e2e": e2e,
        "api_sequence": api,
        "gpu_launches": args.steps * 2 * nst,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_forms and dims == DIMS:
        out["configs"] = configs_rows(args, local) + [r2c_row(local)]
        out["forms"] = forms(args, local)
        out["exchange"] = {"what": "one rank's device steps before a 512^3 complex64 slab exchange: "
                                   "subplan + separate pack vs the pack fused into the subplan's stores",
                           "rows": exchange_rows(local)}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def api_sequence(S, dims, n, args, barrier, dist):
    """The reference's own call sequence through libshafft.so's C ABI on
    device-resident buffers: execute(FORWARD), normalize(), execute(BACKWARD),
    normalize() -- normalize is then a separate pass over the tensor, as in
    the reference (src/cpp/shafft_internal.cpp:129-188).  Every call
    synchronises, so host wall-clock between barriers times it."""
    plan = S.FFTND()
    S.check(plan.init([1] * len(dims), list(dims), S.C2C), "init")
    S.check(plan.plan(), "plan")
    da = S.DeviceBuffer(n, S.C2C)
    db = S.DeviceBuffer(n, S.C2C)
    S.check(plan.set_buffers(da.ptr, db.ptr), "setBuffers")
    def step():
        S.check(plan.execute(S.FORWARD), "execute")
        S.check(plan.normalize(), "normalize")
        S.check(plan.execute(S.BACKWARD), "execute")
        S.check(plan.normalize(), "normalize")

    for _ in range(max(2, min(args.warmup, 3))):
        step()
    k = max(3, min(args.steps, 10))
    barrier()
    w0 = time.perf_counter()
    for _ in range(k):
        step()
    barrier()
    tmax = max_over_ranks(1e3 * (time.perf_counter() - w0), dist)
    plan.release()
    da.free()
    db.free()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"value": world * step_bytes(dims) * k / (tmax / 1e3) / 1e9, "unit": UNIT, "steps": k,
            "ms_per_step": tmax / k, "passes_per_transform": "plan passes + 1 (normalize)",
            "path": "libshafft.so C ABI: shafftExecute, shafftNormalize, shafftExecute, "
                    "shafftNormalize per step, device-resident buffers, host wall clock"}


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


def timed_region(fn, stream, gpu, target_s=0.4, min_reps=3):
    """CUDA-event time of fn() on `stream`, ms per call, over enough calls
    to last about target_s (after 3 untimed calls), with nvidia-smi clocks
    sampled over the timed calls.  Returns (ms, reps, clocks)."""
    import torch
    for _ in range(3):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    one = max(e0.elapsed_time(e1) / 1e3, 1e-6)
    reps = max(min_reps, int(target_s / one))
    clk = ClockSampler(gpu)
    clk.start()
    time.sleep(0.15)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    clk.stop()
    return e0.elapsed_time(e1) / reps, reps, clk.summary()


def batched_form(count, gpu, rank=0, world=1, dist=None):
    """C4: `count` seeded uneven 2-D/3-D complex64 transforms (this rank's
    contiguous block), one persistent graph-captured launch per execute vs
    one plain plan execute per transform; sampled error vs the oracle."""
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    shapes = shard(batched_shapes(count), rank, world)
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

    def run_batch():
        batch.execute(sp, dp, 0, 1.0, stream.cuda_stream)
    t_batch, reps_b, clk_b = timed_region(run_batch, stream, gpu, target_s=0.6)
    batch.status()
    # sampled parity against the oracle
    rng = np.random.Generator(np.random.MT19937(7))
    small = [i for i, n in enumerate(sizes) if n <= (1 << 20)]
    sample = sorted(set(rng.choice(small, size=min(24, len(small)), replace=False).tolist()
                        + [i for i in small if any(_is_prime(d) for d in shapes[i])][:8]))
    errs = []
    for i in sample:
        x = src[offs[i]:offs[i] + sizes[i]].cpu().numpy().reshape(shapes[i])
        y = dst[offs[i]:offs[i] + sizes[i]].cpu().numpy().reshape(shapes[i])
        errs.append((o.rel_l2(y, o.fftn(x.astype(np.complex128))), 1e-6 * math.log2(max(2, sizes[i]))))
    # the plain path: one plan per distinct shape, one execute per transform
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
    # the untimed calls of timed_region let a plan replay a launch sequence
    # it has seen twice (graph replay of executes): steady state is timed
    t_plain, reps_p, clk_p = timed_region(plain, stream, gpu, target_s=0.6, min_reps=2)
    comp = sum(2 * 8 * n for n in sizes)
    comp_all = sum_over_ranks(comp, dist)
    t_batch_all = max_over_ranks(t_batch, dist)
    t_plain_all = max_over_ranks(t_plain, dist)
    out = {
        "workload": f"{count} seeded uneven 2-D/3-D complex64 forward transforms (extents "
                    "log-uniform in [16,256] over 7-smooth lengths, 5% primes), iid U[-1,1)",
        "metric": "compulsory GB/s", "unit": "GB/s",
        "value": comp_all / (t_batch_all / 1e3) / 1e9, "plain_value": comp_all / (t_plain_all / 1e3) / 1e9,
        "speedup_vs_plain": t_plain_all / t_batch_all, "ms_batched": t_batch_all, "ms_plain": t_plain_all,
        "reps": {"batched": reps_b, "plain": reps_p},
        "transforms_per_rank": len(shapes), "elements_rank0": sum(sizes),
        "plan_hbm_gbs_batched": batch.alg_bytes / (t_batch / 1e3) / 1e9,
        "launches_batched_per_execute": 1, "launches_plain_per_execute": launches,
        "create_s": {"batch_with_autotune": t_create, "plain_plans": t_plans},
        "batch": batch.describe(), "max_rel_l2_sample": max(e for e, _ in errs),
        "errors_within_tol": all(e <= t for e, t in errs), "sample": len(errs),
        "tol": "1e-6*log2(N) per transform",
        "clocks": {"batched": clk_b, "plain": clk_p},
    }
    batch.destroy()
    for p in plans.values():
        p.destroy()
    del src, dst, scr
    torch.cuda.empty_cache()
    return out


def suite_batched(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank, world, local, dist = dist_init("nccl")
    out = batched_form(args.count, local, rank, world, dist)
    out["n_gpus"] = world
    if rank == 0:
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


def served_form(count, gpu, loads=(0.5, 1.0, 2.0, 4.0, 8.0), rank=0, world=1, dist=None):
    """C5: the seeded request mix through the serving loop
    (shafft_sm100_server_*, 40 GB budget, 8 streams) at Poisson offered
    loads given as multiples of the serial rate, against the same requests
    run one by one through resident plain plans (H2D, execute, D2H)."""
    import numpy as np
    import torch

    from shafft_b200 import _sm100
    reqs = shard(serve_requests(count * world), rank, world)
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
    clk = ClockSampler(gpu)
    clk.start()
    time.sleep(0.15)
    t0 = time.perf_counter()
    lat = [serial_one(d, p, r) for d, p, r in reqs]
    serial_s = time.perf_counter() - t0
    clk.stop()
    serial_tput = len(reqs) / serial_s
    lat.sort()
    serial = {"throughput_per_s": serial_tput, "p50_ms": lat[len(lat) // 2],
              "p99_ms": lat[min(len(lat) - 1, int(0.99 * (len(lat) - 1) + 0.5))],
              "clocks": clk.summary()}
    for p in plans.values():
        p.destroy()
    del plans, dev, dev2
    torch.cuda.empty_cache()
    srv = _sm100.Server(budget_bytes=40 << 30, streams=8)
    # warm the server's plan cache with one pass over the mix
    ids = [srv.submit(d, p, r, 1.0, hin.data_ptr(), hout.data_ptr()) for d, p, r in reqs]
    for i in ids:
        srv.wait(i)
    rng = np.random.Generator(np.random.MT19937(5))
    sweep = []
    for mult in loads:
        rate = mult * serial_tput
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        srv.reset_stats()
        clk = ClockSampler(gpu)
        clk.start()
        time.sleep(0.15)
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
        clk.stop()
        st = srv.stats()
        st["offered_x_serial"] = mult
        st["offered_per_s"] = rate
        st["achieved_per_s"] = len(reqs) / wall
        st["clocks"] = clk.summary()
        sweep.append(st)
    srv.destroy()
    best = max(s["achieved_per_s"] for s in sweep)
    best_all = sum_over_ranks(best, dist)
    serial_all = sum_over_ranks(serial_tput, dist)
    low = min(sweep, key=lambda s: s["offered_x_serial"])
    return {"workload": f"{len(reqs)} seeded requests per rank: 1-D 2^10-2^22, 2-D 64^2-2048^2, "
                        "3-D 32^3-384^3, 30% complex128, 10% prime lengths, fwd/bwd 50/50; "
                        "pinned host buffers; Poisson arrivals",
            "metric": "served requests/s (best over the offered loads) and p50/p99 latency",
            "unit": "requests/s", "value": best_all, "serial_plain": serial,
            "speedup_vs_serial": best_all / serial_all,
            "p99_below_saturation_vs_serial": low["p99_ms"] / serial["p99_ms"],
            "p50_below_saturation_ms": low["p50_ms"], "p99_below_saturation_ms": low["p99_ms"],
            "requests_per_rank": len(reqs), "budget_bytes": 40 << 30, "streams": 8, "sweep": sweep,
            "results": "bit-identical alone and in the mix (tests/test_gpu_serve.py)"}


def suite_serve(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank, world, local, dist = dist_init("nccl")
    out = served_form(max(40, min(args.count, 400)), local, rank=rank, world=world, dist=dist)
    out["n_gpus"] = world
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


CONFIG_ROWS = [((256, 256, 256), 1), ((64, 64, 32), 0), ((1 << 24,), 0), ((1 << 24,), 1),
               ((1488375,), 0), ((1488375,), 1), ((1000003,), 0), ((1000003,), 1)]


def configs_rows(args, gpu, rows=CONFIG_ROWS):
    """The other configurations: fwd+bwd time (plain kernels, graph replay
    on as by default, CUDA events, clocks sampled), plan traffic, and the
    forward error against the oracle (FP64 for complex64, x87 long double
    for complex128) with its tolerance."""
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    stream = torch.cuda.current_stream()
    peak, _ = peaks()
    res = []
    for dims, prec in rows:
        n = math.prod(dims)
        es = 16 if prec else 8
        x = o.uniform_input(dims, seed=42, dtype=np.complex128 if prec else np.complex64)
        a = torch.from_numpy(x.ravel()).cuda()
        b = torch.empty_like(a)
        p = _sm100.Plan(dims, prec)
        p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
        y = b.cpu().numpy()
        err = o.rel_l2(y, o.fftn(x.astype(np.complex128), precise=bool(prec)).ravel())
        del y

        def fwd_bwd():
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        ms, reps, clk = timed_region(fwd_bwd, stream, gpu)
        plan_bytes = 2 * sum(p.step_bytes(i) for i in range(p.launches))
        tol = (1e-14 if prec else 1e-6) * math.log2(n)
        res.append({"dims": list(dims), "precision": "c128" if prec else "c64", "ms_fwd_bwd": ms,
                    "reps": reps, "compulsory_gbs": 2 * 2 * es * n / (ms / 1e3) / 1e9,
                    "plan_gbs": plan_bytes / (ms / 1e3) / 1e9,
                    "pct_hbm_plan": 100 * plan_bytes / (ms / 1e3) / 1e9 / peak,
                    "launches_per_transform": p.launches, "passes_per_transform": p.passes,
                    "rel_l2_fwd_vs_oracle": err, "tol": tol, "within_tol": err <= tol,
                    "clocks": clk})
        p.destroy()
        del a, b
        torch.cuda.empty_cache()
    return res


def r2c_row(gpu, dims=(256, 256, 256)):
    """Real-to-complex then complex-to-real (fused 1/N) of a float tensor:
    fwd+bwd time, spectrum error against the oracle, round-trip error."""
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    stream = torch.cuda.current_stream()
    n = math.prod(dims)
    H = dims[-1] // 2
    rng = np.random.Generator(np.random.MT19937(42))
    x = rng.uniform(-1, 1, size=dims).astype(np.float32)
    plan = _sm100.RPlan(dims, 0)
    xin = torch.from_numpy(x.copy()).cuda()
    spec = torch.empty(plan.spectrum_elements, dtype=torch.complex64, device="cuda")
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    plan.r2c(xin.data_ptr(), spec.data_ptr(), 1.0, stream.cuda_stream)
    ref = o.fftn(x.astype(np.complex128))[..., :H + 1]
    err = o.rel_l2(spec.cpu().numpy().reshape(ref.shape), ref)
    del ref
    plan.c2r(spec.data_ptr(), y.data_ptr(), 1.0 / n, stream.cuda_stream)
    rt = o.rel_l2(y.cpu().numpy().reshape(dims), x)

    def fwd_bwd():
        plan.r2c(y.data_ptr(), spec.data_ptr(), 1.0, stream.cuda_stream)
        plan.c2r(spec.data_ptr(), y.data_ptr(), 1.0 / n, stream.cuda_stream)
    ms, reps, clk = timed_region(fwd_bwd, stream, gpu)
    plan.destroy()
    tol = 1e-6 * math.log2(n)
    return {"dims": list(dims), "precision": "f32 -> c64 (R2C / C2R)", "ms_fwd_bwd": ms, "reps": reps,
            "compulsory_gbs": 2 * (4 * n + 8 * n // dims[-1] * (H + 1)) / (ms / 1e3) / 1e9,
            "rel_l2_fwd_vs_oracle": err, "roundtrip_rel_l2": rt, "tol": tol,
            "within_tol": err <= tol and rt <= tol, "clocks": clk}


def suite_configs(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    print(json.dumps({"metric": "other configurations (512^3 aside): fwd+bwd time and error",
                      "configs": configs_rows(args, local) + [r2c_row(local)]}), flush=True)
    return 0


TC_SHAPES = [(1 << 24,), (1488375,), (1000003,), (64, 64, 32), (512, 512, 512), (65536, 61), (65536, 47),
             (65536, 31), (65536, 17), (4096, 61, 16), (61, 61, 61), (53, 59, 61)]


def tc_form(shapes, gpu, per_step=False):
    """Tensor-core form (tcgen05 split-FP16 DFT stages) against the plain
    kernels on the same GPU: fwd+bwd time with clocks, and the forward error
    of both forms against the FP64 oracle.  Where the plan has axes with a
    prime factor above 13, also the hybrid plan (tensor cores on those axes
    only)."""
    import numpy as np
    import torch

    from oracle import oracle as o
    from shafft_b200 import _sm100
    stream = torch.cuda.current_stream()
    peak, _ = peaks()
    res = []

    def run(dims, x, flags, ref):
        n = math.prod(dims)
        a = torch.from_numpy(x.ravel()).cuda()
        b = torch.empty_like(a)
        p = _sm100.Plan(dims, 0, flags)
        p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
        p.status()
        err = o.rel_l2(b.cpu().numpy(), ref.ravel())
        a.copy_(torch.from_numpy(x.ravel()))

        def fwd_bwd():
            p.execute(a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
            p.execute(b.data_ptr(), a.data_ptr(), 1, 1.0 / n, stream.cuda_stream)
        ms, reps, clk = timed_region(fwd_bwd, stream, gpu)
        p.status()
        plan_bytes = sum(p.step_bytes(i) for i in range(p.launches))
        out = {"ms_fwd_bwd": ms, "reps": reps, "compulsory_gbs": 2 * 2 * 8 * n / (ms / 1e3) / 1e9,
               "plan_gbs": 2 * plan_bytes / (ms / 1e3) / 1e9,
               "pct_hbm_plan": 100 * 2 * plan_bytes / (ms / 1e3) / 1e9 / peak,
               "launches": p.launches, "rel_l2_fwd_vs_fp64_oracle": err, "clocks": clk}
        if per_step:
            steps = p.describe()["steps"]
            per = []
            for i in range(p.launches):
                def one(i=i):
                    p.execute_step(i, a.data_ptr(), b.data_ptr(), 0, 1.0, stream.cuda_stream)
                t, _, _ = timed_region(one, stream, gpu, target_s=0.05)
                st = steps[i]
                per.append({"kind": st["kind"], "L": st.get("L"), "tc": st.get("tc", 0), "ms": t,
                            "gbs": p.step_bytes(i) / (t / 1e3) / 1e9})
            out["steps"] = per
        del a, b
        p.destroy()
        torch.cuda.empty_cache()
        return out

    for dims in shapes:
        n = math.prod(dims)
        x = o.uniform_input(dims, seed=42, dtype=np.complex64)
        ref = o.fftn(x.astype(np.complex128))
        tol = 1e-6 * math.log2(n)
        plain = run(dims, x, 0, ref)
        tc = run(dims, x, _sm100.PLAN_TENSOR_CORE, ref)
        row = {"dims": list(dims), "tol": tol, "plain": plain, "tensor_core": tc,
               "speedup_tc_vs_plain": plain["ms_fwd_bwd"] / tc["ms_fwd_bwd"],
               "within_tol": plain["rel_l2_fwd_vs_fp64_oracle"] <= tol
               and tc["rel_l2_fwd_vs_fp64_oracle"] <= tol}
        if any(s.get("tc") for s in _sm100.plan_query(dims, 0, _sm100.PLAN_TC_PRIME_AXES)["steps"]):
            hy = run(dims, x, _sm100.PLAN_TC_PRIME_AXES, ref)
            row["tc_prime_axes"] = hy
            row["speedup_hybrid_vs_plain"] = plain["ms_fwd_bwd"] / hy["ms_fwd_bwd"]
            row["within_tol"] = row["within_tol"] and hy["rel_l2_fwd_vs_fp64_oracle"] <= tol
        res.append(row)
    return res


def suite_tc(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    print(json.dumps({"metric": "tensor-core split-FP16 form vs plain FP32 kernels, complex64 fwd+bwd",
                      "configs": tc_form(TC_SHAPES, local, per_step=True),
                      "data": "synthetic, iid uniform[-1,1) seed 42"}), flush=True)
    return 0


def exchange_rows(gpu, cases=((256, 2), (128, 4), (64, 8))):
    """The local device steps before a slab exchange of 512^3 complex64 on
    P ranks (one rank's block of 512/P x 512 x 512: axes 1 and 2, then the
    pack of the last axis into P per-peer blocks, the axis the exchange
    distributes): the plain subplan followed by the separate pack kernel
    against the subplan with the pack fused into its last pass's stores.
    Both outputs are compared."""
    import torch

    from shafft_b200.slab import CudaOps
    ops = CudaOps(0)
    stream = torch.cuda.current_stream()
    rows = []
    for m, parts in cases:
        dims = [m, 512, 512]
        n = math.prod(dims)
        g = torch.Generator(device="cuda").manual_seed(7)
        x0 = (torch.rand(2 * n, device="cuda", generator=g) * 2 - 1).view(torch.complex64)
        a, b, c = torch.empty_like(x0), torch.empty_like(x0), torch.empty_like(x0)
        h0 = ops.plan(dims, [1, 2])
        h1, fused = ops.plan_mapped(dims, [1, 2], None, (m * 512, 512, 1, parts))

        def separate():
            ops.execute(h0, a, b, 0)
            ops.pack(b, c, m * 512, 512, 1, parts)

        def fused_step():
            ops.execute(h1, a, b, 0)
        a.copy_(x0)
        separate()
        ref = c.clone()
        a.copy_(x0)
        fused_step()
        err = float((torch.linalg.vector_norm(b - ref) / torch.linalg.vector_norm(ref)).item())
        del ref
        ms_sep, reps_sep, clk_sep = timed_region(separate, stream, gpu)
        ms_fused, reps_fused, clk_fused = timed_region(fused_step, stream, gpu)
        ops.destroy(h0)
        ops.destroy(h1)
        rows.append({"ranks": parts, "local_block": dims, "fused_bits": fused,
                     "ms_subplan_plus_pack": ms_sep, "ms_fused": ms_fused, "speedup": ms_sep / ms_fused,
                     "rel_l2_fused_vs_separate": err, "tol": 1e-6 * math.log2(n),
                     "clocks": {"separate": clk_sep, "fused": clk_fused}})
        del x0, a, b, c
        torch.cuda.empty_cache()
    return rows


def suite_exchange(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    print(json.dumps({"metric": "device steps before a slab exchange (512^3 complex64): subplan + pack "
                                "vs the pack fused into the subplan's stores",
                      "unit": "ms", "configs": exchange_rows(local),
                      "data": "synthetic, iid uniform[-1,1)"}), flush=True)
    return 0


def forms(args, gpu):
    """The three forms (tensor cores, batched, served) against the plain kernels on this GPU, each
    timing with its own clock record and its error against the oracle:
    tensor cores (one prime-axis shape, FFT1D 2^24), batched (C4) and
    served (C5, one offered load below saturation and one at it)."""
    t0 = time.perf_counter()
    out = {"tensor_core": tc_form([(65536, 61), (1 << 24,)], gpu)}
    t1 = time.perf_counter()
    out["batched"] = batched_form(args.count, gpu)
    t2 = time.perf_counter()
    out["served"] = served_form(400, gpu, loads=(0.5, 8.0))
    out["wall_s"] = {"tensor_core": t1 - t0, "batched": t2 - t1, "served": time.perf_counter() - t2}
    return out


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
    if args.suite == "exchange":
        return suite_exchange(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
