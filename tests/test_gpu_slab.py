"""GPU parts of the distributed (slab-decomposed) FFTND: kernel-library plans
over axis subsets, block pack/unpack, and the whole transform on two
processes.  The two ranks share this run's one GPU; their kernels are
independent (nothing on the device waits for the other rank) and the
exchange goes through host memory on a gloo group.  Tolerances as in the
other parity tests: 1e-6*log2(N) (C2C), 1e-14*log2(N) (Z2Z)."""
import json
import math
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


@pytest.mark.parametrize("dims,axes", [((6, 40, 48), [1, 2]), ((64, 5, 7), [0]), ((8, 12, 10, 6), [1, 3]),
                                       ((97, 33), [1]), ((16, 16), [])])
@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
def test_axis_subset_plans_vs_oracle(dims, axes, prec):
    from shafft_b200.slab import CudaOps
    import torch
    ops = CudaOps(prec)
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=3, dtype=dt)
    a = torch.from_numpy(x.ravel()).cuda()
    b = torch.empty_like(a)
    h = ops.plan(list(dims), axes)
    ops.execute(h, a, b, S.FORWARD)
    torch.cuda.synchronize()
    y = b.cpu().numpy().reshape(dims)
    ref = o.fft_axes(x.astype(np.complex128), axes, precise=(prec == S.Z2Z)) if axes else x
    assert o.rel_l2(y, ref) <= tol(x.size, prec)
    ops.destroy(h)


@pytest.mark.parametrize("outer,n,inner,P", [(6, 48, 1, 2), (5, 7, 1, 3), (1, 10, 1, 4), (33, 64, 1, 8),
                                             (4, 10, 6, 3), (3, 7, 5, 2)])
def test_pack_unpack_blocks(outer, n, inner, P):
    from shafft_b200.slab import CudaOps, block_partition
    import torch
    ops = CudaOps(S.C2C)
    x = o.uniform_input((outer, n, inner), seed=1, dtype=np.complex64)
    a = torch.from_numpy(x.ravel()).cuda()
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    ops.pack(a, b, outer, n, inner, P)
    ops.unpack(b, c, outer, n, inner, P)
    torch.cuda.synchronize()
    want = np.concatenate([x[:, s:s + l, :].ravel() for l, s in (block_partition(n, P, p) for p in range(P))])
    assert np.array_equal(b.cpu().numpy(), want)
    assert np.array_equal(c.cpu().numpy(), x.ravel())


WORKER = r'''
import json, math, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch, torch.distributed as dist
import shafft_b200 as S
from shafft_b200 import slab
from oracle import oracle as o
cfg = json.loads(sys.argv[3])
torch.cuda.set_device(0)
dist.init_process_group("gloo")
dims, prec, P = tuple(cfg["dims"]), cfg["prec"], cfg["P"]
cdims = cfg.get("comm_dims") or [P] + [1] * (len(dims) - 1)
dt = np.complex128 if prec == S.Z2Z else np.complex64
g = o.uniform_input(dims, seed=42, dtype=dt)
ref = o.fftn(g.astype(np.complex128), precise=(prec == S.Z2Z))
plan = slab.FFTND()
assert plan.init(cdims, dims, prec, None, cfg["policy"]) == 0
assert plan.plan() == 0
fused = sum(1 for v in plan._variants.values() if v)
n = plan.alloc_size()
tdt = torch.complex128 if prec == S.Z2Z else torch.complex64
a = torch.zeros(n, dtype=tdt, device="cuda"); b = torch.zeros_like(a)
assert plan.set_buffers(a, b) == 0
_, sub, off = plan.get_layout(S.TENSOR_LAYOUT_INITIAL)
sl = lambda sub, off: tuple(slice(q, q + s) for q, s in zip(off, sub))
_, d, _ = plan.get_buffers(); d[:math.prod(sub)] = torch.from_numpy(np.ascontiguousarray(g[sl(sub, off)]).ravel()).cuda()
assert plan.execute(S.FORWARD) == 0
_, sub, off = plan.get_layout()
_, d, _ = plan.get_buffers()
y = d[:math.prod(sub)].cpu().numpy().reshape(sub)
r = ref[sl(sub, off)]
fwd_layout = [sub, off]
err2 = float(np.sum(np.abs(y - r) ** 2)); ref2 = float(np.sum(np.abs(r) ** 2))
assert plan.execute(S.BACKWARD) == 0
assert plan.normalize() == 0
_, sub, off = plan.get_layout()
_, d, _ = plan.get_buffers()
back = d[:math.prod(sub)].cpu().numpy().reshape(sub)
bt2 = float(np.sum(np.abs(back - g[sl(sub, off)]) ** 2)); g2 = float(np.sum(np.abs(g[sl(sub, off)]) ** 2))
plan.release()
dist.destroy_process_group()
json.dump({"err2": err2, "ref2": ref2, "bt2": bt2, "g2": g2, "fwd_layout": fwd_layout, "fused": fused},
          open(sys.argv[2], "w"))
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("dims,prec,policy", [((64, 48, 40), S.C2C, S.LAYOUT_REDISTRIBUTED),
                                              ((64, 48, 40), S.Z2Z, S.LAYOUT_INITIAL),
                                              ((97, 36, 10), S.C2C, S.LAYOUT_INITIAL),
                                              ((128, 96), S.C2C, S.LAYOUT_REDISTRIBUTED)])
def test_distributed_fftnd_two_ranks(tmp_path, dims, prec, policy):
    _run_nd(tmp_path, 2, {"dims": list(dims), "prec": prec, "P": 2, "policy": policy})


@pytest.mark.parametrize("world,comm_dims,dims,prec,policy", [
    (2, [2, 1, 1], (64, 128, 64), S.C2C, S.LAYOUT_REDISTRIBUTED),
    (2, [2, 1, 1], (32, 64, 128), S.Z2Z, S.LAYOUT_INITIAL),
    (4, [4, 1, 1], (64, 64, 32), S.C2C, S.LAYOUT_INITIAL),
    (2, [2, 1, 1], (128, 64, 256), S.C2C, S.LAYOUT_REDISTRIBUTED),
    (4, [2, 2, 1], (64, 32, 64), S.C2C, S.LAYOUT_REDISTRIBUTED),
    (4, [2, 2, 1, 1], (16, 32, 16, 32), S.Z2Z, S.LAYOUT_INITIAL)])
def test_distributed_fftnd_fused_packing(tmp_path, world, comm_dims, dims, prec, policy):
    """Power-of-two shapes: the pack of every exchange that needs one is
    fused into the stores of the subplan before it (and an unpack into the
    loads of the subplan after it where that subplan starts with an
    out-of-place specialised pass); results against the oracle as above."""
    res = _run_nd(tmp_path, world, {"dims": list(dims), "prec": prec, "P": comm_dims[0],
                                     "comm_dims": comm_dims, "policy": policy})
    assert all(x["fused"] >= 1 for x in res), res


@pytest.mark.parametrize("dims,prec,policy", [((64, 48, 40), S.C2C, S.LAYOUT_REDISTRIBUTED),
                                              ((30, 28, 26), S.Z2Z, S.LAYOUT_INITIAL)])
def test_pencil_fftnd_four_ranks(tmp_path, dims, prec, policy):
    """commDims [2, 2, 1]: two exchange sequences inside 2-rank grid lines."""
    res = _run_nd(tmp_path, 4, {"dims": list(dims), "prec": prec, "P": 2, "comm_dims": [2, 2, 1],
                                "policy": policy})
    if policy == S.LAYOUT_REDISTRIBUTED:  # full axis 0, axes 1 and 2 in blocks
        assert all(x["fwd_layout"][0][0] == dims[0] for x in res)


def _run_nd(tmp_path, world, cfg):
    dims, prec, policy = tuple(cfg["dims"]), cfg["prec"], cfg["policy"]
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(tmp_path / f"r{r}.json"),
                                       json.dumps(cfg)], env=env))
    for p in procs:
        assert p.wait(timeout=300) == 0
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    n = math.prod(dims)
    # global relative L2 error over both ranks' blocks
    err = math.sqrt(sum(x["err2"] for x in res) / sum(x["ref2"] for x in res))
    back = math.sqrt(sum(x["bt2"] for x in res) / sum(x["g2"] for x in res))
    assert err <= tol(n, prec), err
    assert back <= 2 * tol(n, prec), back
    if policy == S.LAYOUT_REDISTRIBUTED and "comm_dims" not in cfg:
        # slab forward output: full axis 0, the last axis in blocks
        assert all(x["fwd_layout"][0][0] == dims[0] for x in res)
        assert sum(x["fwd_layout"][0][-1] for x in res) == dims[-1]
    elif "comm_dims" not in cfg:
        assert sum(x["fwd_layout"][0][0] for x in res) == dims[0]
    return res


WORKER_1D = r'''
import json, math, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch, torch.distributed as dist
import shafft_b200 as S
from shafft_b200 import slab
from oracle import oracle as o
cfg = json.loads(sys.argv[3])
torch.cuda.set_device(0)
dist.init_process_group("gloo")
r, P = dist.get_rank(), dist.get_world_size()
N, prec = cfg["n"], cfg["prec"]
ln, ls, la, active = slab.configuration_1d(N, P, r)
dt = np.complex128 if prec == S.Z2Z else np.complex64
g = o.uniform_input((N,), seed=42, dtype=dt)
ref = o.fftn(g.astype(np.complex128), precise=(prec == S.Z2Z))[ls:ls + ln]
plan = slab.FFT1D()
assert plan.init(N, ln, ls, prec) == 0
assert plan.plan() == 0
path = plan.path if r < active else None
tdt = torch.complex128 if prec == S.Z2Z else torch.complex64
a = torch.zeros(max(la, 1), dtype=tdt, device="cuda"); b = torch.zeros_like(a)
assert plan.set_buffers(a, b) == 0
a[:ln].copy_(torch.from_numpy(g[ls:ls + ln]).cuda())
assert plan.execute(S.FORWARD) == 0
_, d, _ = plan.get_buffers()
y = d[:ln].cpu().numpy()
err2 = float(np.sum(np.abs(y - ref) ** 2)); ref2 = float(np.sum(np.abs(ref) ** 2))
assert plan.execute(S.BACKWARD) == 0 and plan.normalize() == 0
_, d, _ = plan.get_buffers()
x = g[ls:ls + ln]
bt2 = float(np.sum(np.abs(d[:ln].cpu().numpy() - x) ** 2)); g2 = float(np.sum(np.abs(x) ** 2))
plan.release()
dist.destroy_process_group()
json.dump({"err2": err2, "ref2": ref2, "bt2": bt2, "g2": g2, "ln": ln, "path": path}, open(sys.argv[2], "w"))
'''


@pytest.mark.parametrize("world,n,prec,path", [
    (2, 1 << 20, S.C2C, "cooley_tukey"), (2, 121500, S.C2C, "cooley_tukey"), (2, 1 << 18, S.Z2Z, "cooley_tukey"),
    (3, 100003, S.C2C, "bluestein"),   # 2 active ranks (M = 200008), the third inactive
    (6, 100003, S.Z2Z, "bluestein"),   # 3 active ranks (M = 200007), three inactive
    (3, 1000, S.C2C, "cooley_tukey")])  # one inactive rank, four-step re-chosen for two
def test_distributed_fft1d(tmp_path, world, n, prec, path):
    """The reference's distributed FFT1D layout and both paths (four-step,
    Bluestein over it), every device step on the GPU that the ranks share."""
    script = tmp_path / "worker1d.py"
    script.write_text(WORKER_1D)
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(tmp_path / f"r{r}.json"),
                                       json.dumps({"n": n, "prec": prec})], env=env))
    for p in procs:
        assert p.wait(timeout=300) == 0
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    assert sum(x["ln"] for x in res) == n
    assert res[0]["path"] == path
    err = math.sqrt(sum(x["err2"] for x in res) / sum(x["ref2"] for x in res))
    back = math.sqrt(sum(x["bt2"] for x in res) / sum(x["g2"] for x in res))
    assert err <= tol(n, prec), err
    assert back <= 2 * tol(n, prec), back


def _chirp_ref(idx, n, sign):
    r = np.array([(int(k) * int(k)) % (2 * n) for k in idx], dtype=np.float64)
    return np.exp(sign * 1j * np.pi * r / n)


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("n,m,n0,m0,count", [(1001, 2004, 0, 0, 1002), (1001, 2004, 1001, 1002, 1002),
                                             (100003, 200007, 66669, 66669, 66669),
                                             ((1 << 31) - 1, 1 << 32, (1 << 31) - 40, (1 << 32) - 44, 64)])
def test_bluestein_chirp_kernels(prec, n, m, n0, m0, count):
    """shafft_sm100_bluestein_chirps (exact n^2 mod 2N phases, also near
    N = 2^31) and shafft_sm100_chirp_multiply against numpy."""
    from shafft_b200.slab import CudaOps
    import torch
    ops = CudaOps(prec)
    b, v = ops.empty(count), ops.empty(count)
    ops.chirps(b, v, n, m, n0, m0, count)
    i = np.arange(count, dtype=np.int64)
    k = n0 + i
    b_ref = np.where(k < n, _chirp_ref(np.minimum(k, n - 1), n, -1), 0)
    mm = m0 + i
    j = np.where(mm < n, mm, np.where((mm > m - n) & (mm < m), m - mm, -1))
    v_ref = np.where(j >= 0, _chirp_ref(np.maximum(j, 0), n, 1), 0)
    t = 2e-7 if prec == S.C2C else 4e-15  # a few ulp: sincospi on the GPU, exp in numpy
    assert np.abs(b.cpu().numpy() - b_ref).max() <= t
    assert np.abs(v.cpu().numpy() - v_ref).max() <= t
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input((count,), seed=5, dtype=dt)
    xs = torch.from_numpy(x).cuda()
    out = ops.empty(count)
    valid = count * 2 // 3
    for conj_in, conj_out, scale in ((0, 0, 1.0), (1, 0, 0.5), (0, 1, 1.0 / m), (1, 1, 3.0)):
        ops.chirp_mul(xs, out, b, count, valid, conj_in, conj_out, scale)
        a = np.conj(x) if conj_in else x
        want = a * b.cpu().numpy() * scale
        want = np.conj(want) if conj_out else want
        want[valid:] = 0
        got = out.cpu().numpy()
        assert np.abs(got - want).max() <= 4 * t * max(1.0, scale), (conj_in, conj_out, scale)
    ops.chirp_mul(xs, xs, v, count, count, 0, 0, 1.0)  # in place
    assert np.abs(xs.cpu().numpy() - x * v.cpu().numpy()).max() <= 4 * t
