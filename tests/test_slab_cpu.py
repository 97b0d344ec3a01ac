"""Distributed (slab-decomposed) FFTND on CPU: the orchestration of
shafft_b200.slab.FFTND -- stage layouts, block packing, all-to-all counts,
buffer swaps, output layout policies, normalisation -- run on 2 and 3 gloo
ranks.  The device steps are replaced here by numpy (test infrastructure
only; the library's own steps are CUDA kernels, tested on the GPU in
tests/test_gpu_slab.py)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from shafft_b200 import slab  # noqa: E402

WORKER = r'''
import json, math, os, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch, torch.distributed as dist
import shafft_b200 as S
from shafft_b200 import slab

class NumpyOps:
    """Stand-in for the CUDA steps: numpy FFTs over axis subsets and the same
    block layout as shafft_sm100_pack_blocks; plan_mapped fuses every block
    map it is given (unpack before, pack after the FFT)."""
    def plan(self, dims, axes): return (tuple(dims), tuple(axes), None, None)
    def plan_mapped(self, dims, axes, load, store):
        return (tuple(dims), tuple(axes), load, store), (1 if load else 0) | (2 if store else 0)
    def destroy(self, h): pass
    def execute(self, h, src, dst, direction):
        dims, axes, load, store = h
        n = math.prod(dims)
        if load:
            tmp = torch.zeros(n, dtype=torch.complex128)
            self.unpack(src, tmp, *load)
            src = tmp
        x = src[:n].numpy().reshape(dims)
        if direction == S.FORWARD:
            y = np.fft.fftn(x, axes=axes)
        else:
            y = np.fft.ifftn(x, axes=axes) * math.prod(dims[a] for a in axes)
        y = torch.from_numpy(y.ravel().copy())
        if store:
            self.pack(y, dst, *store)
        else:
            dst[:n] = y
    def pack(self, src, dst, outer, n, inner, P):
        a = src[:outer * n * inner].numpy().reshape(outer, n, inner)
        parts = [a[:, s:s + l, :].ravel() for l, s in (slab.block_partition(n, P, p) for p in range(P))]
        dst[:outer * n * inner] = torch.from_numpy(np.concatenate(parts))
    def unpack(self, src, dst, outer, n, inner, P):
        out = np.empty((outer, n, inner), dtype=np.complex128); pos = 0
        for p in range(P):
            l, s = slab.block_partition(n, P, p)
            out[:, s:s + l, :] = src[pos:pos + outer * l * inner].numpy().reshape(outer, l, inner)
            pos += outer * l * inner
        dst[:outer * n * inner] = torch.from_numpy(out.ravel())
    def scale(self, data, count, f): data[:count] *= f
    def twiddle(self, data, rows, cols, col0, n, sign):
        k = np.arange(rows)[:, None]; c = np.arange(cols)[None, :]
        m = ((col0 + c) * k) % n
        w = np.exp(sign * 2j * np.pi * m / n).ravel()
        data[:rows * cols] *= torch.from_numpy(w)
    def alltoall(self, out, inp, oc, ic, group, world):
        o = torch.view_as_real(out[:sum(oc)]).view(-1); i = torch.view_as_real(inp[:sum(ic)]).view(-1)
        dist.all_to_all_single(o, i, [2 * c for c in oc], [2 * c for c in ic], group=group)
    def empty(self, count): return torch.zeros(count, dtype=torch.complex128)
    def chirps(self, b, v, n, m, n0, m0, count):
        def chirp(idx, sign):
            r = (idx.astype(object) ** 2 % (2 * n)).astype(np.float64)
            return np.exp(sign * 1j * np.pi * r / n)
        i = np.arange(count, dtype=np.int64)
        if b is not None:
            k = n0 + i
            b[:count] = torch.from_numpy(np.where(k < n, chirp(np.minimum(k, n - 1), -1), 0))
        if v is not None:
            mm = m0 + i
            j = np.where(mm < n, mm, np.where((mm > m - n) & (mm < m), m - mm, -1))
            v[:count] = torch.from_numpy(np.where(j >= 0, chirp(np.maximum(j, 0), 1), 0))
    def chirp_mul(self, src, dst, f, count, valid, conj_in, conj_out, scale):
        a = src[:count].numpy().copy()
        if conj_in: a = np.conj(a)
        y = a * f[:count].numpy() * scale
        if conj_out: y = np.conj(y)
        y[valid:] = 0
        dst[:count] = torch.from_numpy(y)

class SeparateOps:
    """The same steps without plan_mapped: every exchange packs and unpacks
    with its own kernel."""
    def __init__(self): self._o = NumpyOps()
    def __getattr__(self, k):
        if k == "plan_mapped": raise AttributeError(k)
        return getattr(self._o, k)

cfg = json.loads(sys.argv[3])
make_ops = SeparateOps if cfg.get("separate") else NumpyOps
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
if cfg.get("fft1d"):
    N = cfg["n"]
    ln, ls, la, active = slab.configuration_1d(N, world, rank)
    rng = np.random.Generator(np.random.MT19937(9))
    g = rng.uniform(-1, 1, N) + 1j * rng.uniform(-1, 1, N)
    plan = slab.FFT1D()
    rc = plan.init(N, ln, ls, S.Z2Z, None, device_ops=NumpyOps())
    out = {"rank": rank, "init": rc, "local": [ln, ls, la, active]}
    if rc == 0:
        assert plan.plan() == 0
        out["path"] = plan.path
        assert plan.alloc_size() == la
        a = torch.zeros(max(la, 1), dtype=torch.complex128); b = torch.full_like(a, 7.0)
        assert plan.set_buffers(a, b) == 0
        _, d, _ = plan.get_buffers(); d[:ln] = torch.from_numpy(g[ls:ls + ln])
        assert plan.execute(S.FORWARD) == 0
        _, d2, _ = plan.get_buffers()
        out["swapped"] = d2.data_ptr() != d.data_ptr() or la == 0
        ref = np.fft.fft(g)[ls:ls + ln]
        out["fwd_err"] = float(np.abs(d2[:ln].numpy() - ref).max() / np.abs(np.fft.fft(g)).max()) if ln else 0.0
        assert plan.execute(S.BACKWARD) == 0 and plan.normalize() == 0
        _, d3, _ = plan.get_buffers()
        out["rt_err"] = float(np.abs(d3[:ln].numpy() - g[ls:ls + ln]).max()) if ln else 0.0
        plan.release()
    dist.destroy_process_group()
    json.dump(out, open(sys.argv[2], "w"))
    sys.exit(0)
dims = tuple(cfg["dims"]); P = cfg["P"]
cdims = cfg.get("comm_dims") or [P] + [1] * (len(dims) - 1)
rng = np.random.Generator(np.random.MT19937(5))
g = rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims)
f = S.__dict__
plan = slab.FFTND()
rc = plan.init(cdims, dims, S.Z2Z, None, cfg["policy"], device_ops=make_ops())
assert rc == 0, rc
assert plan.plan() == 0
fused_variants = sum(1 for v in plan._variants.values() if v)
n = plan.alloc_size()
a = torch.zeros(max(n, 1), dtype=torch.complex128); b = torch.zeros_like(a)
assert plan.set_buffers(a, b) == 0
rc, sub, off = plan.get_layout(S.TENSOR_LAYOUT_INITIAL)
sl = tuple(slice(o, o + s) for o, s in zip(off, sub))
loc = g[sl]
_, d, _ = plan.get_buffers(); d[:loc.size] = torch.from_numpy(loc.ravel())
assert plan.execute(S.FORWARD) == 0
rc, sub, off = plan.get_layout(S.TENSOR_LAYOUT_CURRENT)
_, d, _ = plan.get_buffers()
y = d[:math.prod(sub)].numpy().reshape(sub)
ref = np.fft.fftn(g)[tuple(slice(o, o + s) for o, s in zip(off, sub))]
fwd_err = float(np.abs(y - ref).max() / np.abs(ref).max()) if y.size else 0.0
cur_axes = plan.get_axes(S.TENSOR_LAYOUT_CURRENT)
assert plan.execute(S.BACKWARD) == 0
assert plan.normalize() == 0
rc, sub, off = plan.get_layout(S.TENSOR_LAYOUT_CURRENT)
_, d, _ = plan.get_buffers()
back = d[:math.prod(sub)].numpy().reshape(sub)
rt_err = float(np.abs(back - g[tuple(slice(o, o + s) for o, s in zip(off, sub))]).max()) if back.size else 0.0
dist.destroy_process_group()
json.dump({"rank": rank, "fwd_err": fwd_err, "rt_err": rt_err, "fwd_layout": [sub, off],
           "axes": cur_axes, "fused_variants": fused_variants}, open(sys.argv[2], "w"))
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(tmp_path, world, cfg):
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
        assert p.wait(timeout=240) == 0
    return [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]


@pytest.mark.parametrize("separate", [False, True])
@pytest.mark.parametrize("world,dims,policy", [
    (2, (6, 5, 7), 0), (2, (6, 5, 7), 1), (3, (7, 4, 5), 0), (3, (8, 6), 1), (2, (4, 3, 2, 5), 0)])
def test_slab_fftnd_on_gloo_ranks(tmp_path, world, dims, policy, separate):
    """Both forms of the exchanges' packing: fused into the neighbouring
    subplans (plan_mapped) and as separate pack / unpack steps."""
    res = _run(tmp_path, world, {"dims": list(dims), "P": world, "policy": policy, "separate": separate})
    for o in res:
        assert o["fwd_err"] < 1e-12, o
        assert o["rt_err"] < 1e-12, o
        assert (o["fused_variants"] == 0) == separate, o


def test_inactive_rank_owns_nothing(tmp_path):
    """commDims product below the group size: the extra rank owns nothing and
    belongs to no grid line."""
    res = _run(tmp_path, 3, {"dims": [4, 3, 5], "P": 2, "policy": 0})
    assert all(o["fwd_err"] < 1e-12 and o["rt_err"] < 1e-12 for o in res)


@pytest.mark.parametrize("world,comm_dims,dims,policy", [
    (4, [2, 2, 1], (8, 6, 10), 0),        # pencils: two exchange sequences
    (4, [2, 2, 1], (7, 5, 6), 1),         # uneven blocks, INITIAL output
    (6, [2, 3, 1], (8, 6, 10), 0),        # unequal grid dimensions
    (4, [2, 2, 1, 1], (8, 6, 10, 4), 0),  # nca = 2: one sequence of two exchanges
    (5, [2, 2, 1], (6, 4, 5), 1)])        # one inactive rank
@pytest.mark.parametrize("separate", [False, True])
def test_pencil_fftnd_on_gloo_ranks(tmp_path, world, comm_dims, dims, policy, separate):
    res = _run(tmp_path, world, {"dims": list(dims), "P": comm_dims[0], "comm_dims": comm_dims,
                                 "policy": policy, "separate": separate})
    for o in res:
        assert o["fwd_err"] < 1e-12, o
        assert o["rt_err"] < 1e-12, o


def test_layout_bookkeeping_matches_reference_partition():
    L = slab.SlabLayout((6, 5, 7), [3, 1, 1], 1)
    assert L.sub == [[2, 5, 7], [6, 5, 2]] and L.off == [[2, 0, 0], [0, 0, 3]]
    assert L.alloc_size() == 70
    j, a, b, Q, pack, unpack, send, recv = L.exchange(0)
    assert (j, a, b, Q) == (0, 2, 0, 3) and pack == (10, 7, 1) and unpack[0] == 1
    assert (send, recv) == ([30, 20, 20], [20, 20, 20])
    # pencils: rank 4 of a 2 x 3 grid on 8 x 6 x 10
    L = slab.SlabLayout((8, 6, 10), [2, 3, 1], 4)
    assert L.coords == [1, 1] and L.es == [1, 1] and L.tf_axes == [[2], [1], [0]]
    assert L.sub == [[4, 2, 10], [4, 6, 3], [8, 3, 3]]
    assert L.das == [[0, 1], [0, 2], [1, 2]] and L.grid_line(0) == [1, 4] and L.grid_line(1) == [3, 4, 5]
    assert [slab.block_partition(10, 4, r) for r in range(4)] == [(3, 0), (3, 3), (2, 6), (2, 8)]


def test_init_validation():
    import shafft_b200 as S
    p = slab.FFTND()
    assert p.init([1, 2], [8, 8]) == S.ERR_INVALID_DECOMP       # last axis distributed
    p = slab.FFTND()
    assert p.init([1], [8, 8]) == S.ERR_DIM_MISMATCH
    p = slab.FFTND()
    assert p.init([9, 1], [8, 8]) == S.ERR_INVALID_DECOMP       # more parts than rows
    p = slab.FFTND()
    assert p.init([2, 2, 1], [8, 8, 8]) == S.ERR_INVALID_DECOMP  # 4 grid ranks, 1 process
    p = slab.FFTND()
    assert p.init([2, 9, 1], [8, 9, 8]) == S.ERR_INVALID_DECOMP  # grid dim 1 > axis 2 later
    p = slab.FFTND()
    assert p.init([2, 1], [8, 8]) == S.ERR_INVALID_DECOMP       # 2 parts, 1 process
    p = slab.FFTND()
    assert p.plan() == S.ERR_PLAN_NOT_INIT


@pytest.mark.parametrize("world,n", [(2, 64), (3, 9 * 7), (2, 4 * 1000), (4, 16 * 5)])
def test_slab_fft1d_four_step_on_gloo_ranks(tmp_path, world, n):
    res = _run(tmp_path, world, {"fft1d": True, "n": n})
    for o in res:
        assert o["init"] == 0
        assert o["swapped"]
        assert o["fwd_err"] < 1e-12, o
        assert o["rt_err"] < 1e-12, o


@pytest.mark.parametrize("world,n,path,active", [
    (2, 6, "cooley_tukey", 1),      # Bluestein on 2 leaves rank 1 empty: one active rank
    (3, 1001, "bluestein", 2),      # M = 1004 over 2 active ranks, the second holding nothing
    (6, 1001, "bluestein", 3),      # ranks 0-2 active (669 + 332 + 0 points), 3-5 inactive
    (3, 1000, "cooley_tukey", 2),   # re-chosen for the 2 active ranks: 4 divides 1000
    (4, 97 * 13, "bluestein", 2)])
def test_slab_fft1d_bluestein_and_inactive_ranks(tmp_path, world, n, path, active):
    """Lengths that P^2 does not divide: the reference's layout query (empty
    blocks -> inactive ranks, path chosen again for the active ones) and
    path B, Bluestein over the distributed four-step."""
    res = _run(tmp_path, world, {"fft1d": True, "n": n})
    assert sum(o["local"][0] for o in res) == n
    for o in res:
        assert o["init"] == 0 and o["local"][3] == active
        assert o["local"] == list(slab.configuration_1d(n, world, o["rank"]))
        if o["rank"] < active:
            assert o["path"] == path
        assert o["fwd_err"] < 1e-12, o
        assert o["rt_err"] < 1e-12, o


def test_select_path_and_layout_rules():
    assert slab.select_path_1d(1 << 20, 2) == ("cooley_tukey", 1 << 20, 1 << 19)
    assert slab.select_path_1d(1000003, 4) == ("bluestein", 2000016, 500004)  # ceil(1999/16)*16
    assert slab.select_path_1d(7, 1) == ("cooley_tukey", 7, 7)
    # blocks of the re-chosen size, start clamped to N on empty active ranks
    assert [slab.configuration_1d(1001, 6, r) for r in range(6)] == [
        (669, 0, 669, 3), (332, 669, 669, 3), (0, 1001, 669, 3), (0, 0, 0, 3), (0, 0, 0, 3), (0, 0, 0, 3)]
    assert slab.configuration_1d(5, 1, 0) == (5, 0, 5, 1)


def test_configuration_nd_decomposition_search():
    """The restated configurationND: one rank resolves to all ones with
    nda 0 (the reference's single-rank result); slabs are preferred until
    per-axis caps force a second distributed axis; a requested nda is tried
    exactly; a valid user grid is kept, an invalid one falls back to the
    search; memory limits reject blocks that are too large."""
    cfg = slab.configuration_nd
    assert cfg((64, 64, 32), 1)[:3] == (0, [1, 1, 1], 0)
    assert cfg((64, 64, 32), 4)[:3] == (0, [4, 1, 1], 1)
    assert cfg((64, 64, 32), 4, strategy=slab.MINIMIZE_NDA)[:3] == (0, [4, 1, 1], 1)
    assert cfg((4, 64, 64), 8)[:3] == (0, [4, 2, 1], 2)
    assert cfg((8, 8, 8), 64)[:3] == (0, [8, 8, 1], 2)
    assert cfg((64, 64, 32), 4, nda=2)[:3] == (0, [2, 2, 1], 2)
    assert cfg((64, 64, 32), 4, comm_dims=[2, 2, 1])[:3] == (0, [2, 2, 1], 2)
    assert cfg((64, 64, 32), 3, comm_dims=[2, 2, 1])[:3] == (0, [3, 1, 1], 1)  # 4 > 3 ranks
    st, g, d, sub, off, act = cfg((10, 6, 4), 4, rank=3)
    assert (g, d, sub, off, act) == ([4, 1, 1], 1, [2, 6, 4], [8, 0, 0], 4)
    # 64^3 complex64 in two buffers over 2 ranks needs 2 MiB each: a 1 MiB
    # limit forces more ranks' worth of splitting than 2 can give
    assert cfg((64, 64, 64), 2, mem_limit=1 << 20)[0] != 0
    assert cfg((64, 64, 64), 2, mem_limit=4 << 20)[:3] == (0, [2, 1, 1], 1)
    assert [slab._dims_create(n, d) for n, d in ((4, 2), (12, 2), (8, 3), (6, 2))] == \
        [[2, 2], [4, 3], [2, 2, 2], [3, 2]]
