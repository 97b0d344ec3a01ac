"""Exchange block maps fused into a plan (shafft_sm100_plan_create_axes_mapped):
the mapped plan's output equals the plain plan's output packed into the
per-peer blocks of shafft_sm100_pack_blocks (store map), and a plan that
loads packed blocks equals the plain plan on the unpacked input (load map);
both against the oracle too.  Tolerances as in the other parity tests:
1e-6*log2(N) for complex64, 1e-14*log2(N) for complex128."""
import ctypes
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


def blocks_np(x, outer, n, inner, parts):
    """numpy restatement of the block layout (the reference's partition)."""
    from shafft_b200.slab import block_partition
    a = x.reshape(outer, n, inner)
    return np.concatenate([a[:, s:s + l, :].ravel() for l, s in (block_partition(n, parts, p)
                                                                for p in range(parts))])


# (dims, axes, map over the local block, which side, fused bit expected)
CASES = [
    ((8, 64, 32), [1, 2], (512, 32, 1, 2), "store", 2),     # slab: pack of the last axis after axes 1, 2
    ((16, 64, 32), [1, 2], (1024, 32, 1, 4), "load", 1),    # slab backward: unpack of the last axis
    ((8, 64, 32), [1, 2], (8, 64, 32, 2), "store", 2),      # pack along axis 1
    ((16, 128, 64), [1, 2], (16, 128, 64, 4), "store", 2),
    ((4, 32, 16, 32), [2, 3], (128, 16, 32, 8), "store", 2),
    ((64, 8, 32), [0], (1, 64, 256, 2), "load", 1),         # outer = 1: blocks are row ranges
    ((32, 4, 64), [0], (32, 4, 64, 2), "load", 1),          # column pass reads blocks of axis 1
    ((32, 4, 64), [0], (32, 4, 64, 2), "store", 2),
    ((12, 64, 32), [1, 2], (12, 64, 32, 2), "store", 2),    # outer not a power of two: fine
    ((16, 64, 32), [1, 2], (16, 64, 32, 2), "load", 1),     # slab backward: column pass first, reads blocks
    ((16, 256, 128), [1, 2], (16, 256, 128, 4), "load", 1),
    ((8, 48, 32), [1, 2], (8, 48, 32, 2), "store", 0),      # n = 48: separate kernels
]


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("dims,axes,m,side,bit", CASES)
def test_mapped_plan_matches_plain_plan_and_blocks(dims, axes, m, side, bit, prec):
    import torch
    from shafft_b200.slab import CudaOps
    ops = CudaOps(prec)
    n = math.prod(dims)
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=n % 97, dtype=dt)
    h0 = ops.plan(list(dims), axes)
    load = m if side == "load" else None
    store = m if side == "store" else None
    if m[0] * m[1] * m[2] != n:
        with pytest.raises(RuntimeError):
            ops.plan_mapped(list(dims), axes, load, store)
        ops.destroy(h0)
        return
    h1, fused = ops.plan_mapped(list(dims), axes, load, store)
    assert fused == bit, fused
    ref = o.fft_axes(x.astype(np.complex128), axes, precise=(prec == S.Z2Z))
    for direction in (S.FORWARD, S.BACKWARD):
        a = torch.from_numpy(x.ravel().copy()).cuda()
        b = torch.empty_like(a)
        ops.execute(h0, a, b, direction)
        plain = b.cpu().numpy()
        src = blocks_np(x.ravel(), *m) if (side == "load" and bit) else x.ravel()
        a = torch.from_numpy(np.ascontiguousarray(src)).cuda()
        c = torch.empty_like(a)
        ops.execute(h1, a, c, direction)
        torch.cuda.synchronize()
        got = c.cpu().numpy()
        want = blocks_np(plain, *m) if (side == "store" and bit) else plain
        assert o.rel_l2(got, want) <= tol(n, prec), (direction, o.rel_l2(got, want))
        if direction == S.FORWARD:
            oref = ref.ravel()
            if side == "store" and bit:
                oref = blocks_np(oref, *m)
            assert o.rel_l2(got, oref) <= tol(n, prec)
    ops.destroy(h0)
    ops.destroy(h1)


def test_invalid_maps_are_refused():
    import torch  # noqa: F401
    from shafft_b200.slab import CudaOps
    ops = CudaOps(S.C2C)
    for bad in [(8, 64, 32, 0 - 1), (8, 64, 32, 65), (8, 64, 16, 2)]:
        with pytest.raises(RuntimeError):
            ops.plan_mapped([8, 64, 32], [1, 2], None, bad)
