"""Serving form (shafft_sm100_server_*): concurrent requests admitted under a
device-memory budget.  A request's result must be identical alone and in a
mix of overlapping requests, and correct against the oracle."""
import math

import numpy as np
import pytest

import shafft_b200 as S  # noqa: F401
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def pinned(x):
    t = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    return t


def test_alone_equals_mixed_and_matches_oracle():
    srv = _sm100.Server(budget_bytes=2 << 30, streams=4)
    probe_shape, probe_prec = (64, 64, 32), 0
    xp = o.uniform_input(probe_shape, seed=1, dtype=np.complex64)
    hin = pinned(xp)
    hout_alone = pinned(np.zeros_like(xp))
    rid = srv.submit(probe_shape, probe_prec, 0, 1.0, hin.data_ptr(), hout_alone.data_ptr())
    srv.wait(rid)
    alone = hout_alone.numpy().copy()
    # a mix of overlapping requests with the probe in the middle
    mix = [((1 << 14,), 0), ((96, 96), 1), ((32, 32, 32), 0), ((1009,), 0), ((128, 128), 0),
           ((48, 48, 48), 1), ((4096,), 1), ((97, 64), 0)]
    reqs = []
    for i, (shape, prec) in enumerate(mix * 3):
        dt = np.complex128 if prec else np.complex64
        x = o.uniform_input(shape, seed=10 + i, dtype=dt)
        a, b = pinned(x), pinned(np.zeros_like(x))
        direction = i % 2
        rid = srv.submit(shape, prec, direction, 1.0, a.data_ptr(), b.data_ptr())
        reqs.append((rid, x, a, b, prec, direction))
        if i == len(mix):
            hout_mix = pinned(np.zeros_like(xp))
            probe_id = srv.submit(probe_shape, probe_prec, 0, 1.0, hin.data_ptr(), hout_mix.data_ptr())
    for rid, x, a, b, prec, direction in reqs:
        srv.wait(rid)
        ref = o.fftn(x.astype(np.complex128), sign=-1 if direction == 0 else 1, precise=bool(prec))
        tol = (1e-6 if prec == 0 else 1e-14) * max(1.0, math.log2(x.size))
        assert o.rel_l2(b.numpy(), ref) <= tol
    srv.wait(probe_id)
    np.testing.assert_array_equal(hout_mix.numpy(), alone)
    st = srv.stats()
    assert st["completed"] == len(reqs) + 2 and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert st["max_inflight"] >= 2  # requests really overlapped
    srv.destroy()


def test_budget_too_small_fails_cleanly():
    srv = _sm100.Server(budget_bytes=1 << 20, streams=2)
    x = np.zeros((512, 512), np.complex64)  # 2 MiB per buffer > 1 MiB budget
    a, b = pinned(x), pinned(x)
    rid = srv.submit(x.shape, 0, 0, 1.0, a.data_ptr(), b.data_ptr())
    with pytest.raises(_sm100.Sm100Error):
        srv.wait(rid)
    srv.destroy()
