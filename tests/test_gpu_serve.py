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


def _check_result(x, b, prec, direction):
    ref = o.fftn(x.astype(np.complex128), sign=-1 if direction == 0 else 1, precise=bool(prec))
    tol = (1e-6 if prec == 0 else 1e-14) * max(1.0, math.log2(x.size))
    assert o.rel_l2(b.numpy(), ref) <= tol


@pytest.mark.timeout(300)
def test_plan_builds_run_beside_other_requests():
    """A request whose shape needs a new plan (built by the server's builder
    thread) does not hold back the requests queued behind it; every result
    is correct."""
    srv = _sm100.Server(budget_bytes=8 << 30, streams=4)
    small = (64, 64, 32)
    xs = o.uniform_input(small, seed=2, dtype=np.complex64)
    a0, b0 = pinned(xs), pinned(np.zeros_like(xs))
    srv.wait(srv.submit(small, 0, 0, 1.0, a0.data_ptr(), b0.data_ptr()))  # plan resident
    big = (256, 256, 128)
    xb = o.uniform_input(big, seed=3, dtype=np.complex64)
    ab, bb = pinned(xb), pinned(np.zeros_like(xb))
    rid_big = srv.submit(big, 0, 0, 1.0, ab.data_ptr(), bb.data_ptr())
    reqs = []
    for i in range(24):
        x = o.uniform_input(small, seed=100 + i, dtype=np.complex64)
        a, b = pinned(x), pinned(np.zeros_like(x))
        reqs.append((srv.submit(small, 0, i % 2, 1.0, a.data_ptr(), b.data_ptr()), x, a, b, i % 2))
    for rid, x, a, b, d in reqs:
        srv.wait(rid)
        _check_result(x, b, 0, d)
    srv.wait(rid_big)
    _check_result(xb, bb, 0, 0)
    st = srv.stats()
    assert st["failed"] == 0 and st["completed"] == 26
    assert st["plans_created"] >= 2
    srv.destroy()


@pytest.mark.timeout(300)
def test_tight_budget_alternating_shapes_evicts_and_completes():
    """A budget that holds one Bluestein plan (its scratch and kernel
    spectrum are several times the request's buffers) and its buffers at a
    time: alternating prime lengths must evict the other shape's idle plan
    (never the waiting request's own) and every request completes
    correctly."""
    A, B = (1000003,), (999983,)
    need = [2 * 8 * math.prod(s) + _sm100.Plan(s, 0).device_bytes for s in (A, B)]
    budget = max(need) + (1 << 20)
    assert budget < sum(need)
    srv = _sm100.Server(budget_bytes=budget, streams=2)
    reqs = []
    for i, s in enumerate([A, B, A, B, A, B]):
        x = o.uniform_input(s, seed=200 + i, dtype=np.complex64)
        a, b = pinned(x), pinned(np.zeros_like(x))
        reqs.append((srv.submit(s, 0, 0, 1.0, a.data_ptr(), b.data_ptr()), x, a, b))
    for rid, x, a, b in reqs:
        srv.wait(rid)
        _check_result(x, b, 0, 0)
    st = srv.stats()
    assert st["failed"] == 0 and st["completed"] == 6
    assert st["plans_evicted"] >= 1
    srv.destroy()


def test_large_requests_through_the_copy_pump():
    """Requests with buffers of 256 MiB or more go through the copy pump
    (pieces fed a few at a time, one large request per direction at a time,
    held back while smaller copies are pending).  Two of them overlapping
    each other and a stream of small requests: every result is bit-identical
    to the same request served alone, and the large ones match a plain plan
    execute."""
    shape = (256, 512, 256)  # 256 MiB of complex64
    n = math.prod(shape)
    srv = _sm100.Server(budget_bytes=8 << 30, streams=4)
    bigs = []
    for i in range(2):
        g = torch.Generator().manual_seed(100 + i)
        x = (torch.rand(2 * n, generator=g) * 2 - 1).view(torch.complex64).pin_memory()
        bigs.append((x, torch.empty_like(x).pin_memory(), i % 2))
    smalls = []
    for i in range(12):
        x = o.uniform_input((64, 128), seed=200 + i, dtype=np.complex64)
        smalls.append((pinned(x), pinned(np.zeros_like(x)), pinned(np.zeros_like(x))))
    # alone
    alone_big = []
    for x, out, d in bigs:
        rid = srv.submit(shape, 0, d, 1.0, x.data_ptr(), out.data_ptr())
        srv.wait(rid)
        alone_big.append(out.clone())
    for a, out_alone, _ in smalls:
        srv.wait(srv.submit((64, 128), 0, 0, 1.0, a.data_ptr(), out_alone.data_ptr()))
    # mixed: both large ones, small ones between them
    ids = [srv.submit(shape, 0, bigs[0][2], 1.0, bigs[0][0].data_ptr(), bigs[0][1].data_ptr())]
    for a, _, out_mix in smalls[:6]:
        ids.append(srv.submit((64, 128), 0, 0, 1.0, a.data_ptr(), out_mix.data_ptr()))
    ids.append(srv.submit(shape, 0, bigs[1][2], 1.0, bigs[1][0].data_ptr(), bigs[1][1].data_ptr()))
    for a, _, out_mix in smalls[6:]:
        ids.append(srv.submit((64, 128), 0, 0, 1.0, a.data_ptr(), out_mix.data_ptr()))
    for rid in ids:
        srv.wait(rid)
    for (x, out, d), ref in zip(bigs, alone_big):
        assert torch.equal(out, ref)
    for _, out_alone, out_mix in smalls:
        np.testing.assert_array_equal(out_mix.numpy(), out_alone.numpy())
    assert srv.stats()["failed"] == 0
    srv.destroy()
    # the large results against a plain plan on the device
    plan = _sm100.Plan(shape, 0)
    for (x, _, d), ref in zip(bigs, alone_big):
        a = x.cuda()
        b = torch.empty_like(a)
        plan.execute(a.data_ptr(), b.data_ptr(), d, 1.0, 0)
        torch.cuda.synchronize()
        assert torch.equal(b.cpu(), ref)
    plan.destroy()
