"""Batched form (shafft_sm100_batch_*): many transforms of different shapes
in one persistent launch, each checked against the CPU oracle."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16), (64, 32, 8), (97, 24), (131, 5, 7), (211, 16), (12, 10, 14), (256, 256), (5,),
          (1, 1), (63, 47, 31), (1000,), (4096, 3), (7, 11, 13), (2, 128, 2), (128, 1, 64), (243, 25),
          (331, 3), (17, 353), (700,), (600, 5)]


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
def test_batch_matches_oracle_and_replays(prec):
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    b = _sm100.Batch(SHAPES, prec, autotune=False)
    xs = [o.uniform_input(s, seed=i, dtype=dt) for i, s in enumerate(SHAPES)]
    src = [S.DeviceBuffer(x.size, prec) for x in xs]
    dst = [S.DeviceBuffer(x.size, prec) for x in xs]
    for x, d in zip(xs, src):
        d.upload(x)
    for rep in range(2):  # second call replays the captured graph
        b.execute([d.ptr for d in src], [d.ptr for d in dst], 0, 1.0, 0)
        for i, (x, d) in enumerate(zip(xs, dst)):
            y = d.download().reshape(x.shape)
            ref = o.fftn(x.astype(np.complex128), precise=(prec == S.Z2Z))
            assert o.rel_l2(y, ref) <= tol(x.size, prec), (rep, SHAPES[i])
    # backward with a fused scale; src is read only, so it still holds x
    b.execute([d.ptr for d in src], [d.ptr for d in dst], 1, 0.5, 0)
    b.status()
    for i, (x, d) in enumerate(zip(xs, dst)):
        y = d.download().reshape(x.shape)
        ref = 0.5 * o.fftn(x.astype(np.complex128), sign=1, precise=(prec == S.Z2Z))
        assert o.rel_l2(y, ref) <= tol(x.size, prec), SHAPES[i]


def test_batch_autotune_cache(tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("SHAFFT_SM100_TUNE_CACHE", str(cache))
    shapes = [(64, 96), (96, 64, 10)]
    b = _sm100.Batch(shapes, S.C2C, autotune=True)
    text = cache.read_text()
    assert "c64:L=96" in text and "c64:L=64" in text
    xs = [o.uniform_input(s, seed=3, dtype=np.complex64) for s in shapes]
    src = [S.DeviceBuffer(x.size) for x in xs]
    dst = [S.DeviceBuffer(x.size) for x in xs]
    for x, d in zip(xs, src):
        d.upload(x)
    b.execute([d.ptr for d in src], [d.ptr for d in dst])
    for x, d in zip(xs, dst):
        assert o.rel_l2(d.download().reshape(x.shape), o.fftn(x.astype(np.complex128))) <= tol(x.size, 0)


def test_batch_wait_timeout_sets_error_and_context_stays_usable():
    """The bounded wait of a tile for the previous pass of its transform
    running out: with the bound cut to one poll, tiles of the second pass
    that are claimed while first-pass tiles are still running give up, set
    the batch's error word and carry on, so the launch ends and
    shafft_sm100_batch_status reports SHAFFT_SM100_ECUDA with its message.
    Restoring the default bound, the next execute on the same context is
    correct again.  (No trap, no unbounded wait: the kernel always returns.)"""
    shapes = [(2048, 2048)]  # one transform, so pass-1 tiles follow pass-0 tiles at once
    x = o.uniform_input(shapes[0], seed=9, dtype=np.complex64)
    b = _sm100.Batch(shapes, S.C2C, autotune=False)
    src, dst = S.DeviceBuffer(x.size), S.DeviceBuffer(x.size)
    src.upload(x)
    b.set_wait_limit(1)
    messages = []
    for _ in range(3):  # timing-dependent: one attempt is expected to suffice
        b.execute([src.ptr], [dst.ptr], 0, 1.0, 0)
        dst.download()  # synchronises
        try:
            b.status()
        except _sm100.Sm100Error as e:
            messages.append(str(e))
            break
    assert messages and "rc=3" in messages[0] and "timed out" in messages[0], messages
    b.set_wait_limit(0)
    b.execute([src.ptr], [dst.ptr], 0, 1.0, 0)
    y = dst.download().reshape(x.shape)
    b.status()
    assert o.rel_l2(y, o.fftn(x.astype(np.complex128))) <= tol(x.size, 0)


@pytest.mark.parametrize("window_mb", ["0", "1"])
def test_batch_ticket_lookup_and_window_forms_agree(monkeypatch, window_mb):
    """The ticket -> slot table and the binary search over slot starts (the
    form batches above 2^26 tiles use, forced here with
    SHAFFT_SM100_BATCH_TICKET_TABLE=0), with pass-major tickets (window 0) and
    1 MiB windows: the same tiles with the same arithmetic, so the results
    are bit-identical, and they match the oracle."""
    xs = [o.uniform_input(s, seed=30 + i, dtype=np.complex64) for i, s in enumerate(SHAPES)]
    monkeypatch.setenv("SHAFFT_SM100_BATCH_WINDOW_MB", window_mb)
    outs = []
    for table in ("1", "0"):
        monkeypatch.setenv("SHAFFT_SM100_BATCH_TICKET_TABLE", table)
        b = _sm100.Batch(SHAPES, S.C2C, autotune=False)
        src = [S.DeviceBuffer(x.size, S.C2C) for x in xs]
        dst = [S.DeviceBuffer(x.size, S.C2C) for x in xs]
        for x, d in zip(xs, src):
            d.upload(x)
        b.execute([d.ptr for d in src], [d.ptr for d in dst], 0, 1.0, 0)
        b.status()
        outs.append([d.download() for d in dst])
        b.destroy()
    for i, (x, y0, y1) in enumerate(zip(xs, *outs)):
        assert np.array_equal(y0, y1), SHAPES[i]
        ref = o.fftn(x.astype(np.complex128))
        assert o.rel_l2(y0.reshape(x.shape), ref) <= tol(x.size, S.C2C), SHAPES[i]
