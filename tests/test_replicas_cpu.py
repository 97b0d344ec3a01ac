"""Multi-GPU host logic on CPU: the bench runs one process per GPU as
independent replicas (the transform does not shard; batched transform lists
and served request streams are partitioned).  These tests run the same
helpers in two `gloo` processes: the timing reductions (max / sum over
ranks) and the partition of the batched and served workloads."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local, dist = bench.dist_init("gloo")
out = {
    "rank": rank, "world": world,
    "max": bench.max_over_ranks(1.5 + rank, dist, "cpu"),
    "sum": bench.sum_over_ranks(10.0 * (rank + 1), dist, "cpu"),
    "shapes": [list(s) for s in bench.shard(bench.batched_shapes(64), rank, world)],
    "reqs": [[list(d), p, r] for d, p, r in bench.shard(bench.serve_requests(30), rank, world)],
}
dist.barrier()
dist.destroy_process_group()
with open(sys.argv[2], "w") as f:
    json.dump(out, f)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_reductions_and_partition(tmp_path):
    world = 2
    port = _free_port()
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(tmp_path / f"r{r}.json")],
                                      env=env))
    for p in procs:
        assert p.wait(timeout=240) == 0
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r, o in enumerate(res):
        assert o["rank"] == r and o["world"] == world
        assert o["max"] == pytest.approx(2.5)     # slowest rank's time
        assert o["sum"] == pytest.approx(30.0)    # whole-job totals add
    # the ranks' blocks partition the workloads, in order, sizes within one
    full_shapes = [list(s) for s in bench.batched_shapes(64)]
    assert res[0]["shapes"] + res[1]["shapes"] == full_shapes
    assert abs(len(res[0]["shapes"]) - len(res[1]["shapes"])) <= 1
    full_reqs = [[list(d), p, r] for d, p, r in bench.serve_requests(30)]
    assert res[0]["reqs"] + res[1]["reqs"] == full_reqs


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 3), (4096, 8), (5, 8)])
def test_shard_partitions_any_length(n, world):
    seq = list(range(n))
    blocks = [bench.shard(seq, r, world) for r in range(world)]
    assert sum(blocks, []) == seq
    sizes = [len(b) for b in blocks]
    assert max(sizes) - min(sizes) <= 1


def test_single_rank_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    rank, world, local, dist = bench.dist_init("gloo")
    assert (rank, world, local, dist) == (0, 1, 0, None)
    assert bench.max_over_ranks(3.0, None) == 3.0
    assert bench.sum_over_ranks(3.0, None) == 3.0
