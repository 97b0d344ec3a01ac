"""The library's all-to-all step (shafft_b200.slab.CudaOps.alltoall) on 2
and 3 gloo ranks, CPU tensors: the branch taken for an NCCL group (the
tensors go to all_to_all_single directly) and the host-staged branch of a
gloo group must move the same blocks with the same counts.  The NCCL branch
is forced by reporting the group's backend as "nccl"; its only difference
from a real NCCL group is the transport, so this pins its counts, views and
element order without a second GPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import json, sys
sys.path.insert(0, sys.argv[1])
import torch, torch.distributed as dist
from shafft_b200 import slab

dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
ops = slab.CudaOps(1)          # complex128; loads libshafft_sm100.so, no GPU call
# uneven blocks: rank r sends (r + q + 1) elements to rank q
send = [rank + q + 1 for q in range(world)]
recv = [q + rank + 1 for q in range(world)]
inp = torch.zeros(sum(send) + 3, dtype=torch.complex128)
pos = 0
for q in range(world):
    for e in range(send[q]):
        inp[pos] = complex(1000 * rank + 10 * q + e, -rank - 0.5 * e)
        pos += 1
results = {}
real_backend = dist.get_backend
for name in ("gloo", "nccl"):
    out = torch.full((sum(recv) + 3,), complex(-7, -7), dtype=torch.complex128)
    dist.get_backend = (lambda g=None, _n=name: _n)
    try:
        ops.alltoall(out, inp, recv, send, None, world)
    finally:
        dist.get_backend = real_backend
    results[name] = [[z.real, z.imag] for z in out.tolist()]
expect = []
for q in range(world):
    for e in range(recv[q]):
        expect.append([1000 * q + 10 * rank + e, -q - 0.5 * e])
expect += [[-7.0, -7.0]] * 3
dist.destroy_process_group()
json.dump({"results": results, "expect": expect}, open(sys.argv[2], "w"))
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_alltoall_nccl_branch_matches_host_staged_branch(tmp_path, world):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(r), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(tmp_path / f"r{r}.json")],
                                      env=env))
    for p in procs:
        assert p.wait(timeout=240) == 0
    for r in range(world):
        out = json.loads((tmp_path / f"r{r}.json").read_text())
        assert out["results"]["gloo"] == out["expect"], r
        assert out["results"]["nccl"] == out["expect"], r
