"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (world size 2,
127.0.0.1), the max-over-ranks timing, the sum of per-rank counts and the
split of a T-P table's states across ranks (disjoint, each state once)."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import bench, torch.distributed as dist
sys.path.insert(0, sys.argv[1] + "/helios-k_b200")
ws, rank, lrank = bench.dist_setup()
assert dist.get_backend() == "gloo"
m = bench.barrier_max(ws, 1.5 + rank)          # rank 1 is the slower one
assert m == 2.5, m
assert bench.barrier_sum(ws, 10.0 + rank) == 21.0
from hkb import synth
T, P = synth.table_states()
mine = bench.rank_states(len(T), ws, rank)
parts = [None] * ws
dist.all_gather_object(parts, [int(v) for v in mine])
allst = sorted(v for p in parts for v in p)
assert allst == list(range(len(T))), "every state exactly once"
assert abs(len(parts[0]) - len(parts[1])) <= 1
print("rank", rank, "max", m, "states", len(mine), flush=True)
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_take_the_max_time():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), HKB_DIST_BACKEND="gloo",
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("gloo ranks did not finish")
        outs.append(out)
        assert p.returncode == 0, out
    assert "rank 0 max 2.5 states 300" in outs[0] and "rank 1 max 2.5 states 300" in outs[1]
