"""Row-block sharding of the FP64 system (one shard per GPU).

Shard r of R owns the target fibers [r M / R, (r + 1) M / R) and assembles
their rows with no communication; products, the right-hand side and the
velocities are completed by NCCL all-gathers.

* CPU: the partition (every fiber in exactly one shard, in order, sizes
  within one of each other), and two gloo ranks agreeing on it;
* GPU, one device: R shards without a communicator assemble exactly the rows
  of the whole system (bit for bit) and its right-hand side rows; a sharded
  handle of one rank (NCCL communicator of one) steps exactly like the
  unsharded handle (every product, right-hand side and velocity through the
  all-gather and the compaction).  More shards need more GPUs.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import rigidfibers_kth_b200 as rf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("M,R", [(1, 1), (7, 3), (100, 8), (4000, 7), (8000, 64)])
def test_shard_ranges_tile_the_fibers(M, R):
    ranges = [rf.shard_range(M, R, r) for r in range(R)]
    assert ranges[0][0] == 0 and ranges[-1][1] == M
    for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in ranges]
    assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_shard_range_refuses_bad_arguments():
    for args in [(10, 0, 0), (10, 11, 0), (10, 3, 3), (0, 1, 0)]:
        with pytest.raises(rf.RfError):
            rf.shard_range(*args)


RANK_CODE = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
import rigidfibers_kth_b200 as rf
dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
mine = torch.tensor(rf.shard_range({M}, world, rank), dtype=torch.int64)
allr = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
dist.all_gather(allr, mine)
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "ranges": [r.tolist() for r in allr]}}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_the_partition():
    M = 4001
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE.format(root=ROOT, M=M)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("a rank did not finish")
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for d in outs:
        assert d["ranges"] == [[0, 2000], [2000, 4001]]


def _params(**kw):
    return rf.FiberParams(slenderness=1e-3, gmres_tol=1e-10, gmres_max_iters=300, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("R", [2, 3])
def test_shards_assemble_the_rows_of_the_whole_system(R):
    M = 301
    pos, ori = rf.generate_layout(M, "gaussian", 1.3, 0.2, seed=2101)
    with rf.Simulation(rf.Configuration(_params(), pos, ori)) as whole:
        whole.assemble_system()
        A = whole.matrix()
        b = whole.rhs()
    n3 = 15
    for r in range(R):
        t0, t1 = rf.shard_range(M, R, r)
        with rf.Simulation(rf.Configuration(_params(shard_index=r, shard_count=R), pos, ori)) as s:
            s.assemble_system()
            rows = s.matrix_rows(t0 * n3, (t1 - t0) * n3)
            bs = s.rhs()
            with pytest.raises(rf.RfError):
                s.solve_system()  # a shard solves only with its communicator
        assert np.array_equal(rows, A[t0 * n3:t1 * n3])
        assert np.array_equal(bs[t0 * n3:t1 * n3], b[t0 * n3:t1 * n3])
        assert not bs[:t0 * n3].any() and not bs[t1 * n3:].any()


@pytest.mark.gpu
def test_one_rank_communicator_steps_like_the_whole_system():
    M = 257
    pos, ori = rf.generate_layout(M, "gaussian", 1.2, 0.2, seed=2102)
    out = []
    for sharded in (False, True):
        kw = dict(nccl_id=rf.shard_unique_id()) if sharded else {}
        with rf.Simulation(rf.Configuration(_params(shard_index=0, shard_count=1), pos, ori), **kw) as s:
            for t in range(2):
                s.step(t)
            out.append(s.state() + s.velocities() + (s.coeffs(), s.rhs()))
            stats = s.solve_stats()
        assert stats["converged"]
    for a, b in zip(*out):
        assert np.array_equal(a, b)
