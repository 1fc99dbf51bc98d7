"""Multi-GPU plumbing, world_size 2 on the gloo backend (CPU).  A single
system does not shard: bench.py runs one replica per rank and reports the
max over ranks.  The batched independent systems (--config c4) shard by cost
over the ranks, with no exchange while solving and one gather of the
per-system results at the end."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench
    r, w, local = bench.dist_init(world)
    assert (r, w) == (rank, world)
    import torch.distributed as dist
    assert dist.get_backend() == "gloo"
    # each replica times its own solve; the job reports the slowest
    m = bench.max_over_ranks(1.5 if rank == 0 else 2.5, w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((rank, m))


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5), (1, 2.5)]


def test_reference_arm_nonzero_rank_prints_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_shard_systems_balances_by_cost():
    sys.path.insert(0, ROOT)
    import bench
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = bench.shard_systems(costs, 3)
    assert sorted(q for p in parts for q in p) == list(range(len(costs)))
    loads = [sum(costs[q] for q in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert bench.shard_systems(costs, 1) == [list(range(len(costs)))]


def _shard_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench
    r, w, local = bench.dist_init(world)
    costs = [int(c) for c in range(10, 74)]  # 64 systems
    mine = bench.shard_systems(costs, w)[r]
    # each rank "solves" its shard (no exchange), then rank 0 gathers
    merged = bench.gather_per_system({s: (s % 7, 1e-7 * s) for s in mine}, w, len(costs))
    import torch.distributed as dist
    dist.destroy_process_group()
    q.put((rank, len(mine), sorted(merged) == list(range(64)), merged[63]))


def test_c4_shards_gather_gloo_world2():
    """The batched-systems configuration shards its systems over the ranks
    (no collective while solving) and gathers each system's result once."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got[0][1] + got[1][1] == 64 and got[0][2] and got[1][2]
    assert got[0][3] == (0, 63e-7)
