"""Multi-rank docking host logic (vdock.multi) on CPU with gloo, world size 2.

The data path of a rank (one GPU) is replaced by a CPU stand-in for the
docking call; what is tested is the multi-rank plumbing the GPU runs use:
the cost-balanced ligand shards, the result gather back into the caller's
order, the max-over-ranks step time, and that a failing rank makes the other
rank fail promptly instead of hanging.
"""
import datetime
import os
import socket
import sys

import pytest

from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "vina-cuda_b200"))

from vdock import multi  # noqa: E402


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shards_partition_and_balance():
    costs = [float(c) for c in (50, 3, 41, 7, 7, 19, 33, 2, 2, 28, 11, 60, 5)]
    for world in (1, 2, 3, 4, 8, 20):
        shards = multi.shard_by_cost(costs, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        # LPT bound: the largest shard exceeds the mean by at most one ligand
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert multi.shard_by_cost(costs, 2) == multi.shard_by_cost(list(costs), 2)  # deterministic


def test_cost_matches_search_heuristics():
    # 24 atoms / 5 torsions: depth int((0.24*24 + 0.29*5 - 3.41) * 2) = 7, steps (30+24)//3 = 18
    c = multi.ligand_cost(24, 24, 5, 200)
    assert c == 7 * 18 * (32.0 * 24 + 16.0 * 200)
    assert multi.ligand_cost(24, 24, 5, 200, search_depth=1000, max_bfgs_steps=5) == 1000 * 5 * (32.0 * 24 + 16.0 * 200)
    # dense BFGS (--rilc_bfgs 0): depth int((...) * 2.4) = 9, steps (25+24)//3 = 16 (main.cpp:367-389)
    assert multi.ligand_cost(24, 24, 5, 200, dense_bfgs=True) == 9 * 16 * (32.0 * 24 + 16.0 * 200)
    # a negative depth runs no MC step (chains return their initial poses)
    assert multi.ligand_cost(24, 24, 5, 200, search_depth=-1) == 32.0 * 24 + 16.0 * 200


def _worker(rank, world, port, mode, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
        ligands = [f"lig{i}" for i in range(11)]
        costs = [float((7 * i) % 5 + 1) for i in range(11)]

        def dock(sub):
            if mode == "fail" and rank == 1:
                raise RuntimeError("docking failed on rank 1")
            return [{"ligand": l, "rank": rank, "energy": -float(len(l))} for l in sub]

        res = multi.dock_sharded(dock, ligands, costs)
        t = multi.max_over_ranks(0.5 + rank)
        q.put((rank, "ok", [r["ligand"] for r in res], sorted({r["rank"] for r in res}), t))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, "error", type(e).__name__ + ": " + str(e)[:200], None, None))


def _run(mode):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=120)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_dock_sharded_two_ranks_gloo():
    out = _run("ok")
    for rank in (0, 1):
        _, status, names, ranks, t = out[rank]
        assert status == "ok", out[rank]
        assert names == [f"lig{i}" for i in range(11)]  # every ligand once, caller's order
        assert ranks == [0, 1]  # both ranks docked a shard
        assert t == 1.5  # max over ranks


def test_failing_rank_fails_the_other_promptly():
    out = _run("fail")
    assert out[1][1] == "error" and "docking failed on rank 1" in out[1][2]
    assert out[0][1] == "error"  # the gather ends with an error, not a hang
