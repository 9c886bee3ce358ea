"""Multi-GPU docking by ligand shards: one process per GPU, no data-path collective.

The reference's multi-GPU driver (Multi_GPU_docking.py:395-423) starts one
docking process per GPU over disjoint slices of a ligand directory.  Here
every rank of a torch.distributed group (NCCL between GPUs, gloo on CPU):

* takes its shard of the ligand list -- ligands assigned largest-cost-first
  to the least-loaded rank (greedy LPT bins), with the same cost estimate
  vd_dock_batched uses to order its work queue (MC steps x BFGS steps x bytes
  touched per evaluation), so ranks finish together;
* docks its shard with its own context (its own grid maps: rebuilding them
  costs about a millisecond, less than moving 213 MB between GPUs);
* returns per-ligand results, which come back to every rank in the caller's
  order through one host-side object gather (a few KB per ligand).

Timing of a multi-rank step is the maximum over ranks (max_over_ranks).
"""
import heapq

MAX_TORS = 48


def ligand_cost(n_atoms, n_heavy, ntors, n_pairs, search_depth=0, max_bfgs_steps=0, dense_bfgs=False):
    """Relative cost of docking one ligand: MC steps x BFGS steps x bytes per
    evaluation, with the heuristics of main.cpp:367-389 when the depth / steps
    are 0 (x2 and (30 + atoms)/3 for RILC-BFGS, x2.4 and (25 + atoms)/3 for
    dense BFGS) and, as the docking kernel does, no MC steps for a negative
    depth (each chain returns its initial pose: one evaluation's bytes)."""
    per_eval = 32.0 * n_heavy + 16.0 * n_pairs
    if search_depth < 0:
        return per_eval
    depth = search_depth
    if depth == 0:
        depth = max(1, int((0.24 * n_atoms + 0.29 * ntors - 3.41) * (2.4 if dense_bfgs else 2.0)))
    steps = max_bfgs_steps if max_bfgs_steps > 0 else ((25 if dense_bfgs else 30) + n_atoms) // 3
    return float(depth) * steps * per_eval


def desc_cost(lig, search_depth=0, max_bfgs_steps=0, dense_bfgs=False):
    """ligand_cost of a ligand description dict (vdock.synth / PDBQT form)."""
    n_heavy = int(sum(1 for t in lig["xs"] if t >= 0))
    ntors = len(lig["node_parent"]) - 1
    return ligand_cost(int(lig["n_atoms"]), n_heavy, ntors, len(lig["pairs"]), search_depth, max_bfgs_steps,
                       dense_bfgs)


def shard_by_cost(costs, world):
    """Greedy LPT partition of ligand indices into `world` shards.

    Ligands are taken in decreasing cost (ties by index) and each goes to the
    shard with the smallest total so far (ties by rank), so the largest shard
    is at most 4/3 of the optimum plus one ligand.  Each shard lists its
    indices in increasing order.  Deterministic: every rank computes the same
    partition without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def dock_sharded(dock_fn, ligands, costs, group=None):
    """Docks `ligands` across the ranks of a torch.distributed group.

    dock_fn(list_of_ligands) -> list of per-ligand results (same order); it
    runs on this rank's shard only.  Returns the results of all ligands in
    the given order, on every rank.  Every rank must call this with the same
    ligands and costs.  A rank that fails raises here; the others then fail
    in the gather (process-group timeout or a closed connection) instead of
    waiting forever."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if len(costs) != len(ligands):
        raise ValueError("one cost per ligand")
    shards = shard_by_cost(costs, world)
    mine = shards[rank]
    local = dock_fn([ligands[i] for i in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError(f"rank {rank}: dock_fn returned {len(local)} results for {len(mine)} ligands")
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(local)), group=group)
    out = [None] * len(ligands)
    for idx, res in gathered:
        for i, r in zip(idx, res):
            out[i] = r
    return out


def max_over_ranks(seconds, group=None, device=None):
    """Maximum of a per-rank duration over the group (the time of a
    multi-rank step).  device: "cuda" for NCCL groups, None for CPU (gloo)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
