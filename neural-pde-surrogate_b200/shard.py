"""Independent trajectories spread over GPUs: one process per GPU, no data-path collective.

The reference generates its dataset and runs its baselines as independent processes, one trajectory
each (data/generate.py:60-105 in a process pool, experiments/solver_baseline.py:116-117).  Nothing is
exchanged between trajectories, so the multi-GPU form is a partition: every rank takes a share of
the trajectories and runs them on its own GPU.  Shares are balanced by cost with the greedy
longest-processing-time rule (each item, most expensive first, goes to the least-loaded rank), a cost
being the trajectory's cell-updates: n^2 cells x steps, and steps grow like n t_end at a fixed CFL.

The one optional collective is the final gather of per-trajectory results (summaries, not states)
to rank 0 with torch.distributed.gather_object, after all work is done.
"""
import heapq


def trajectory_cost(n, t_end, t_start=0.0):
    """Relative cost of an n x n trajectory run to t_end: cells x steps ~ n^2 * (n * t_end)."""
    return float(n) ** 3 * max(float(t_end), 1e-12)


def balanced_split(costs, world):
    """Partition item indices 0..len(costs)-1 into `world` lists by greedy LPT.  Deterministic: ties
    are broken by item index, then by rank.  Each rank's list is in ascending item order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def dist_info():
    """(rank, world) of the default process group, or (0, 1) when none is initialised."""
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except ImportError:
        pass
    return 0, 1


def run_sharded(items, fn, costs=None, gather=True):
    """Runs fn(item) for this rank's share of `items`.  With gather, rank 0 returns the results of
    every item in the order of `items` (other ranks return None); without, every rank returns
    {index: result} of its own share.  A rank whose fn raises never reaches the gather; its peers'
    gather then ends with the process group's timeout error instead of waiting for good."""
    rank, world = dist_info()
    costs = [1.0] * len(items) if costs is None else list(costs)
    mine = balanced_split(costs, world)[rank]
    results = {i: fn(items[i]) for i in mine}
    if not gather:
        return results
    if world == 1:
        return [results[i] for i in range(len(items))]
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(results, parts, dst=0)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in range(len(items))]
