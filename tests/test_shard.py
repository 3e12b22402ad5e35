"""Multi-process path on CPU: independent trajectories split over ranks (gloo, world size 2).

The per-item work here is the CPU oracle on small grids (test infrastructure); on GPU boxes the same
run_sharded call drives the GPU solver, one rank per GPU.
"""
import datetime
import importlib
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
shard = importlib.import_module("neural-pde-surrogate_b200.shard")


def test_balanced_split_covers_every_item_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = rng.choice([64, 128, 256, 512], size=256)
    costs = [shard.trajectory_cost(n, 0.25) for n in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = shard.balanced_split(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT is within 4/3 of the optimum, and the optimum is at least max(mean load, largest item)
        bound = max(sum(costs) / world, max(costs))
        assert max(loads) <= 4.0 / 3.0 * bound + 1e-9
        assert parts == shard.balanced_split(costs, world)  # deterministic


def test_balanced_split_edge_cases():
    assert shard.balanced_split([], 3) == [[], [], []]
    assert shard.balanced_split([5.0], 2) == [[0], []]
    assert shard.balanced_split([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.balanced_split([1.0], 0)


def test_single_process_run_keeps_item_order():
    out = shard.run_sharded(list(range(7)), lambda x: x * x, costs=[7 - i for i in range(7)])
    assert out == [x * x for x in range(7)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


ITEMS = [("riemann", 0, 16), ("blast", 1, 32), ("riemann", 2, 24), ("blast", 3, 16), ("riemann", 4, 32)]


def _solve(item):
    """Final density checksum of one small trajectory on the CPU oracle (t = 0.01)."""
    from oracle.oracle import OracleSolver
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    fam, idx, n = item
    rho, u, v, p, _, _ = ic.sample(fam, idx, n)
    o = OracleSolver(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic", "hllc", "vanleer", 0.5)
    o.set_state(ic.to_conserved(rho, u, v, p))
    o.advance_to(0.01)
    return o.steps, o.get_state().tobytes().hex()[:64], float(o.get_state()[..., 0].sum())


def _worker(rank, world, port, out_dir, fail_rank):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    sh = importlib.import_module("neural-pde-surrogate_b200.shard")
    costs = [sh.trajectory_cost(n, 0.01) for _, _, n in ITEMS]

    def fn(item):
        if rank == fail_rank:
            raise RuntimeError("planted failure on the host")
        return _solve(item)

    try:
        res = sh.run_sharded(ITEMS, fn, costs=costs)
        (Path(out_dir) / f"rank{rank}.txt").write_text(repr(res))
    except Exception as e:  # noqa: BLE001 - the test reads what each rank saw
        (Path(out_dir) / f"rank{rank}.txt").write_text("ERROR " + type(e).__name__ + ": " + str(e)[:200])
    finally:
        dist.destroy_process_group()


def _spawn(tmp_path, fail_rank=-1):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), fail_rank), nprocs=2, join=True,
                       start_method="spawn")
    return [(tmp_path / f"rank{r}.txt").read_text() for r in range(2)]


def test_two_gloo_ranks_match_a_serial_run(tmp_path):
    r0, r1 = _spawn(tmp_path)
    assert r1 == "None"  # only rank 0 holds the gathered results
    serial = [_solve(it) for it in ITEMS]
    assert r0 == repr(serial)


def test_a_failing_rank_ends_its_peer_with_an_error(tmp_path):
    """Host-side failure: rank 1 raises before the gather; rank 0's gather must end with an error
    within the process group's timeout instead of waiting for good."""
    r0, r1 = _spawn(tmp_path, fail_rank=1)
    assert r1.startswith("ERROR RuntimeError: planted failure")
    assert r0.startswith("ERROR")
