"""A discrete-event model of the persistent stepper's scheduling protocol (csrc/fv_stepper.cuh),
run on the CPU: the order of items (tile order rotated by one tile row per stage), taken by each CTA
from its own static sequence b, b + G, ... (the single-grid stepper) or from a shared queue (an
ensemble member), stage 1's check of the previous step and its wait on the neighbours' stage-2
flags, its wait for the step's publication before its update, stage 2's waits, the completion of
each item (flag release, step count, the last stage-2 item's publication) deferred to a separate
thread that runs while the CTA's next item waits and must end before that item's body, and the stop
rule.  CTAs and completions run with random durations.  The model must always terminate with the
expected step count, every read must see the expected step's data (no stale read) and no tile may be
overwritten while an older version of it is still being read.  The dependency lists are the
library's own (fv_stepper_dependencies)."""
import ctypes as C
import heapq
import importlib
import random

import numpy as np
import pytest

fv = importlib.import_module("neural-pde-surrogate_b200")


def library_deps(nx, ny, bcx, bcy, tx, ty):
    nnz = C.c_int()
    L = fv.lib()
    assert L.fv_stepper_dependencies(nx, ny, bcx, bcy, tx, ty, None, 0, None, 0, C.byref(nnz)) == 0
    T = -(-nx // tx) * -(-ny // ty)
    off, idx = np.zeros(T + 1, np.int32), np.zeros(nnz.value, np.int32)
    L.fv_stepper_dependencies(nx, ny, bcx, bcy, tx, ty, C.c_void_p(off.ctypes.data), T + 1,
                              C.c_void_p(idx.ctypes.data), nnz.value, C.byref(nnz))
    return [idx[off[t]:off[t + 1]].tolist() for t in range(T)]


def halo_reads(nx, ny, bcx, bcy, tx, ty):
    """Tiles whose data each tile's halo box reads (the boundary mapping of grid2d.hpp:43-66)."""
    def bc(g, n, b):
        return g % n if b == 1 else min(max(g, 0), n - 1)
    ntx, nty = -(-nx // tx), -(-ny // ty)
    out = []
    for b in range(nty):
        for a in range(ntx):
            xs = {bc(c, nx, bcx) // tx for c in range(a * tx - 2, a * tx + tx + 2)}
            ys = {bc(r, ny, bcy) // ty for r in range(b * ty - 2, b * ty + ty + 2)}
            out.append({y * ntx + x for y in ys for x in xs})
    return out


def simulate(nx, ny, bcx, bcy, tx, ty, ctas, n_run, budget, seed, bad_at=None, assign="static"):
    """Steps s0 .. run until the loop's target (n_run steps), the launch budget, or a bad state."""
    rng = random.Random(seed)
    dep = library_deps(nx, ny, bcx, bcy, tx, ty)
    reads = halo_reads(nx, ny, bcx, bcy, tx, ty)
    T = len(dep)
    ntx, nty = -(-nx // tx), -(-ny // ty)
    s0 = 5
    flag1, flag2 = [s0] * T, [s0] * T
    W, W1 = [s0] * T, [None] * T            # the step whose state / stage-1 output each tile holds
    rW, rW1 = [0] * T, [0] * T              # readers inside their read window
    ctl = dict(complete=s0 - 1, stop=None, queue=0, done2=0, srun={})

    def publish(j):  # publish_step: does step j+1 run?
        s1 = j + 1
        run = s1 < s0 + budget and s1 < s0 + n_run and s1 != bad_at
        ctl["srun"][s1] = run
        if not run and ctl["stop"] is None:
            ctl["stop"] = s1
        ctl["complete"] = j

    publish(s0 - 1)  # the launch prologue

    def done_or_stopped(target):
        return ctl["complete"] >= target or (ctl["stop"] is not None and ctl["stop"] <= target)

    def complete(step, stage, tile):  # item_tail
        if stage == 1:
            flag1[tile] = step + 1
        else:
            flag2[tile] = step + 1
            ctl["done2"] += 1
            if ctl["done2"] == (step - s0 + 1) * T:
                publish(step)

    def tail(item, box):  # the completion thread: runs while the next item waits, never waits itself
        yield 0.4 * rng.random()
        complete(*item)
        box["done"] = True

    spawn = []  # completions started by the CTAs, picked up by the event loop

    def cta(cid):
        i, prev = 0, None
        while True:
            if assign == "static":
                k = cid + i * ctas
                i += 1
            else:
                k = ctl["queue"]
                ctl["queue"] += 1
            box = {"done": prev is None}
            if prev is not None:
                spawn.append(tail(prev, box))
                prev = None
            blk = k // T  # stage block: step s0 + blk // 2, stage 1 + blk % 2, tile order rotated by blk rows
            step, stage, tile = s0 + blk // 2, 1 + blk % 2, (k % T + (blk % nty) * ntx) % T
            go = step < s0 + budget
            if go and stage == 1:
                if step > s0:
                    while not done_or_stopped(step - 2):
                        yield "wait"
                    go = ctl["complete"] >= step - 2 and ctl["srun"].get(step - 1) and step < s0 + n_run
                    while go and not all(flag2[d] >= step for d in dep[tile]):
                        yield "wait"
                else:
                    go = ctl["srun"][s0]
            elif go:
                while not done_or_stopped(step - 1):
                    yield "wait"
                go = ctl["complete"] >= step - 1 and ctl["srun"].get(step)
                while go and not all(flag1[d] >= step + 1 for d in dep[tile]):
                    yield "wait"
            while not box["done"]:  # the claim barrier: the previous completion has ended
                yield "wait"
            if not go:
                return
            if stage == 1:
                for d in reads[tile]:
                    assert W[d] == step, ("stale W", step, tile, d, W[d])
                    rW[d] += 1
                yield rng.random()
                for d in reads[tile]:
                    rW[d] -= 1
                yield 3 * rng.random()  # slopes and fluxes before the step is published
                while not done_or_stopped(step - 1):
                    yield "wait"
                if ctl["complete"] < step - 1 or not ctl["srun"].get(step):
                    return
                assert rW1[tile] == 0, ("W1 overwritten while read", step, tile)
                W1[tile] = step
                yield 0.5 * rng.random()
            else:
                for d in reads[tile]:
                    assert W1[d] == step, ("stale W1", step, tile, d, W1[d])
                    rW1[d] += 1
                yield rng.random()
                for d in reads[tile]:
                    rW1[d] -= 1
                yield 3 * rng.random()
                assert rW[tile] == 0, ("W overwritten while read", step, tile)
                W[tile] = step + 1
                yield 0.5 * rng.random()
            prev = (step, stage, tile)

    gens = [cta(c) for c in range(ctas)]
    events = [(0.1 * rng.random(), c) for c in range(ctas)]
    heapq.heapify(events)
    while events:
        now, c = heapq.heappop(events)
        assert now < 1e6, "no progress"
        try:
            d = next(gens[c])
        except StopIteration:
            d = None
        while spawn:
            gens.append(spawn.pop())
            heapq.heappush(events, (now, len(gens) - 1))
        if d is not None:
            heapq.heappush(events, (now + (0.05 if d == "wait" else d), c))
    return ctl["complete"] - (s0 - 1)


GRIDS = [(128, 128, 1, 1, 16, 14), (65, 33, 1, 1, 16, 16), (70, 45, 1, 0, 16, 14), (17, 3, 0, 1, 16, 7),
         (1, 5, 1, 0, 16, 7), (33, 17, 0, 0, 32, 8)]


@pytest.mark.parametrize("assign", ["static", "queue"])
@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("ctas", [1, 7, 64])
def test_protocol_terminates_with_the_right_steps_and_no_stale_reads(grid, ctas, assign):
    for n_run, budget, bad in [(6, 40, None), (9, 4, None), (6, 40, 8), (1, 40, None), (0, 40, None)]:
        steps = simulate(*grid, ctas, n_run, budget, seed=ctas * 7 + n_run, bad_at=bad, assign=assign)
        expect = min(n_run, budget) if bad is None else min(n_run, budget, bad - 5)
        assert steps == expect, (grid, ctas, n_run, budget, bad, steps)


def test_protocol_at_the_bench_size_with_every_resident_cta():
    """512^2 in 16 x 14 tiles (1184 tiles, partial last tile row) with 592 CTAs, as on a B200."""
    for n_run, budget in [(3, 40), (2, 2)]:
        assert simulate(512, 512, 1, 1, 16, 14, 592, n_run, budget, seed=n_run) == min(n_run, budget)
