"""The persistent stepper's tile dependency lists (host code of libfv, no GPU), checked against an
independent restatement: every cell of a tile's halo box, mapped through the boundary conditions
like apply_bcs (grid2d.hpp:43-66), must lie in a listed tile, and the relation must hold in reverse
(a tile waits for the tiles that read what it overwrites)."""
import ctypes as C
import importlib

import numpy as np
import pytest

fv = importlib.import_module("neural-pde-surrogate_b200")


def deps(nx, ny, bcx, bcy, tx, ty):
    nnz = C.c_int()
    L = fv.lib()
    assert L.fv_stepper_dependencies(nx, ny, bcx, bcy, tx, ty, None, 0, None, 0, C.byref(nnz)) == 0
    T = -(-nx // tx) * -(-ny // ty)
    off = np.zeros(T + 1, np.int32)
    idx = np.zeros(nnz.value, np.int32)
    assert L.fv_stepper_dependencies(nx, ny, bcx, bcy, tx, ty, C.c_void_p(off.ctypes.data), T + 1,
                                     C.c_void_p(idx.ctypes.data), nnz.value, C.byref(nnz)) == 0
    return [set(idx[off[t]:off[t + 1]].tolist()) for t in range(T)], [idx[off[t]:off[t + 1]] for t in range(T)]


def bc_index(g, n, bc):
    return g % n if bc == 1 else min(max(g, 0), n - 1)


@pytest.mark.parametrize("nx,ny,bcx,bcy,tx,ty", [(512, 512, 1, 1, 16, 14), (65, 33, 1, 1, 16, 16), (70, 45, 1, 0, 16, 14),
                                                 (17, 3, 0, 1, 16, 7), (1, 5, 1, 0, 32, 8), (33, 17, 0, 0, 32, 8),
                                                 (49, 97, 1, 1, 16, 14), (64, 64, 1, 1, 16, 16)])
def test_dependency_lists_cover_every_halo_cell_both_ways(nx, ny, bcx, bcy, tx, ty):
    got, raw = deps(nx, ny, bcx, bcy, tx, ty)
    ntx, nty = -(-nx // tx), -(-ny // ty)
    reads = []
    for b in range(nty):
        for a in range(ntx):
            xs = {bc_index(c, nx, bcx) // tx for c in range(a * tx - 2, a * tx + tx + 2)}
            ys = {bc_index(r, ny, bcy) // ty for r in range(b * ty - 2, b * ty + ty + 2)}
            reads.append({y * ntx + x for y in ys for x in xs})
    for t in range(ntx * nty):
        expect = set(reads[t]) | {u for u in range(ntx * nty) if t in reads[u]} | {t}
        assert got[t] == expect, (t, sorted(got[t]), sorted(expect))
        assert (np.diff(raw[t]) > 0).all()  # sorted, no repeats
    if nx >= 3 * tx and ny >= 3 * ty and nx % tx == 0 and ny % ty == 0 and bcx == bcy == 1:
        assert all(len(d) == 9 for d in got)  # full tiles, periodic: the 3 x 3 neighbourhood


def test_dependency_lists_reject_bad_arguments():
    nnz = C.c_int()
    assert fv.lib().fv_stepper_dependencies(0, 4, 1, 1, 16, 14, None, 0, None, 0, C.byref(nnz)) == 1
    assert fv.lib().fv_stepper_dependencies(4, 4, 2, 1, 16, 14, None, 0, None, 0, C.byref(nnz)) == 1
