"""The row ring of the weight-gradient conv kernel (conv3x3_wgrad_mn_kernel in csrc/fvnet_conv.cu),
modelled on the CPU.  Input row u of an image lives in slot s = (u + 1) mod 8, stored twice (planes s
and s + 8).  An iteration takes one or two output rows of one image; output row y's MMA reads the
four planes p0 .. p0 + 3, p0 = y mod 8, of which the first three must hold rows y - 1, y, y + 1 (the
fourth feeds unused accumulator rows).  While an iteration's MMAs run, the next iteration's new rows
are copied in.  The model replays the kernel's schedule over every CTA range of a few batch shapes
and checks:
  * every plane an MMA uses holds the row it needs (periodic in y);
  * a copy issued during an iteration's MMAs never writes a plane those MMAs use (only their unused
    fourth planes);
  * at most 16 planes are ever addressed.
The formulas are the kernel's: rows_in, the staged row ranges and the plane addressing."""
import pytest


def rows_in(row, r1, H):
    return 2 if (row + 1 < r1 and (row + 1) % H != 0) else 1


def replay(B, H, rows_per_cta, slots=8):
    """The kernel's schedule with a ring of `slots` slots (8 in the kernel), each row stored twice."""
    total = B * H
    for r0 in range(0, total, rows_per_cta):
        r1 = min(total, r0 + rows_per_cta)
        planes = [None] * (2 * slots)  # (image, row mod H) held by each plane

        def stage(n, u):
            s = (u + 1) % slots
            for p in (s, s + slots):
                planes[p] = (n, u % H)
            return {s, s + slots}

        n, y, k = r0 // H, r0 % H, rows_in(r0, r1, H)
        for u in range(y - 1, y + k + 1):
            stage(n, u)
        row = r0
        while row < r1:
            n, y, k = row // H, row % H, rows_in(row, r1, H)
            used = set()
            for j in range(k):
                p0 = (y + j) % slots
                assert p0 + 3 < 2 * slots
                for ky in range(3):
                    assert planes[p0 + ky] == (n, (y + j + ky - 1) % H), (r0, row, j, ky)
                    used.add(p0 + ky)
            nrow = row + k
            has_next = nrow < r1
            next_cont = has_next and nrow % H != 0
            k2 = rows_in(nrow, r1, H) if has_next else 0
            if next_cont:  # copies issued while this iteration's MMAs run
                for u in range(y + k + 1, y + k + k2 + 1):
                    written = stage(n, u)
                    assert not (written & used), (r0, row, u, written & used)
            elif has_next:  # a new image, staged after the MMAs completed
                n2 = nrow // H
                for u in range(-1, k2 + 1):
                    stage(n2, u)
            row = nrow


@pytest.mark.parametrize("B,H,rows_per_cta", [
    (64, 64, 14),   # the bench's batch: 4096 rows over 296 CTAs
    (3, 296, 3),    # three rows per CTA, image boundaries inside ranges
    (2, 8, 1), (1, 4, 1), (5, 8, 1), (1, 16, 1),  # the GPU test's small shapes
    (7, 9, 5), (3, 10, 7), (2, 3, 4),             # odd heights and ranges
])
def test_the_ring_holds_every_row_an_mma_reads(B, H, rows_per_cta):
    replay(B, H, rows_per_cta)


def test_the_model_catches_a_four_slot_ring():
    """Four slots (enough for one output row per iteration) are too few for two: the next rows'
    copies would overwrite rows the MMAs in flight read, and the model must say so."""
    with pytest.raises(AssertionError):
        replay(64, 64, 14, slots=4)
