"""Host-side facts the level-1 Galerkin kernels (hmfem_b200/csrc/rap19.cu)
rely on, checked without a GPU.

Level 1 of an assembled grid is the 19-offset graph on the even cells
(offsets 0, +-2e_a, +-e_a+-e_b); its C cells form an independent set of
that graph.  The (A P) row of a cell holds C cells within fine L1 distance
4 (85 candidate offsets), a level-2 row C cells within distance 6 (231):
the padded row sizes kCap0 / kCap1 must hold the largest independent set
of those balls.  The slots are ordered by (dz, dy, dx), which must be the
order of the fine index for every pair of in-grid cells, so that slot
order is column order.
"""
import itertools
import os
import re

import numpy as np
import pytest

SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "hmfem_b200", "csrc",
                   "rap19.cu")

STENCIL = {o for a in range(3) for sg in (-2, 2)
           for o in [tuple(sg if i == a else 0 for i in range(3))]}
STENCIL |= {tuple(sa if i == a else sb if i == b else 0 for i in range(3))
            for a, b in ((0, 1), (0, 2), (1, 2)) for sa in (-1, 1) for sb in (-1, 1)}


def ball(R):
    """Offsets with |dx|+|dy|+|dz| <= R and an even sum, (dz, dy, dx) order."""
    return [(x, y, z) for z in range(-R, R + 1) for y in range(-R, R + 1)
            for x in range(-R, R + 1) if abs(x) + abs(y) + abs(z) <= R and (x + y + z) % 2 == 0]


def max_independent(points):
    from scipy.optimize import Bounds, LinearConstraint, milp
    idx = {p: i for i, p in enumerate(points)}
    rows = []
    for p in points:
        for o in STENCIL:
            q = (p[0] + o[0], p[1] + o[1], p[2] + o[2])
            if q in idx and idx[q] > idx[p]:
                r = np.zeros(len(points))
                r[idx[p]] = r[idx[q]] = 1
                rows.append(r)
    res = milp(c=-np.ones(len(points)), constraints=LinearConstraint(np.array(rows), -np.inf, 1),
               integrality=np.ones(len(points)), bounds=Bounds(0, 1))
    assert res.success
    return int(round(-res.fun))


def constant(name):
    m = re.search(rf"\b{name} = (\d+)[;,]", open(SRC).read())
    return int(m.group(1))


def test_stencil_has_18_neighbour_offsets():  # the 19-offset set without 0
    assert len(STENCIL) == 18


@pytest.mark.parametrize("R,count,cap", [(4, "kB4", "kCap0"), (6, "kB6", "kCap1")])
def test_padded_rows_hold_every_independent_set(R, count, cap):
    pts = ball(R)
    assert len(pts) == constant(count)
    assert max_independent(pts) <= constant(cap)


@pytest.mark.parametrize("nx,ny,nz", [(4, 4, 4), (6, 4, 9), (8, 6, 5), (16, 4, 3)])
def test_slot_order_is_fine_index_order(nx, ny, nz):
    """For every even cell and every two in-grid ball-6 offsets, (dz, dy,
    dx) order equals fine-index order (and the level row s >> 1 follows)."""
    pts = ball(6)
    nxy = nx * ny
    for x, y, z in itertools.product(range(nx), range(ny), range(nz)):
        if (x + y + z) % 2:
            continue
        s = x + nx * y + nxy * z
        ins = [p for p in pts if 0 <= x + p[0] < nx and 0 <= y + p[1] < ny and 0 <= z + p[2] < nz]
        fine = [s + p[0] + nx * p[1] + nxy * p[2] for p in ins]
        assert fine == sorted(fine)
        rows = [f >> 1 for f in fine]
        assert rows == sorted(rows) and len(set(rows)) == len(rows)
