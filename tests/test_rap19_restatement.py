"""A host restatement of the level-1 Galerkin product from the 19-offset
structure (hmfem_b200/csrc/rap19.cu: k_g19_ap, k_g19_ptap) against the
oracle's generic product (amg.h:408-582 order), bit for bit.

It follows the kernels' formulation, not the generic one: (A P)(i, k) as a
fixed-order fold over the (offset, offset) pairs with -0.0 for the terms
that do not apply, then each coarse row summed over R(e) ascending by ball
slot.  Agreement with the oracle's level 2 shows that formulation (the
-0.0 start, the slot order, the C/F cases) reproduces the reference's sums.
"""
import numpy as np
import pytest

from hmfem_b200.problem import config_problem, make_problem

Q19 = sorted([(0, 0, 0)] + [tuple(s if i == a else 0 for i in range(3))
                            for a in range(3) for s in (-2, 2)]
             + [tuple(sa if i == a else sb if i == b else 0 for i in range(3))
                for a, b in ((0, 1), (0, 2), (1, 2)) for sa in (-1, 1) for sb in (-1, 1)],
             key=lambda o: (o[2], o[1], o[0]))
CENTRE = Q19.index((0, 0, 0))


def ball(R):
    return [(x, y, z) for z in range(-R, R + 1) for y in range(-R, R + 1)
            for x in range(-R, R + 1) if abs(x) + abs(y) + abs(z) <= R and (x + y + z) % 2 == 0]


CASES = {
    "hetero_8x8x6": lambda: make_problem(8, 8, 6, log10k=(-14.0, 1.0, 1.5), n_conduits=1, seed=4),
    "mixed_10x6x7": lambda: make_problem(10, 6, 7, log10k=(-13.0, 1.5, 1.0), seed=9,
                                         bc_type=(0, 1, 0, 1, 0, 1),
                                         bc_value=(1.0, 0.5, 0.0, 0.0, 0.2, 0.0)),
    "config2_12": lambda: config_problem(2, size=12),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_structured_level1_product_equals_generic(name, port):
    p = CASES[name]()
    nx, ny, nz = p.nx, p.ny, p.nz
    assert nx % 2 == 0 and nx >= 4 and ny >= 4
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    H = port.amg(cnt, col, ele)
    assert H.nlevels >= 3
    L1, L2 = H.level(1), H.level(2)
    n1 = L1["n"]
    hx = nx // 2
    assert n1 == hx * ny * nz
    rp = np.concatenate([[0], np.cumsum(L1["cnt"])])
    sel = L1["sel"]
    pw = 1.0 / L1["pcnt"].astype(np.float64)
    cid = np.cumsum(sel == 1) - 1  # coarse id of C rows

    def cell(r):
        t, xh = divmod(r, hx)
        z, y = divmod(t, ny)
        return 2 * xh + ((y + z) & 1), y, z

    def row_of(x, y, z):
        return (x + nx * (y + ny * z)) >> 1

    def inside(x, y, z):
        return 0 <= x < nx and 0 <= y < ny and 0 <= z < nz

    b4 = ball(4)
    pairs = {P: [] for P in range(len(b4))}  # (Q, through the centre?) per slot
    for P, off in enumerate(b4):
        for Q, oq in enumerate(Q19):
            d = (off[0] - oq[0], off[1] - oq[1], off[2] - oq[2])
            if d in Q19:
                pairs[P].append((Q, Q19.index(d) == CENTRE))
    # ---- stage 0: (A P) rows, slot -> value (already times w_i)
    ap = []
    for i in range(n1):
        x, y, z = cell(i)
        stored = [q for q, o in enumerate(Q19) if inside(x + o[0], y + o[1], z + o[2])]
        assert rp[i + 1] - rp[i] == len(stored)
        t = [0.0] * 19
        fmask = [False] * 19
        for pos, q in enumerate(stored):
            o = Q19[q]
            j = row_of(x + o[0], y + o[1], z + o[2])
            assert L1["col"][rp[i] + pos] == j
            t[q] = L1["ele"][rp[i] + pos] * pw[j]
            fmask[q] = sel[j] == 2
        row = {}
        for P, off in enumerate(b4):
            kx, ky, kz = x + off[0], y + off[1], z + off[2]
            if not inside(kx, ky, kz) or sel[row_of(kx, ky, kz)] != 1:
                continue
            acc, on = -0.0, False
            for Q, centre in pairs[P]:
                if centre:
                    acc = acc + t[Q]
                    on = True
                else:
                    acc = acc + (t[Q] if fmask[Q] else -0.0)
                    on = on or fmask[Q]
            if on:
                row[off] = acc * pw[i]
        ap.append(row)
    # ---- stage 1: coarse rows by ball-6 slot, R(e) ascending
    cptr = np.concatenate([[0], np.cumsum(L2["cnt"])])
    for c in np.nonzero(sel == 1)[0]:
        x, y, z = cell(c)
        acc = {}
        for o in Q19:
            if not inside(x + o[0], y + o[1], z + o[2]):
                continue
            i = row_of(x + o[0], y + o[1], z + o[2])
            if i != c and sel[i] != 2:
                continue
            for off, v in ap[i].items():
                key = (o[0] + off[0], o[1] + off[1], o[2] + off[2])
                acc[key] = acc[key] + v if key in acc else v
        keys = sorted(acc, key=lambda k: (k[2], k[1], k[0]))
        cols = [cid[row_of(x + k[0], y + k[1], z + k[2])] for k in keys]
        vals = np.array([acc[k] for k in keys])
        e = cid[c]
        assert list(L2["col"][cptr[e]:cptr[e + 1]]) == cols, e
        got = np.ascontiguousarray(L2["ele"][cptr[e]:cptr[e + 1]])
        assert np.array_equal(got.view(np.uint64), vals.view(np.uint64)), e  # bits
