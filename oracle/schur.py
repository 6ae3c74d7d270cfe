"""Restatement of the exact red-black reduction of level 0 (TEST
INFRASTRUCTURE ONLY: the checker for hmfem_options.schur0).

Level 1 = the Schur complement S = A_CC - A_CF A_FF^-1 A_FC of the parity
split (C: i+j+k even), evaluated in the order the device kernel uses
(k_schur_fill) so the values can be compared bit for bit; plus the
algebraic reference P^T A P with P_F = -A_FF^-1 A_FC (scipy) that the
restatement is checked against.
"""
import numpy as np

# level-0 row order d, l, c, r, u, t, b (solve_linearsystem_AMG.c:103-139)
DIRS = [("d", (0, -1, 0)), ("l", (-1, 0, 0)), ("c", (0, 0, 0)), ("r", (1, 0, 0)),
        ("u", (0, 1, 0)), ("t", (0, 0, 1)), ("b", (0, 0, -1))]
ELE = {"u": 0, "d": 1, "l": 2, "r": 3, "c": 4, "t": 5, "b": 6}
# the 19 coarse offsets by slot (k_sg_fill / k_schur_fill numbering)
SLOTS = [(0, 0, 0), (2, 0, 0), (-2, 0, 0), (0, 2, 0), (0, -2, 0), (0, 0, 2), (0, 0, -2),
         (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1), (-1, 0, 1),
         (-1, 0, -1), (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1)]


def schur_level1(perm, nx, ny, nz):
    """(cnt, col, ele) of level 1, rows and columns in coarse-id order
    (C cells by ascending fine index), every value in k_schur_fill's order."""
    perm = np.asarray(perm).reshape(-1, 7)
    nxy = nx * ny

    def inside(i, j, k):
        return 0 <= i < nx and 0 <= j < ny and 0 <= k < nz

    def a(s, name):          # matrix entry of row s toward `name` (CSR value)
        return perm[s, ELE["c"]] if name == "c" else -perm[s, ELE[name]]

    cidx = {}
    for s in range(nx * ny * nz):
        i, j, k = s % nx, (s // nx) % ny, s // nxy
        if (i + j + k) % 2 == 0:
            cidx[s] = len(cidx)
    cnt, col, ele = [], [], []
    for s, c in cidx.items():
        i, j, k = s % nx, (s // nx) % ny, s // nxy
        acc = {}
        dsum = a(s, "c")
        for name, (dx, dy, dz) in DIRS:
            if name == "c" or not inside(i + dx, j + dy, k + dz):
                continue
            f = s + dx + dy * nx + dz * nxy
            a_ce, a_ff = a(s, name), a(f, "c")
            dsum = dsum - (a_ce * a_ce) / a_ff
            for n2, (ex, ey, ez) in DIRS:
                if n2 == "c" or not inside(i + dx + ex, j + dy + ey, k + dz + ez):
                    continue
                off = (dx + ex, dy + ey, dz + ez)
                if off == (0, 0, 0) or off not in SLOTS:
                    continue
                t = (a_ce * a(f, n2)) / a_ff
                acc[off] = acc[off] + t if off in acc else t
        row = []
        for off in SLOTS:
            q = (i + off[0], j + off[1], k + off[2])
            if not inside(*q):
                continue
            v = dsum if off == (0, 0, 0) else -acc[off]
            row.append((cidx[q[0] + q[1] * nx + q[2] * nxy], v))
        row.sort()
        cnt.append(len(row))
        col += [r[0] for r in row]
        ele += [r[1] for r in row]
    return np.array(cnt, np.int32), np.array(col, np.int32), np.array(ele)


def galerkin_direct(A, nx, ny, nz):
    """P^T A P (scipy) with P_F = -A_FF^-1 A_FC, P_C = I for the parity
    split: the same operator in exact arithmetic."""
    import scipy.sparse as sp
    A = sp.csr_matrix(A)
    n = A.shape[0]
    s = np.arange(n)
    par = (s % nx + (s // nx) % ny + s // (nx * ny)) % 2
    C = np.where(par == 0)[0]
    cid = -np.ones(n, np.int64)
    cid[C] = np.arange(len(C))
    d = A.diagonal()
    rows, cols, vals = [], [], []
    for i in range(n):
        if par[i] == 0:
            rows.append(i); cols.append(cid[i]); vals.append(1.0)
        else:
            a, b = A.indptr[i], A.indptr[i + 1]
            for q in range(a, b):
                j = A.indices[q]
                if j != i:
                    rows.append(i); cols.append(cid[j]); vals.append(-A.data[q] / d[i])
    P = sp.csr_matrix((vals, (rows, cols)), shape=(n, len(C)))
    return (P.T @ A @ P).tocsr()
