"""The exact red-black reduction of level 0 (hmfem_options.schur0) on the
GPU: level 1 bit-exact with the restatement (oracle/schur.py), the
reference's structure on every level, an exact preconditioner when level 1
is solved exactly, and solves that land on the FP64 oracle's pressure."""
import numpy as np
import pytest
import scipy.sparse as sp

from hmfem_b200 import gpu
from hmfem_b200.problem import config_problem, make_problem
from oracle import schur as S

pytestmark = pytest.mark.gpu

CASES = {
    "mixed_8x6x5": lambda: make_problem(8, 6, 5, log10k=(-14.0, 1.0, 1.5), n_conduits=1, seed=4,
                                        bc_type=(0, 1, 0, 1, 0, 1),
                                        bc_value=(1.0, 0.5, 0.0, 0.0, 0.2, 0.0)),
    "odd_7x6x5": lambda: make_problem(7, 6, 5, log10k=(-14.0, 1.0, 1.5), seed=9),
    "config1_24": lambda: config_problem(1, size=24),
    "config2_32": lambda: config_problem(2, size=32),
}


def _solver(**kw):
    return gpu.Solver(precision=1, schur0=1, **kw)


@pytest.mark.parametrize("name", sorted(CASES))
def test_level1_is_the_schur_complement_bit_exact(name, port):
    p = CASES[name]()
    perm, ind, b = port.assemble(p)
    s = _solver()
    s.assemble(p)
    s.setup()
    L1 = s.level(1)
    cnt, col, ele = S.schur_level1(perm, p.nx, p.ny, p.nz)
    assert np.array_equal(L1["cnt"], cnt) and np.array_equal(L1["col"], col)
    assert np.array_equal(L1["ele"], ele)
    # every level keeps the reference's structure
    r = gpu.Solver(precision=1)
    r.assemble(p)
    r.setup()
    assert s.num_levels() == r.num_levels()
    for l in range(s.num_levels()):
        a, c = s.level(l), r.level(l)
        for key in ("cnt", "col", "sel", "pcnt", "pcol"):
            assert np.array_equal(a[key], c[key]), (l, key)
    s.close()
    r.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_levels_below_the_schur_level_bit_exact(name, port):
    """Levels >= 2 are the reference's setup (split, P, Galerkin product)
    applied to the Schur level 1, so the oracle's setup of that matrix gives
    them bit for bit -- the product from the 19-offset structure (even nx)
    and the generic one (odd nx) alike."""
    p = CASES[name]()
    perm, ind, b = port.assemble(p)
    cnt, col, ele = S.schur_level1(perm, p.nx, p.ny, p.nz)
    H = port.amg(cnt, col, ele)
    s = _solver()
    s.assemble(p)
    s.setup()
    depth = min(H.nlevels, s.num_levels() - 1)
    assert depth >= 2
    for l in range(depth):
        g, o = s.level(l + 1), H.level(l)
        keys = ("cnt", "col", "ele", "dinv")
        if l < depth - 1:
            keys += ("sel", "pcnt", "pcol")
        for key in keys:
            assert np.array_equal(g[key], o[key]), (l + 1, key)
    s.close()


@pytest.mark.parametrize("dims", [(8, 8, 8), (10, 9, 7), (6, 5, 3), (10, 10, 10)],
                         ids=lambda d: "x".join(map(str, d)))
def test_exact_when_level1_is_solved_exactly(dims, port):
    """The dense direct solve below level 0's size (at most 512 rows):
    level 1 (n/2 rows: 256, 315, 45 and 500 -- whole and ragged blocks of
    the Gauss-Jordan steps, up to the dense limit) is solved exactly, so one
    cycle is A^-1 (to the cycle's rounding) and the flexible CG needs two
    steps."""
    p = make_problem(*dims, log10k=(-14.0, 1.0, 1.0), seed=2)
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    ptr = np.zeros(p.n + 1, np.int64)
    ptr[1:] = np.cumsum(cnt)
    A = sp.csr_matrix((ele, col, ptr), shape=(p.n, p.n)).toarray()
    s = _solver(tol=1e-10, coarse_direct=min(512, p.n - 1))
    s.assemble(p)
    s.setup()
    f = np.random.default_rng(0).standard_normal(p.n)
    u = s.vcycle(f)  # the FP64 cycle
    want = np.linalg.solve(A, f)
    assert np.linalg.norm(u - want) <= 1e-10 * np.linalg.norm(want)
    x, st = s.solve()
    assert st["status"] == 0 and st["iterations"] <= 2, st
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_solve_matches_oracle(name, port):
    p = CASES[name]()
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    H = port.amg(cnt, col, ele)
    xo, _, _ = H.pcg(b, eps=1e-12, stop=1)
    its = {}
    for schur in (0, 1):
        s = gpu.Solver(precision=1, schur0=schur, tol=1e-12, bf16_from=1)
        s.assemble(p)
        s.setup()
        x, st = s.solve()
        s.close()
        assert st["status"] == 0 and st["relres"] <= 1e-12
        assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)
        its[schur] = st["iterations"]
    assert its[1] <= its[0], its


def test_packed_bf16_levels_match_the_unpacked_form(monkeypatch):
    """BF16 levels stored as one word per entry (int16 column offset + BF16
    bits) give the very same solve as the column + value arrays."""
    p = config_problem(2, size=48)
    out = {}
    for pack in ("1", "0"):
        monkeypatch.setenv("HMFEM_PACK16", pack)
        s = gpu.Solver(precision=1, schur0=1, bf16_from=1, tol=1e-10)
        s.assemble(p)
        s.setup()
        x, st = s.solve()
        s.close()
        assert st["status"] == 0
        out[pack] = (x, st["iterations"])
    assert out["1"][1] == out["0"][1]
    assert np.array_equal(out["1"][0], out["0"][0])
