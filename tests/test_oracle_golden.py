"""The CPU oracle (oracle/hmfem_oracle.c) against fixtures produced by the
reference's own sources (tests/golden/make_golden.py): bit-exact."""
import hashlib
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
_spec = importlib.util.spec_from_file_location(
    "make_golden", os.path.join(GOLD, "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)
CASES = make_golden.CASES


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, port):
    name = request.param
    g = dict(np.load(os.path.join(GOLD, name + ".npz")))
    p = CASES[name]()
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    H = port.amg(cnt, col, ele)
    return name, g, p, (perm, ind, b), (cnt, col, ele), H


def test_inputs_and_assembly(case):
    name, g, p, (perm, ind, b), csr, H = case
    assert digest(p.KX) == str(g["K_digest"])          # generator pinned
    assert digest(b) == str(g["b_digest"])
    assert digest(*csr) == str(g["csr_digest"])
    if "perm" in g:
        np.testing.assert_array_equal(perm, g["perm"])
        np.testing.assert_array_equal(ind, g["ind"])


def test_hierarchy_bit_exact(case, port):
    name, g, p, _, csr, H = case
    assert H.nlevels == int(g["nlevels"])
    for l in range(H.nlevels):
        d = H.level(l)
        assert d["n"] == g["level_n"][l]
        assert len(d["col"]) == g["level_nnz"][l]
        assert len(d["pcol"]) == g["level_pnnz"][l]
        assert digest(d["cnt"], d["col"], d["sel"], d["pcnt"], d["pcol"]) == str(g[f"L{l}_struct"])
        assert digest(d["ele"], d["dinv"], d["pele"]) == str(g[f"L{l}_values"])


def test_vcycle_pcg_flux_bit_exact(case):
    name, g, p, (perm, ind, b), csr, H = case
    f = np.random.default_rng(7).standard_normal(p.n)
    assert digest(H.vcycle(f, smoother=0)) == str(g["vcycle_digest"])
    x8, it8, _ = H.pcg(b, eps=1e-8, stop=0)
    assert it8 == int(g["iters_ref8"])
    assert digest(x8) == str(g["x_ref8_digest"])
    x, it, rel = H.pcg(b, eps=1e-12, stop=1)
    assert it == int(g["iters"])
    assert digest(x) == str(g["x_digest"])
    assert rel == pytest.approx(float(g["relres"]), rel=0, abs=0)


def test_flux_bit_exact(case, port):
    name, g, p, (perm, ind, b), csr, H = case
    x, _, _ = H.pcg(b, eps=1e-12, stop=1)
    v, dmin, dmax = port.fluxes(p, perm, x)
    assert digest(v[:, [0, 1, 2, 3, 5, 6]]) == str(g["flux_digest"])


def test_config0_closed_form(port):
    """Homogeneous K, Dirichlet 1/0 on x, no-flow elsewhere: TPFA is exact
    for the linear solution p_i = 1 - (i + 1/2)/nx."""
    p = CASES["config0_32"]()
    perm, ind, b = port.assemble(p)
    H = port.amg(*port.pack(perm, ind))
    x, it, rel = H.pcg(b, eps=1e-12, stop=1)
    i = np.arange(p.n) % p.nx
    np.testing.assert_allclose(x, 1.0 - (i + 0.5) / p.nx, rtol=1e-9, atol=1e-11)
    v, dmin, dmax = port.fluxes(p, perm, x)
    # divvel_pontual's per-cell divergence is the row residual (A p - b)_s,
    # so max |div| = ||r||_inf <= ||r||_2 = relres * ||b||_2
    r = b - port.spmv(*port.pack(perm, ind), x)
    # (the two differ by rounding of O(eps * |diag * p|))
    assert dmax == pytest.approx(np.abs(r).max(), rel=0, abs=1e-15 * np.abs(b).max())
    assert dmax <= rel * np.linalg.norm(b) * (1 + 1e-9)


def test_first_levels_are_parity_colouring(port):
    """Level 0 coarsening of the 7-point stencil = (i+j+k) even."""
    p = CASES["config1_24"]()
    perm, ind, b = port.assemble(p)
    H = port.amg(*port.pack(perm, ind))
    d = H.level(0)
    s = np.arange(p.n)
    i, j, k = s % p.nx, (s // p.nx) % p.ny, s // (p.nx * p.ny)
    np.testing.assert_array_equal(d["sel"] == 1, (i + j + k) % 2 == 0)
