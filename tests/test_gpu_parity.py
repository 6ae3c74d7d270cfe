"""GPU parity: the sm_100a path (through the C-ABI) against the CPU oracle.

Bit-exact for assembly, right-hand side, the whole AMG hierarchy (integer
structure and values), SpMV, one V-cycle and the fluxes of a given pressure;
within stated tolerances for the iterative solves (the GPU smoother is
Jacobi-type, the oracle's is Gauss-Seidel, so iterates differ while both
converge to the same discrete solution).
"""
import importlib.util
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import config_problem, make_problem  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location(
    "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

CASES = dict(make_golden.CASES)
CASES.update({
    "line_1x1x9": lambda: make_problem(1, 1, 9, log10k=None, seed=1,
                                       bc_type=(0, 0, 1, 1, 0, 1),
                                       bc_value=(1.0, 0.0, 0, 0, 0.25, 0)),
    "single_cell": lambda: make_problem(1, 1, 1, bc_type=(0, 0, 1, 1, 1, 1)),
    "ragged_5x3x7": lambda: make_problem(5, 3, 7, log10k=(-14.0, 2.0, 1.0),
                                         n_conduits=1, seed=9),
    "conduit_40": lambda: config_problem(1, size=40),
    "slab_8x6x1": lambda: make_problem(8, 6, 1, log10k=(-13.0, 1.0, 1.0), seed=4),
})

# Pressure / flux tolerance against the FP64 oracle when both are solved to
# ||b - A x|| / ||b|| <= 1e-12: 1e-9 relative (the bar the FP64 path is held to).
P_RTOL = 1e-9


def _oracle(port, p):
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    return perm, ind, b, (cnt, col, ele), port.amg(cnt, col, ele)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, port):
    p = CASES[request.param]()
    return request.param, p, _oracle(port, p)


def test_assembly_and_rhs_bit_exact(case):
    name, p, (perm, ind, b, csr, H) = case
    s = gpu.Solver()
    s.assemble(p)
    s.setup()
    d = s.level(0)
    np.testing.assert_array_equal(d["cnt"], csr[0])
    np.testing.assert_array_equal(d["col"], csr[1])
    np.testing.assert_array_equal(d["ele"], csr[2])
    np.testing.assert_array_equal(s.rhs(), b)


def test_stencil_packing_bit_exact(case):
    name, p, (perm, ind, b, csr, H) = case
    s = gpu.Solver()
    s.set_stencil(p.nx, p.ny, p.nz, np.ascontiguousarray(perm),
                  np.ascontiguousarray(ind), b)
    s.setup()
    d = s.level(0)
    np.testing.assert_array_equal(d["cnt"], csr[0])
    np.testing.assert_array_equal(d["col"], csr[1])
    np.testing.assert_array_equal(d["ele"], csr[2])


@pytest.mark.parametrize("generic_setup", [0, 1])
def test_hierarchy_bit_exact(case, generic_setup):
    """Level 0 from hmfem_assemble is coarsened from its 7-point structure
    (generic_setup=0) or by the generic kernels; both must equal the
    reference's hierarchy bit for bit."""
    name, p, (perm, ind, b, csr, H) = case
    s = gpu.Solver(generic_setup=generic_setup)
    s.assemble(p)
    s.setup()
    assert s.num_levels() == H.nlevels
    for l in range(H.nlevels):
        g, o = s.level(l), H.level(l)
        assert g["n"] == o["n"]
        for k in ("cnt", "col", "ele", "dinv", "sel", "pcnt", "pcol"):
            np.testing.assert_array_equal(g[k], o[k], err_msg=f"L{l} {k}")


@pytest.mark.parametrize("smoother,gs_from,cheb,oracle_smoother,omega",
                         [(0, -1, None, 1, 1.0), (0, -1, None, 1, 0.6),
                          (1, -1, None, 2, 1.0), (1, 2, None, 12, 1.0),
                          (1, 1, None, 11, 1.0), (1, 2, (2, 3), 223, 1.0),
                          (1, 2, (1, 2), 212, 1.0), (1, 2, (2, 4), 224, 1.0)])
@pytest.mark.parametrize("generic_setup", [0, 1])
def test_vcycle_bit_exact(case, smoother, gs_from, cheb, oracle_smoother, omega,
                          generic_setup):
    """generic_setup=0 runs the two finest levels of an assembled grid in
    their structured forms (7-point stencil, 19-offset level 1),
    generic_setup=1 everything on SELL-32; both equal the oracle's cycle.
    cheb = (first level, degree) of the Chebyshev coarse smoother."""
    name, p, (perm, ind, b, csr, H) = case
    cheb_from, cheb_degree = cheb if cheb else (-1, 3)
    # coarse_direct=0: the reference's diagonal solve on the coarsest level
    s = gpu.Solver(smoother=smoother, gs_from=gs_from, omega=omega,
                   coarse_direct=0, generic_setup=generic_setup,
                   cheb_from=cheb_from, cheb_degree=cheb_degree)
    s.assemble(p)
    s.setup()
    f = np.random.default_rng(11).standard_normal(p.n)
    np.testing.assert_array_equal(s.vcycle(f), H.vcycle(f, oracle_smoother, omega))


@pytest.mark.parametrize("gs_from,oracle_smoother", [(2, 12), (1, 11)])
def test_vcycle_gs_fused_sweeps(case, gs_from, oracle_smoother):
    """gs_fused=1: each Gauss-Seidel sweep as one cooperative launch with
    grid barriers between colours instead of one launch per colour; the
    same bits either way."""
    name, p, (perm, ind, b, csr, H) = case
    s = gpu.Solver(smoother=1, gs_from=gs_from, coarse_direct=0, gs_fused=1,
                   cheb_from=-1)
    s.assemble(p)
    s.setup()
    f = np.random.default_rng(11).standard_normal(p.n)
    np.testing.assert_array_equal(s.vcycle(f), H.vcycle(f, oracle_smoother, 1.0))


@pytest.mark.parametrize("generic_setup", [0, 1])
def test_spmv_bit_exact(case, port, generic_setup):
    name, p, (perm, ind, b, csr, H) = case
    s = gpu.Solver(generic_setup=generic_setup)
    s.assemble(p)
    s.setup()
    x = np.random.default_rng(3).standard_normal(p.n)
    np.testing.assert_array_equal(s.spmv(0, x), port.spmv(*csr, x))
    if H.nlevels > 1:
        d = H.level(1)
        x1 = np.random.default_rng(4).standard_normal(d["n"])
        np.testing.assert_array_equal(s.spmv(1, x1),
                                      port.spmv(d["cnt"], d["col"], d["ele"], x1))


@pytest.mark.parametrize("dims", [(64, 48, 40), (130, 6, 5), (2, 3, 4), (96, 1, 7)],
                         ids=lambda d: "x".join(map(str, d)))
def test_spmv_pairs_bit_exact(dims, port):
    """The level-0 SpMV on x-adjacent cell pairs (nx even, 16-byte loads)
    against the oracle's CSR SpMV, bit for bit: rows, planes and the grid's
    faces."""
    p = make_problem(*dims, log10k=(-14.0, 1.0, 1.5), n_conduits=1, seed=sum(dims))
    perm, ind, b = port.assemble(p)
    s = gpu.Solver()
    s.assemble(p)
    s.setup()
    x = np.random.default_rng(5).standard_normal(p.n)
    np.testing.assert_array_equal(s.spmv(0, x), port.spmv(*port.pack(perm, ind), x))
    s.close()


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_and_fluxes_match_oracle(case, port, precision):
    name, p, (perm, ind, b, csr, H) = case
    xo, ito, relo = H.pcg(b, eps=1e-12, stop=1)
    s = gpu.Solver(precision=precision, tol=1e-12)
    s.assemble(p)
    s.setup()
    x, st = s.solve()
    assert st["status"] == 0
    assert st["relres"] <= 1e-12
    r = b - port.spmv(*csr, x)
    assert np.linalg.norm(r) <= 1.001e-12 * np.linalg.norm(b)
    assert _rel(x, xo) <= P_RTOL
    v, dmin, dmax = s.fluxes(x)
    vo, _, _ = port.fluxes(p, perm, xo)
    faces = [0, 1, 2, 3, 5, 6]
    assert _rel(v[:, faces], vo[:, faces]) <= P_RTOL
    # per-cell mass balance: divergence = row residual
    assert dmax <= np.abs(r).max() + 1e-14 * np.abs(b).max()
    # fluxes of the same pressure are bit-identical to flux_reconstruction.c
    v2, _, _ = s.fluxes(xo)
    np.testing.assert_array_equal(v2[:, faces], vo[:, faces])


def test_plain_solve_meets_metric_tolerance(port):
    p = config_problem(2, size=48)
    perm, ind, b, csr, H = _oracle(port, p)
    s = gpu.Solver(tol=1e-10)
    s.assemble(p)
    s.setup()
    x, st = s.solve()
    r = b - port.spmv(*csr, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10
    assert st["iterations"] < 200


def test_compute_dropin_matches_reference_rule(port):
    p = config_problem(1, size=24)
    perm, ind, b, (cnt, col, ele), H = _oracle(port, p)
    hdr = np.array([p.n, len(col)], np.int32)
    x = np.zeros(p.n)
    assert gpu.compute(hdr, cnt, col, ele, b.copy(), x) == 0
    # reference rule at 1e-8 on the preconditioned residual (compute.cpp:41)
    xo, it, rel = H.pcg(b, eps=1e-8, stop=0)
    assert _rel(x, xo) < 1e-6
    assert gpu.iter_amg() > 1


def test_solve_linsys_dropin_warm_start(port):
    p = config_problem(2, size=16)
    perm, ind, b, csr, H = _oracle(port, p)
    xo, _, _ = H.pcg(b, eps=1e-12, stop=1)
    x = xo * (1 + 1e-6)  # warm start (reservoir passes the previous p)
    gpu.solve_linsys(np.ascontiguousarray(perm), np.ascontiguousarray(ind),
                     b.copy(), x, p.nx, p.ny, p.nz)
    assert _rel(x, xo) < 1e-6


def test_setup_reuse_keeps_hierarchy_for_unchanged_matrix(port):
    """reuse_setup=1 (the reference bridge's setting): handing the same
    matrix again keeps the hierarchy -- the solve with a new right-hand side
    is bit-identical to a fresh solver's -- and any changed value rebuilds
    it."""
    p = config_problem(2, size=24)
    perm, ind, b, (cnt, col, ele), H = _oracle(port, p)
    s = gpu.Solver(tol=1e-10, reuse_setup=1)
    s.set_matrix(cnt, col, ele, b)
    s.setup()
    x1, st1 = s.solve()
    assert st1["setup_reused"] == 0
    b2 = np.random.default_rng(8).standard_normal(p.n)
    s.set_matrix(cnt, col, ele.copy(), b2)
    s.setup()
    x2, st2 = s.solve()
    assert st2["setup_reused"] == 1
    fresh = gpu.Solver(tol=1e-10)
    fresh.set_matrix(cnt, col, ele, b2)
    fresh.setup()
    x3, st3 = fresh.solve()
    np.testing.assert_array_equal(x2, x3)
    # one changed value (a larger diagonal keeps it SPD): rebuilt
    ele4 = ele.copy()
    rp = np.concatenate([[0], np.cumsum(cnt)])
    d0 = rp[0] + int(np.nonzero(col[rp[0]:rp[1]] == 0)[0][0])
    ele4[d0] *= 1.5
    s.set_matrix(cnt, col, ele4, b)
    s.setup()
    x4, st4 = s.solve()
    assert st4["setup_reused"] == 0
    H4 = port.amg(cnt, col, ele4)
    xo, _, _ = H4.pcg(b, eps=1e-12, stop=1)
    assert _rel(x4, xo) < 1e-8


def test_compute_bridge_repeated_calls(port):
    """The reservoir loop calls compute with the same matrix each Picard
    iteration; the second call reuses the setup and returns the same x."""
    p = config_problem(1, size=16)
    perm, ind, b, (cnt, col, ele), H = _oracle(port, p)
    hdr = np.array([p.n, len(col)], np.int32)
    xa = np.zeros(p.n)
    xb = np.zeros(p.n)
    assert gpu.compute(hdr, cnt, col, ele, b.copy(), xa) == 0
    ia = gpu.iter_amg()
    assert gpu.compute(hdr, cnt, col, ele, b.copy(), xb) == 0
    np.testing.assert_array_equal(xa, xb)
    assert gpu.iter_amg() == ia


def test_device_pointers_in_place():
    p = config_problem(2, size=24)
    s = gpu.Solver(tol=1e-10)
    K = torch.tensor(p.KX, device="cuda")
    s.assemble(p, KX=K, KY=K, KZ=K)
    s.setup()
    x = torch.zeros(p.n, dtype=torch.float64, device="cuda")
    s.solve(x=x)
    torch.cuda.synchronize()
    s2 = gpu.Solver(tol=1e-10)
    s2.assemble(p)
    xh, _ = s2.solve()
    assert _rel(x.cpu().numpy(), xh) < 1e-9


def test_device_abi_layer_matches_formulas():
    """The reference's _device_* entry points (toolbox.cu) on device data."""
    import ctypes as C
    L = gpu.lib()
    rng = np.random.default_rng(5)
    n = 1000
    xh, yh, zh = rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(n)
    x, y, z = (torch.tensor(a, device="cuda") for a in (xh, yh, zh))
    vp = C.c_void_p
    L._device_add_scale.argtypes = [vp, vp, C.c_double, C.c_uint]
    L._device_add_scale(x.data_ptr(), y.data_ptr(), 0.5, n)
    L._device_scale_add.argtypes = [vp, vp, C.c_double, C.c_uint]
    L._device_scale_add(y.data_ptr(), z.data_ptr(), 2.0, n)
    L._device_rsb.argtypes = [vp, vp, C.c_uint]
    L._device_rsb(z.data_ptr(), x.data_ptr(), n)
    torch.cuda.synchronize()
    x1 = xh + yh * 0.5
    y1 = yh * 2.0 + zh
    np.testing.assert_array_equal(y.cpu().numpy(), y1)
    np.testing.assert_array_equal(x.cpu().numpy(), zh - x1)
    w = torch.zeros(60, dtype=torch.float64, device="cuda")
    L._device_vector_product.argtypes = [vp, vp, vp, C.c_uint, C.c_uint]
    L._device_vector_product(y.data_ptr(), y.data_ptr(), w.data_ptr(), n, 60)
    torch.cuda.synchronize()
    assert w.sum().item() == pytest.approx(float(y1 @ y1), rel=1e-12)


def test_notconv_status_is_reported():
    p = config_problem(2, size=24)
    s = gpu.Solver(tol=1e-14, max_iter=3)
    s.assemble(p)
    x, st = s.solve(allow_notconv=True)
    assert st["status"] == gpu.E_NOTCONV
    assert st["iterations"] == 3


def test_bad_boundary_type_rejected():
    p = make_problem(4, 4, 4, bc_type=(2, 0, 1, 1, 1, 1))
    s = gpu.Solver()
    with pytest.raises(gpu.HmfemError) as e:
        s.assemble(p)
    assert e.value.code == gpu.E_ARG
