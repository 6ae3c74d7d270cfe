"""The coupled reservoir / conduit model on the GPU (include/hmfem_karst.h)
against the CPU oracle's restatement and the reference's own coupled run
(tests/golden/karst_*.npz).

Bars: the batched conduit solve (keff, source terms, Thomas) is bit-exact
with the oracle's; the coupled run agrees with the oracle run with the same
solves (Thomas conduits, reservoir to ||r||/||b|| <= 1e-12) to 1e-8 in the
pressures (the Picard tolerance), and with the reference's run (its solves
stop at 1e-8) to 1e-7.
"""
import ctypes as C
import os

import numpy as np
import pytest

import karst_cases as KC
from hmfem_b200 import gpu, karst

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", params=sorted(KC.CASES))
def case(request, port):
    name = request.param
    g = dict(np.load(os.path.join(GOLD, f"karst_{name}.npz")))
    prob, k, WI, pw = KC.CASES[name]()
    perm, _, _ = port.assemble(prob)
    return name, g, prob, k, WI, pw, perm


@pytest.fixture(scope="module")
def oracle_runs(port):
    out = {}
    for name, mk in KC.CASES.items():
        prob, k, WI, pw = mk()
        out[name] = port.picard(k, prob, WI, pw, rho=KC.RHO, solve_eps=1e-12,
                                solve_stop=1, conduit_solver=0)
    return out


@pytest.mark.parametrize("seed", [5, 6])
def test_conduit_step_bit_exact(case, port, seed):
    name, g, prob, k, WI, pw, perm = case
    st = KC.step_state(prob, k, seed)
    a = karst.conduit_step(k, prob, *st, rho=KC.RHO)
    b = port.conduit_step(k, prob, perm, *st, rho=KC.RHO, solver=0)
    for key in ("pc", "kl", "kr", "kc", "ucR", "ucL"):
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("precision", [0, 1])
def test_picard_matches_oracle_and_reference(case, oracle_runs, precision):
    name, g, prob, k, WI, pw, perm = case
    s = gpu.Solver(precision=precision, tol=1e-12, stop_rule=0)
    r = karst.picard(s, k, prob, WI, pw, rho=KC.RHO)
    s.close()
    o = oracle_runs[name]
    st = r["stats"]
    assert st["status"] == 0 and st["setups"] == 2
    assert abs(st["iterations"] - o["iterations"]) <= 1
    assert st["error"] <= 1e-8
    # Both runs stop when the reservoir pressure changes by <= 1e-8 and solve
    # each reservoir system to 1e-12 (their AMG-PCG iterates round
    # differently), so the pressures agree to about the Picard tolerance.
    for key in ("p", "pc"):
        assert np.abs(r[key] - o[key]).max() <= 1e-8 * np.abs(o[key]).max(), key
        ref = g["run_" + key]
        assert np.abs(r[key] - ref).max() <= 1e-7 * np.abs(ref).max(), key
    # fluxes and balances are differences of those pressures (a few kPa out
    # of 60 MPa), so their relative agreement is correspondingly looser
    for key in ("ucl", "ucr"):
        assert np.abs(r[key] - o[key]).max() <= 1e-5 * np.abs(o[key]).max(), key
    assert np.allclose(r["qk"], o["qk"], rtol=1e-4, atol=1e-5 * np.abs(o["qk"]).max())
    v = r["v"][:, [0, 1, 2, 3, 5, 6]]
    vo = o["v"][:, [0, 1, 2, 3, 5, 6]]
    assert np.abs(v - vo).max() <= 1e-5 * np.abs(vo).max()
    assert abs(st["q_well"] - o["out"][1]) <= 1e-6 * abs(o["out"][1])
    assert abs(st["p_mean"] - o["out"][2]) <= 1e-8 * abs(o["out"][2])


def test_picard_device_arrays_match_host():
    """mem = 1: K, WI, pw and the outputs in device memory."""
    torch = pytest.importorskip("torch")
    prob, k, WI, pw = KC.case_multi()
    s = gpu.Solver(precision=1, tol=1e-12, stop_rule=0)
    host = karst.picard(s, k, prob, WI, pw, rho=KC.RHO, fluxes=False)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    K = dev(prob.KX)
    dWI, dpw = dev(WI), dev(pw)
    p = torch.zeros(prob.n, dtype=torch.float64, device="cuda")
    pc = torch.zeros(k.mmax * k.nk, dtype=torch.float64, device="cuda")
    o = karst.PicardOptions(KC.RHO, 1e-8, 1000)
    st = karst.PicardStats()
    bct = np.asarray(prob.bc_type, dtype=np.int32)
    bcv = np.asarray(prob.bc_value, dtype=np.float64)
    ks = k.struct()
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = karst._lib().hmfem_picard(
        s.h, C.byref(ks), prob.nx, prob.ny, prob.nz, prob.hx, prob.hy, prob.hz, prob.visc,
        vp(K), vp(K), vp(K), C.c_void_p(bct.ctypes.data), C.c_void_p(bcv.ctypes.data),
        vp(dWI), vp(dpw), C.byref(o), vp(p), vp(pc), 1, C.byref(st))
    torch.cuda.synchronize()
    s.close()
    assert rc == 0, gpu.last_error()
    assert st.iterations == host["stats"]["iterations"]
    assert np.array_equal(p.cpu().numpy(), host["p"])
    assert np.array_equal(pc.cpu().numpy().reshape(k.mmax, k.nk), host["pc"])


def test_picard_rejects_a_conduit_leaving_the_grid():
    prob, k, WI, pw = KC.case_single()
    k.len[0] = 40
    s = gpu.Solver()
    with pytest.raises(gpu.HmfemError):
        karst.picard(s, k, prob, WI, pw)
    s.close()


def test_picard_fluxes_need_a_run():
    s = gpu.Solver()
    rc = karst._lib().hmfem_picard_fluxes(s.h, None, None, None, 0)
    s.close()
    assert rc == gpu.E_ARG
