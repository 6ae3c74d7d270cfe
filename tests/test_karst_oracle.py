"""The conduit model of the CPU oracle (oracle/hmfem_oracle.c: or_conduit,
or_picard ...) against fixtures made by the reference's own karst.c /
reservoir.c / main.c-loop sources (tests/golden/make_golden_karst.py), the
data-file readers, and the conduit-set checks of the library (host code, no
GPU needed)."""
import ctypes as C
import hashlib
import os

import numpy as np
import pytest

import karst_cases as KC
from hmfem_b200 import gpu, karst

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module", params=sorted(KC.CASES))
def case(request, port):
    name = request.param
    g = dict(np.load(os.path.join(GOLD, f"karst_{name}.npz")))
    prob, k, WI, pw = KC.CASES[name]()
    perm, _, _ = port.assemble(prob)
    return name, g, prob, k, WI, pw, perm


def test_fixture_inputs_pinned(case):
    name, g, prob, k, WI, pw, perm = case
    assert digest(prob.KX) == str(g["K_digest"])
    assert digest(perm) == str(g["perm_digest"])
    st = KC.step_state(prob, k, 5)
    assert digest(*st) == str(g["state_digest"])


def test_conduit_step_bit_exact_with_reference(case, port):
    """keff (permeabilidade_karst), source terms with fractures and Robin
    ends (source_term1d), the compute()-solved conduit pressures and the
    updated fracture velocities: identical bits."""
    name, g, prob, k, WI, pw, perm = case
    st = KC.step_state(prob, k, 5)
    a = port.conduit_step(k, prob, perm, *st, rho=KC.RHO, solver=1)
    for key in ("kl", "kr", "kc", "f", "pc", "ucR", "ucL"):
        assert np.array_equal(a[key], g["step_" + key]), key


def test_thomas_solves_the_conduit_system(case, port):
    """The batched solve the GPU runs (Thomas) on the same system: residual
    at rounding level; the reference's compute() stops at 1e-8 (pcg.h rule),
    so the two conduit pressures agree to about that."""
    name, g, prob, k, WI, pw, perm = case
    st = KC.step_state(prob, k, 5)
    a = port.conduit_step(k, prob, perm, *st, rho=KC.RHO, solver=0)
    for j in range(k.nk):
        m = k.len[j]
        kl, kc, kr = a["kl"][:m, j], a["kc"][:m, j], a["kr"][:m, j]
        f, x = a["f"][:m, j], a["pc"][:m, j]
        A = np.diag(kc) - np.diag(kl[1:], -1) - np.diag(kr[:-1], 1)
        assert np.linalg.norm(A @ x - f) <= 1e-13 * np.linalg.norm(f)
        ref = g["step_pc"][:m, j]
        assert np.abs(x - ref).max() <= 1e-7 * np.abs(ref).max()
    assert np.array_equal(a["ucR"], g["step_ucR"])


def test_picard_bit_exact_with_reference(case, port):
    """or_picard with the reference's solves (compute(): AMG-PCG, pcg.h
    rule at 1e-8, for the reservoir and every conduit) reproduces the
    reference's coupled run bit for bit, iterations included."""
    name, g, prob, k, WI, pw, perm = case
    r = port.picard(k, prob, WI, pw, rho=KC.RHO, solve_eps=1e-8, solve_stop=0,
                    conduit_solver=1)
    assert r["iterations"] == int(g["run_iterations"])
    for key in ("p", "pc", "ucl", "ucr", "qk", "out"):
        assert np.array_equal(r[key], g["run_" + key]), key
    assert digest(r["v"]) == str(g["run_v_digest"])


def test_picard_with_exact_solves_near_reference(case, port):
    """The GPU's method (Thomas conduits, reservoir to ||r||/||b|| <= 1e-12)
    lands on the reference's answer to the reference's own solver tolerance."""
    name, g, prob, k, WI, pw, perm = case
    r = port.picard(k, prob, WI, pw, rho=KC.RHO, solve_eps=1e-12, solve_stop=1,
                    conduit_solver=0)
    assert abs(r["iterations"] - int(g["run_iterations"])) <= 2
    for key, tol in (("p", 1e-7), ("pc", 1e-7), ("qk", 1e-5)):
        ref = g["run_" + key]
        assert np.abs(r[key] - ref).max() <= tol * np.abs(ref).max(), key


# ---- conduit-set checks: the oracle and the library agree ----------------------

def _bad_sets():
    base = dict(len=[6], sxi=[2], syi=[1], szi=[1], pos=[1], Kc=[1e-11], bound_l=[3],
                bound_r=[3], cont=[[1.0], [1.0]], ccont=[[1.0], [1.0]], kindex=[1e-12],
                area=[1.0], n_brechas=[1], beta=[[1.0]], cb=[[1.0]], brechas=[[2]])
    good = dict(base)
    out = [("ok", good, 0)]
    for label, change in (("x past the grid", dict(len=[8])),
                          ("robin left at the face", dict(sxi=[0], len=[5])),
                          ("robin right at the face", dict(sxi=[3])),
                          ("z robin right", dict(pos=[3], sxi=[2], szi=[0], bound_l=[0],
                                                 len=[3])),
                          ("bad position", dict(pos=[4])),
                          ("bad end code", dict(bound_l=[2])),
                          ("fracture on the last element", dict(brechas=[[5]])),
                          ("negative fracture element", dict(brechas=[[-1]]))):
        d = dict(base)
        d.update(change)
        out.append((label, d, -1))
    return out


@pytest.mark.parametrize("label,spec,want", _bad_sets(), ids=[b[0] for b in _bad_sets()])
def test_conduit_set_checks(label, spec, want, port):
    k = karst.Karst(**spec)
    assert port.karst_check(k, 9, 4, 4) == want
    rc = karst._lib().hmfem_karst_check(C.byref(k.struct()), 9, 4, 4)
    assert (rc == 0) == (want == 0), gpu.last_error()


# ---- the data-file readers -----------------------------------------------------

def _c_read(path, nk):
    L = karst._lib()
    L.hmfem_karst_read.argtypes = [C.c_char_p, C.c_int, C.POINTER(karst.KarstStruct)]
    L.hmfem_karst_release.argtypes = [C.POINTER(karst.KarstStruct)]
    s = karst.KarstStruct()
    rc = L.hmfem_karst_read(path.encode(), nk, C.byref(s))
    assert rc == 0, gpu.last_error()
    mb = s.max_brechas

    def arr(ptr, n, ct):
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), (n,)).copy() if n else \
            np.zeros(0)
    out = dict(len=arr(s.len, nk, C.c_int), sxi=arr(s.sxi, nk, C.c_int),
               syi=arr(s.syi, nk, C.c_int), szi=arr(s.szi, nk, C.c_int),
               pos=arr(s.pos, nk, C.c_int), Kc=arr(s.Kc, nk, C.c_double),
               bound_l=arr(s.bound_l, nk, C.c_int), bound_r=arr(s.bound_r, nk, C.c_int),
               cont=arr(s.cont, 2 * nk, C.c_double), ccont=arr(s.ccont, 2 * nk, C.c_double),
               kindex=arr(s.kindex, nk, C.c_double), area=arr(s.area, nk, C.c_double),
               n_brechas=arr(s.n_brechas, nk, C.c_int),
               beta=arr(s.beta, mb * nk, C.c_double), cb=arr(s.cb, mb * nk, C.c_double),
               brechas=arr(s.brechas, mb * nk, C.c_int))
    L.hmfem_karst_release(C.byref(s))
    return out


@pytest.mark.parametrize("fname,nk", [("karst_data_1_2.dat", 1), ("karst_data_3_2.dat", 3)])
def test_data_file_readers(fname, nk):
    path = os.path.join(GOLD, fname)
    k = karst.Karst.read(path, nk)
    c = _c_read(path, nk)
    for f in c:
        assert np.array_equal(np.asarray(getattr(k, f)).reshape(-1), c[f].reshape(-1)), f
    # the reference run's conduit (data_1_2.dat): 123 elements along x from
    # (44, 21, 9), nonlinear Robin ends, fractures at elements 25 and 96
    if nk == 1:
        assert k.len[0] == 123 and (k.sxi[0], k.syi[0], k.szi[0]) == (44, 21, 9)
        assert k.bound_l[0] == 3 and k.bound_r[0] == 3
        assert list(k.brechas[:, 0]) == [25, 96] and k.beta[0, 0] == 1e8 - 1


def test_short_data_file_is_rejected(tmp_path):
    p = tmp_path / "short.dat"
    p.write_text("123\n44\n21\n")
    with pytest.raises(ValueError):
        karst.Karst.read(str(p), 1)
    L = karst._lib()
    L.hmfem_karst_read.argtypes = [C.c_char_p, C.c_int, C.POINTER(karst.KarstStruct)]
    s = karst.KarstStruct()
    assert L.hmfem_karst_read(str(p).encode(), 1, C.byref(s)) == gpu.E_ARG
