"""ctypes front-end of the correctness oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline leg, always as the checker or the timed CPU
baseline, never by the GPU product path.

Two back-ends with one interface:
  * ``Port``: the C restatement (oracle/hmfem_oracle.c ->
    oracle/_build/liboracle_port.so);
  * ``Ref``: the reference's own sources compiled from the hmfem tree
    (oracle/ref_harness.cpp -> oracle/_ref/libhmfem_ref.so), present only
    where that build ran.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libhmfem_ref.so")

ELE_FIELDS = ("u", "d", "l", "r", "c", "t", "b")   # structs.h:7-17
IND_FIELDS = ("c", "u", "d", "l", "r", "t", "b")   # structs.h:38-48

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_cp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the restatement (and the reference harness when the tree is
    present) with oracle/Makefile."""
    targets = ["port"] + (["ref"] if ref else [])
    tree = os.environ.get("HMFEM_REFERENCE", "/root/reference")
    subprocess.run(["make", "-s", "-C", HERE] + targets + [f"REF={tree}"], check=True)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class _Bound(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("l", "r", "u", "d", "t", "b")]


class Hierarchy:
    """Per-level arrays copied out of either back-end."""

    def __init__(self):
        self.levels = []   # dicts: n, cnt, col, ele, dinv, sel, pcnt, pcol, pele


class Port:
    """The C restatement of the reference algorithm."""

    def __init__(self):
        if not os.path.exists(PORT_SO):
            build(ref=False)
        L = C.CDLL(PORT_SO)
        self.L = L
        L.or_amg_create.restype = C.c_void_p
        L.or_amg_create.argtypes = [C.c_int, _ip, _ip, _dp, C.c_int, C.c_int,
                                    C.c_double]
        L.or_amg_destroy.argtypes = [C.c_void_p]
        L.or_amg_nlevels.argtypes = [C.c_void_p]
        L.or_level_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.or_level_copy.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8
        L.or_vcycle.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.or_pcg.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp,
                             C.c_double, C.c_int, C.c_int,
                             C.POINTER(C.c_double)]
        L.or_spmv.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
        L.or_pack_csr.restype = C.c_long
        L.or_pack_csr.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]
        L.or_assemble.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [
            _dp, _dp, _dp, _ip, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_source_term.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [
            C.POINTER(_Bound), _ip, C.c_void_p] + [C.c_void_p] * 4 + [_dp]
        L.or_fluxes.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [
            _dp, C.c_void_p, C.POINTER(_Bound), _ip, C.c_void_p,
            C.POINTER(C.c_double), C.POINTER(C.c_double)]

    # -- assembly ------------------------------------------------------
    def assemble(self, p):
        """permeabilidade_arestas + source_term -> (perm[n,7], ind[n,7], b)."""
        n = p.n
        perm = np.zeros((n, 7), dtype=np.float64)
        ind = np.full((n, 7), -1, dtype=np.int32)
        bc = np.asarray(p.bc_type, dtype=np.int32)
        self.L.or_assemble(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, p.visc, p.KX,
                           p.KY, p.KZ, bc, None, None, _ptr(perm), _ptr(ind))
        b = np.zeros(n)
        faces = p.face_arrays()
        B = _Bound(*[f.ctypes.data for f in faces])
        self.L.or_source_term(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, p.visc,
                              C.byref(B), bc, _ptr(perm), None, None, None,
                              None, b)
        return perm, ind, b

    def pack(self, perm, ind):
        n = perm.shape[0]
        nnz = self.L.or_pack_csr(n, _ptr(perm), _ptr(ind), None, None, None)
        cnt = np.zeros(n, np.int32)
        col = np.zeros(nnz, np.int32)
        ele = np.zeros(nnz)
        self.L.or_pack_csr(n, _ptr(perm), _ptr(ind), _ptr(cnt), _ptr(col),
                           _ptr(ele))
        return cnt, col, ele

    # -- AMG -----------------------------------------------------------
    def amg(self, cnt, col, ele, max_level=16, max_size=1, eps=0.0):
        h = self.L.or_amg_create(len(cnt), cnt, col, ele, max_level, max_size,
                                 eps)
        return _PortAMG(self, h)

    def spmv(self, cnt, col, ele, x):
        y = np.zeros(len(cnt))
        self.L.or_spmv(len(cnt), cnt, col, ele, np.ascontiguousarray(x), y)
        return y

    def fluxes(self, p, perm, x):
        n = p.n
        v = np.zeros((n, 7))
        faces = p.face_arrays()
        B = _Bound(*[f.ctypes.data for f in faces])
        dmin, dmax = C.c_double(), C.c_double()
        bc = np.asarray(p.bc_type, dtype=np.int32)
        self.L.or_fluxes(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz,
                         np.ascontiguousarray(x), _ptr(perm), C.byref(B), bc,
                         _ptr(v), C.byref(dmin), C.byref(dmax))
        return v, dmin.value, dmax.value


class _PortAMG:
    def __init__(self, port, h):
        self.port, self.h = port, h
        self.nlevels = port.L.or_amg_nlevels(C.c_void_p(h))

    def __del__(self):
        try:
            self.port.L.or_amg_destroy(C.c_void_p(self.h))
        except Exception:
            pass

    def level(self, l):
        L = self.port.L
        n, nnz, pnnz = C.c_int(), C.c_long(), C.c_long()
        L.or_level_info(C.c_void_p(self.h), l, C.byref(n), C.byref(nnz),
                        C.byref(pnnz))
        d = dict(n=n.value, cnt=np.zeros(n.value, np.int32),
                 col=np.zeros(nnz.value, np.int32), ele=np.zeros(nnz.value),
                 dinv=np.zeros(n.value), sel=np.zeros(n.value, np.int8),
                 pcnt=np.zeros(n.value, np.int32),
                 pcol=np.zeros(pnnz.value, np.int32),
                 pele=np.zeros(pnnz.value))
        L.or_level_copy(C.c_void_p(self.h), l, *[
            _ptr(d[k]) for k in ("cnt", "col", "ele", "dinv", "sel", "pcnt",
                                 "pcol", "pele")])
        if l == self.nlevels - 1:
            for k in ("sel", "pcnt", "pcol", "pele"):
                d[k] = d[k][:0]
        return d

    def vcycle(self, f, smoother=0, omega=1.0):
        u = np.zeros(len(f))
        self.port.L.or_vcycle(C.c_void_p(self.h), smoother, omega,
                              np.ascontiguousarray(f), u)
        return u

    def pcg(self, b, x0=None, eps=1e-10, stop=1, smoother=0, omega=1.0,
            max_it=10000):
        x = np.zeros(len(b)) if x0 is None else np.array(x0, dtype=np.float64)
        rel = C.c_double()
        it = self.port.L.or_pcg(C.c_void_p(self.h), smoother, omega,
                                np.ascontiguousarray(b), x, eps, max_it, stop,
                                C.byref(rel))
        return x, it, rel.value


class Ref:
    """The reference's own sources, compiled from the hmfem tree."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(REF_SO)
        self.L = L
        L.ref_assemble.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [
            _dp, _dp, _dp, _ip, _dp, C.c_void_p, C.c_void_p, _dp]
        L.ref_pack.restype = C.c_long
        L.ref_pack.argtypes = [C.c_int] * 3 + [C.c_void_p, C.c_void_p]
        L.ref_packed.argtypes = [_ip, _ip, _dp]
        L.ref_compute.argtypes = [C.c_int, C.c_long, _ip, _ip, _dp, _dp, _dp,
                                  C.c_double, C.c_int] + [
                                      C.POINTER(C.c_double)] * 3
        L.ref_amg_build.argtypes = [C.c_int, C.c_long, _ip, _ip, _dp]
        L.ref_amg_level.argtypes = [C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.ref_amg_copy.argtypes = [C.c_int] + [C.c_void_p] * 8
        L.ref_amg_apply.argtypes = [_dp, _dp]
        L.ref_fluxes.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [
            _ip, _dp, _dp, C.c_void_p, C.c_void_p]
        L.ref_solve_all.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [
            _dp, _dp, _dp, _ip, _dp, C.c_double, _dp, C.c_void_p, _dp,
            C.POINTER(C.c_double)]

    def assemble(self, p):
        n = p.n
        perm = np.zeros((n, 7))
        ind = np.full((n, 7), -1, dtype=np.int32)
        b = np.zeros(n)
        self.L.ref_assemble(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, p.visc, p.KX,
                            p.KY, p.KZ, np.asarray(p.bc_type, np.int32),
                            np.asarray(p.bc_value, np.float64), _ptr(perm),
                            _ptr(ind), b)
        return perm, ind, b

    def pack(self, p, perm, ind):
        nnz = self.L.ref_pack(p.nx, p.ny, p.nz, _ptr(perm), _ptr(ind))
        cnt = np.zeros(p.n, np.int32)
        col = np.zeros(nnz, np.int32)
        ele = np.zeros(nnz)
        self.L.ref_packed(cnt, col, ele)
        return cnt, col, ele

    def compute(self, cnt, col, ele, b, x0=None, eps=1e-10, stop=2):
        x = np.zeros(len(b)) if x0 is None else np.array(x0, dtype=np.float64)
        ts, tv, rr = C.c_double(), C.c_double(), C.c_double()
        it = self.L.ref_compute(len(cnt), len(col), cnt, col, ele,
                                np.ascontiguousarray(b), x, eps, stop,
                                C.byref(ts), C.byref(tv), C.byref(rr))
        return x, it, rr.value, ts.value, tv.value

    def hierarchy(self, cnt, col, ele):
        nl = self.L.ref_amg_build(len(cnt), len(col), cnt, col, ele)
        H = Hierarchy()
        for l in range(nl):
            n, nnz, pnnz = C.c_int(), C.c_long(), C.c_long()
            self.L.ref_amg_level(l, C.byref(n), C.byref(nnz), C.byref(pnnz))
            last = l == nl - 1
            d = dict(n=n.value, cnt=np.zeros(n.value, np.int32),
                     col=np.zeros(nnz.value, np.int32),
                     ele=np.zeros(nnz.value), dinv=np.zeros(n.value),
                     sel=np.zeros(0 if last else n.value, np.int8),
                     pcnt=np.zeros(0 if last else n.value, np.int32),
                     pcol=np.zeros(pnnz.value, np.int32),
                     pele=np.zeros(pnnz.value))
            self.L.ref_amg_copy(l, *[_ptr(d[k]) for k in (
                "cnt", "col", "ele", "dinv", "sel", "pcnt", "pcol", "pele")])
            H.levels.append(d)
        return H

    def vcycle(self, f):
        u = np.zeros(len(f))
        self.L.ref_amg_apply(np.ascontiguousarray(f), u)
        return u

    def fluxes(self, p, perm, x):
        v = np.zeros((p.n, 7))
        self.L.ref_fluxes(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz,
                          np.asarray(p.bc_type, np.int32),
                          np.asarray(p.bc_value, np.float64),
                          np.ascontiguousarray(x), _ptr(perm), _ptr(v))
        return v

    def solve_all(self, p, eps=1e-10):
        x = np.zeros(p.n)
        v = np.zeros((p.n, 7))
        times = np.zeros(5)
        rr = C.c_double()
        it = self.L.ref_solve_all(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, p.visc,
                                  p.KX, p.KY, p.KZ,
                                  np.asarray(p.bc_type, np.int32),
                                  np.asarray(p.bc_value, np.float64), eps, x,
                                  _ptr(v), times, C.byref(rr))
        return x, v, it, rr.value, times

    def job(self, p, eps=1e-10):
        """The path of solve_all in steps (ref_job_*): assemble() -> setup()
        -> iterate(k)... -> flux(); one job per process."""
        return RefJob(self, p, eps)


class RefJob:
    """ref_solve_all's work split into callable parts (for timing the
    reference in steps).  Keeps the problem's arrays alive."""

    def __init__(self, ref, p, eps):
        L = ref.L
        vp = C.c_void_p
        L.ref_job_new.restype = vp
        L.ref_job_new.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [
            _dp, _dp, _dp, _ip, _dp, C.c_double]
        for f in ("ref_job_assemble", "ref_job_setup"):
            getattr(L, f).argtypes = [vp]
        L.ref_job_iterate.argtypes = [vp, C.c_int]
        L.ref_job_set_eps.argtypes = [vp, C.c_double]
        L.ref_job_flux.argtypes = [vp, vp]
        L.ref_job_result.argtypes = [vp, vp, _dp, C.POINTER(C.c_double)]
        L.ref_job_free.argtypes = [vp]
        self.L, self.p = L, p
        self._bc = np.asarray(p.bc_type, np.int32)
        self._bv = np.asarray(p.bc_value, np.float64)
        self.h = L.ref_job_new(p.nx, p.ny, p.nz, p.hx, p.hy, p.hz, p.visc, p.KX, p.KY,
                               p.KZ, self._bc, self._bv, eps)

    def assemble(self):
        self.L.ref_job_assemble(self.h)

    def setup(self):
        self.L.ref_job_setup(self.h)

    def iterate(self, k=-1):
        """Up to k CG iterations (k < 0: to convergence); True once converged."""
        return bool(self.L.ref_job_iterate(self.h, k))

    def set_eps(self, eps):
        """A new tolerance; iterate() continues the same CG to it."""
        self.L.ref_job_set_eps(self.h, eps)

    def flux(self, v=None):
        self.L.ref_job_flux(self.h, None if v is None else _ptr(v))

    def result(self, want_p=True):
        x = np.zeros(self.p.n) if want_p else None
        times = np.zeros(5)
        rr = C.c_double()
        it = self.L.ref_job_result(self.h, None if x is None else _ptr(x), times,
                                   C.byref(rr))
        return x, it, rr.value, times

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_job_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the coupled conduit model (karst.c, main.c:383-557) ----------------------

class _KGrid(C.Structure):      # or_kgrid
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
                ("visc", C.c_double), ("rho", C.c_double),
                ("KX", C.c_void_p), ("KY", C.c_void_p), ("KZ", C.c_void_p),
                ("perm", C.c_void_p), ("p_old", C.c_void_p)]


class _KState(C.Structure):     # or_kstate
    _fields_ = [("mmax", C.c_int)] + [(f, C.c_void_p) for f in (
        "kl", "kr", "kc", "kic", "paux", "pc", "pc_old", "ucR", "ucL")]


def _vp(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _picard_out(k, n):
    mm = (k.mmax, k.nk)
    return dict(p=np.zeros(n), pc=np.zeros(mm), ucl=np.zeros(mm), ucr=np.zeros(mm),
                v=np.zeros((n, 7)), out=np.zeros(3), qk=np.zeros((3, k.nk)))


def karst_state_inputs(k, prob, p_old):
    """paux and KI_c of main.c:410-449 for a conduit set (matrices
    [i, j] with max(len) rows)."""
    paux = np.zeros((k.mmax, k.nk))
    kic = np.zeros((k.mmax, k.nk))
    hs = k.hs(prob.hx, prob.hy, prob.hz)
    for j, c in enumerate(k.cells(prob.nx, prob.ny)):
        paux[:len(c), j] = p_old[c]
        kic[:len(c), j] = k.kindex[j] / (k.area[j] * hs[j])
    return paux, kic


def _port_bind(L):
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.or_karst_check.argtypes = [vp, i, i, i]
    L.or_karst_keff.argtypes = [vp, vp, vp, i]
    L.or_source_term1d.argtypes = [vp, vp, vp, i, vp]
    L.or_conduit.argtypes = [vp, vp, vp, i]
    L.or_fluxo1d.argtypes = [vp, vp, vp, vp, vp]
    L.or_picard.argtypes = ([vp, i, i, i, d, d, d, d, d, vp, vp, vp, vp, vp, vp, vp,
                             d, i, d, i, i] + [vp] * 7)


def _port_karst_check(self, k, nx, ny, nz):
    _port_bind(self.L)
    ks = k.struct()
    return self.L.or_karst_check(C.addressof(ks), nx, ny, nz)


def _port_conduit_step(self, k, prob, perm, p_old, pc_old, ucR, ucL, rho=1000.0,
                       solver=0):
    """karst.c:8-40 from given state; also the source term f of each conduit
    (from the same starting fracture state)."""
    _port_bind(self.L)
    ks = k.struct()
    p_old = _f64(p_old)
    perm = np.ascontiguousarray(perm, dtype=np.float64)
    KX, KY, KZ = _f64(prob.KX), _f64(prob.KY), _f64(prob.KZ)
    G = _KGrid(prob.nx, prob.ny, prob.nz, prob.hx, prob.hy, prob.hz, prob.visc, rho,
               KX.ctypes.data, KY.ctypes.data, KZ.ctypes.data, perm.ctypes.data,
               p_old.ctypes.data)
    paux, kic = karst_state_inputs(k, prob, p_old)
    mm = (k.mmax, k.nk)
    arr = dict(kl=np.zeros(mm), kr=np.zeros(mm), kc=np.zeros(mm), kic=kic, paux=paux,
               pc=np.zeros(mm), pc_old=_f64(pc_old).copy(),
               ucR=_f64(ucR).copy().reshape(-1) if k.max_brechas else np.zeros(1),
               ucL=_f64(ucL).copy().reshape(-1) if k.max_brechas else np.zeros(1))

    def state(a):
        return _KState(k.mmax, *[a[f].ctypes.data for f in (
            "kl", "kr", "kc", "kic", "paux", "pc", "pc_old", "ucR", "ucL")])

    # source terms on a copy of the fracture state
    a2 = {f: v.copy() for f, v in arr.items()}
    S2 = state(a2)
    f = np.zeros(mm)
    for j in range(k.nk):
        fj = np.zeros(k.mmax + 1)
        self.L.or_karst_keff(C.addressof(ks), C.addressof(G), C.addressof(S2), j)
        self.L.or_source_term1d(C.addressof(ks), C.addressof(G), C.addressof(S2), j,
                                _vp(fj))
        f[:k.len[j], j] = fj[:k.len[j]]
    S = state(arr)
    self.L.or_conduit(C.addressof(ks), C.addressof(G), C.addressof(S), solver)
    out = {x: arr[x] for x in ("kl", "kr", "kc", "pc")}
    out["ucR"] = arr["ucR"][:k.max_brechas * k.nk].reshape(k.max_brechas, k.nk)
    out["ucL"] = arr["ucL"][:k.max_brechas * k.nk].reshape(k.max_brechas, k.nk)
    out["f"] = f
    return out


def _port_picard(self, k, prob, WI=None, pw=None, rho=1000.0, tol=1e-8, iter_max=1000,
                 solve_eps=1e-10, solve_stop=1, conduit_solver=0):
    """main.c:383-557 on this oracle (or_picard)."""
    _port_bind(self.L)
    ks = k.struct()
    n = prob.n
    o = _picard_out(k, n)
    KX, KY, KZ = _f64(prob.KX), _f64(prob.KY), _f64(prob.KZ)
    bct = np.asarray(prob.bc_type, np.int32)
    bcv = np.asarray(prob.bc_value, np.float64)
    WI, pw = _f64(WI), _f64(pw)
    it = self.L.or_picard(C.addressof(ks), prob.nx, prob.ny, prob.nz, prob.hx, prob.hy,
                          prob.hz, prob.visc, rho, _vp(KX), _vp(KY), _vp(KZ), _vp(bct),
                          _vp(bcv), _vp(WI), _vp(pw), tol, iter_max, solve_eps,
                          solve_stop, conduit_solver, _vp(o["p"]), _vp(o["pc"]),
                          _vp(o["ucl"]), _vp(o["ucr"]), _vp(o["v"]), _vp(o["out"]),
                          _vp(o["qk"]))
    if it < 0:
        raise ValueError("conduit set does not fit the grid")
    o["iterations"] = it
    return o


Port.karst_check = _port_karst_check
Port.conduit_step = _port_conduit_step
Port.picard = _port_picard


def _ref_bind(L):
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.ref_conduit_step.argtypes = [vp, i, i, i, d, d, d, d, d] + [vp] * 15 + [d]
    L.ref_picard.argtypes = ([vp, i, i, i, d, d, d, d, d, vp, vp, vp, vp, vp, vp, vp,
                              d, i, d] + [vp] * 8)


def _ref_conduit_step(self, k, prob, perm, p_old, pc_old, ucR, ucL, rho=1000.0, eps=1e-8):
    """The reference's conduit() (and source_term1d alone for f) on given
    state; 1-D solves through compute() at eps with the pcg.h rule."""
    _ref_bind(self.L)
    ks = k.struct()
    p_old = _f64(p_old)
    perm = np.ascontiguousarray(perm, dtype=np.float64)
    paux, kic = karst_state_inputs(k, prob, p_old)
    mm = (k.mmax, k.nk)
    kl, kr, kc, f, pc = (np.zeros(mm) for _ in range(5))
    uR = _f64(ucR).copy().reshape(-1) if k.max_brechas else np.zeros(1)
    uL = _f64(ucL).copy().reshape(-1) if k.max_brechas else np.zeros(1)
    KX, KY, KZ = _f64(prob.KX), _f64(prob.KY), _f64(prob.KZ)
    pco = _f64(pc_old)
    self.L.ref_conduit_step(C.addressof(ks), prob.nx, prob.ny, prob.nz, prob.hx, prob.hy,
                            prob.hz, prob.visc, rho, _vp(KX), _vp(KY), _vp(KZ), _vp(perm),
                            _vp(p_old), _vp(paux), _vp(kic), _vp(pco), _vp(uR), _vp(uL),
                            _vp(kl), _vp(kr), _vp(kc), _vp(f), _vp(pc), eps)
    mb = k.max_brechas
    return dict(kl=kl, kr=kr, kc=kc, f=f, pc=pc,
                ucR=uR[:mb * k.nk].reshape(mb, k.nk), ucL=uL[:mb * k.nk].reshape(mb, k.nk))


def _ref_picard(self, k, prob, WI=None, pw=None, rho=1000.0, tol=1e-8, iter_max=1000,
                eps=1e-8):
    """The reference's coupled run (its reservoir(), conduit(), fluxo1d(),
    fluxos()) with every solve through compute() at eps (pcg.h rule)."""
    _ref_bind(self.L)
    ks = k.struct()
    n = prob.n
    o = _picard_out(k, n)
    times = np.zeros(2)
    KX, KY, KZ = _f64(prob.KX), _f64(prob.KY), _f64(prob.KZ)
    bct = np.asarray(prob.bc_type, np.int32)
    bcv = np.asarray(prob.bc_value, np.float64)
    WI, pw = _f64(WI), _f64(pw)
    it = self.L.ref_picard(C.addressof(ks), prob.nx, prob.ny, prob.nz, prob.hx, prob.hy,
                           prob.hz, prob.visc, rho, _vp(KX), _vp(KY), _vp(KZ), _vp(bct),
                           _vp(bcv), _vp(WI), _vp(pw), tol, iter_max, eps, _vp(o["p"]),
                           _vp(o["pc"]), _vp(o["ucl"]), _vp(o["ucr"]), _vp(o["v"]),
                           _vp(o["out"]), _vp(o["qk"]), _vp(times))
    o["iterations"] = it
    o["seconds"] = float(times[0])
    o["computes"] = int(times[1])
    return o


Ref.conduit_step = _ref_conduit_step
Ref.picard = _ref_picard
