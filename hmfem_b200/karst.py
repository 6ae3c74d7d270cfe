"""The coupled reservoir / karst-conduit model on the GPU.

The reference application couples the 3-D Darcy reservoir with 1-D conduits
by a Picard loop (main.c:383-489): reservoir solve with the conduit
pressures in the exchange term, then one tridiagonal system per conduit with
the new reservoir pressure, until the reservoir pressure stops changing.
`picard` runs that loop through the library's `hmfem_picard` (include/
hmfem_karst.h): one AMG setup for the coupled matrix, the exchange
right-hand side patched in place, warm-started 3-D solves and one batched
Thomas launch for all conduits per iteration.

`Karst` holds a conduit set in the layout of the reference's data file
data_<nk>_<type>.dat (main.c:197-280); `Karst.read` parses such a file.
Per-element matrices use the reference's pc[i][j] layout, flattened
row-major as [i * nk + j] with max(len) rows.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import gpu


class KarstStruct(C.Structure):
    """hmfem_karst (include/hmfem_karst.h); the oracle's or_karst has the
    same layout."""
    _fields_ = [("nk", C.c_int), ("max_brechas", C.c_int),
                ("len", C.c_void_p), ("sxi", C.c_void_p), ("syi", C.c_void_p),
                ("szi", C.c_void_p), ("pos", C.c_void_p), ("Kc", C.c_void_p),
                ("bound_l", C.c_void_p), ("bound_r", C.c_void_p),
                ("cont", C.c_void_p), ("ccont", C.c_void_p),
                ("kindex", C.c_void_p), ("area", C.c_void_p),
                ("n_brechas", C.c_void_p), ("beta", C.c_void_p),
                ("cb", C.c_void_p), ("brechas", C.c_void_p)]


DIRICHLET, NEUMANN, ROBIN = 0, 1, 3   # BoundKarst codes (permeabilities.c:826-858)


@dataclass
class Karst:
    len: np.ndarray        # M[j].s
    sxi: np.ndarray        # start cell of conduit j
    syi: np.ndarray
    szi: np.ndarray
    pos: np.ndarray        # 1 along x, 2 along y, 3 along z
    Kc: np.ndarray         # conduit permeability
    bound_l: np.ndarray    # end conditions (DIRICHLET / NEUMANN / ROBIN)
    bound_r: np.ndarray
    cont: np.ndarray       # (2, nk) cont_karst: end values
    ccont: np.ndarray      # (2, nk) C_contorno: Robin end coefficients
    kindex: np.ndarray     # karst index (exchange coefficient)
    area: np.ndarray       # Ac: cross-section
    n_brechas: np.ndarray  # fractures per conduit
    beta: np.ndarray       # (max_brechas, nk) R^4 - 1
    cb: np.ndarray         # (max_brechas, nk) fracture C
    brechas: np.ndarray    # (max_brechas, nk) element of each fracture

    def __post_init__(self):
        ints = ("len", "sxi", "syi", "szi", "pos", "bound_l", "bound_r", "n_brechas")
        for f in ints:
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.int32).reshape(-1))
        for f in ("Kc", "kindex", "area"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64).reshape(-1))
        nk = self.nk
        self.cont = np.ascontiguousarray(self.cont, dtype=np.float64).reshape(2, nk)
        self.ccont = np.ascontiguousarray(self.ccont, dtype=np.float64).reshape(2, nk)
        mb = int(self.n_brechas.max()) if nk else 0
        mb = max(mb, np.asarray(self.beta).reshape(-1, nk).shape[0] if np.size(self.beta) else 0)
        self.beta = np.ascontiguousarray(self.beta, dtype=np.float64).reshape(mb, nk)
        self.cb = np.ascontiguousarray(self.cb, dtype=np.float64).reshape(mb, nk)
        self.brechas = np.ascontiguousarray(self.brechas, dtype=np.int32).reshape(mb, nk)

    @property
    def nk(self) -> int:
        return int(self.len.shape[0])

    @property
    def max_brechas(self) -> int:
        return int(self.beta.shape[0])

    @property
    def mmax(self) -> int:
        return int(self.len.max()) if self.nk else 0

    def cells(self, nx, ny):
        """Reservoir cell of every element, per conduit (main.c:416-448)."""
        out = []
        for j in range(self.nk):
            i = np.arange(self.len[j])
            x = self.sxi[j] + (i if self.pos[j] == 1 else 0)
            y = self.syi[j] + (i if self.pos[j] == 2 else 0)
            z = self.szi[j] + (i if self.pos[j] == 3 else 0)
            out.append(x + nx * (y + ny * z))
        return out

    def hs(self, hx, hy, hz):
        return np.where(self.pos == 1, hx, np.where(self.pos == 2, hy, hz))

    def struct(self) -> KarstStruct:
        """ctypes view; the arrays stay owned by this object."""
        p = lambda a: a.ctypes.data  # noqa: E731
        return KarstStruct(self.nk, self.max_brechas, p(self.len), p(self.sxi),
                           p(self.syi), p(self.szi), p(self.pos), p(self.Kc),
                           p(self.bound_l), p(self.bound_r), p(self.cont),
                           p(self.ccont), p(self.kindex), p(self.area),
                           p(self.n_brechas), p(self.beta), p(self.cb),
                           p(self.brechas))

    @classmethod
    def read(cls, path, number_karst):
        """main.c:197-280: the data file's whitespace-separated fields in
        order; beta is stored as R^4 - 1 (main.c:256)."""
        tok = open(path).read().split()
        pos = [0]
        nk = number_karst

        def take(k, conv):
            if pos[0] + k > len(tok):
                raise ValueError(f"{path}: short conduit data file")
            out = [conv(t) for t in tok[pos[0]:pos[0] + k]]
            pos[0] += k
            return out

        def ints(k):
            return take(k, lambda t: int(t, 0))

        def dbls(k):
            return take(k, float)

        ln, sx, sy, sz, ps = [ints(nk) for _ in range(5)]
        Kc = dbls(nk)
        bl, br = ints(nk), ints(nk)
        cont = dbls(2 * nk)
        ccont = dbls(2 * nk)
        kidx, area = dbls(nk), dbls(nk)
        nb = ints(nk)
        mb = max(max([-1] + nb), 0)   # main.c:245-250
        beta = [v - 1.0 for v in dbls(mb * nk)]
        cb = dbls(mb * nk)
        br_ = ints(mb * nk)
        return cls(ln, sx, sy, sz, ps, Kc, bl, br, cont, ccont, kidx, area, nb,
                   np.reshape(beta, (mb, nk)), np.reshape(cb, (mb, nk)),
                   np.reshape(br_, (mb, nk)))


# ---- the library entry points -------------------------------------------------

class PicardOptions(C.Structure):
    _fields_ = [("rho", C.c_double), ("tol", C.c_double), ("iter_max", C.c_int)]


class PicardStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("error", C.c_double),
                ("cg_iterations", C.c_int), ("setups", C.c_int),
                ("q_well", C.c_double), ("p_mean", C.c_double),
                ("t_setup_ms", C.c_double), ("t_loop_ms", C.c_double),
                ("t_total_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def _lib():
    L = gpu.lib()
    if not getattr(L, "_karst_bound", False):
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.hmfem_karst_check.argtypes = [C.POINTER(KarstStruct), i, i, i]
        L.hmfem_picard_default_options.argtypes = [C.POINTER(PicardOptions)]
        L.hmfem_picard.argtypes = ([vp, C.POINTER(KarstStruct), i, i, i, d, d, d, d,
                                    vp, vp, vp, vp, vp, vp, vp,
                                    C.POINTER(PicardOptions), vp, vp, i,
                                    C.POINTER(PicardStats)])
        L.hmfem_picard_fluxes.argtypes = [vp, vp, vp, vp, i]
        L.hmfem_conduit_step.argtypes = ([C.POINTER(KarstStruct), i, i, i, d, d, d, d, d]
                                         + [vp] * 11 + [i])
        L._karst_bound = True
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def check(k: Karst, nx, ny, nz):
    """Raises gpu.HmfemError when the conduit set cannot run on the grid."""
    rc = _lib().hmfem_karst_check(C.byref(k.struct()), nx, ny, nz)
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())


def default_options():
    o = PicardOptions()
    _lib().hmfem_picard_default_options(C.byref(o))
    return o


def picard(solver, k: Karst, prob, WI=None, pw=None, rho=1000.0, tol=1e-8,
           iter_max=1000, fluxes=True):
    """The coupled run on `solver` (a gpu.Solver) for grid problem `prob`
    (hmfem_b200.problem.Problem, host K).  Returns a dict with p, pc (mmax x
    nk), the stats and, with fluxes, ucl / ucr (mmax x nk), qk (3 x nk) and
    the reservoir face fluxes v (n x 7, ELE order)."""
    L = _lib()
    ks = k.struct()
    o = PicardOptions(rho, tol, iter_max)
    st = PicardStats()
    n = prob.n
    p = np.zeros(n)
    pc = np.zeros((k.mmax, k.nk))
    KX = np.ascontiguousarray(prob.KX, dtype=np.float64)
    KY = np.ascontiguousarray(prob.KY, dtype=np.float64)
    KZ = np.ascontiguousarray(prob.KZ, dtype=np.float64)
    bct = np.asarray(prob.bc_type, dtype=np.int32)
    bcv = np.asarray(prob.bc_value, dtype=np.float64)
    WI = None if WI is None else np.ascontiguousarray(WI, dtype=np.float64)
    pw = None if pw is None else np.ascontiguousarray(pw, dtype=np.float64)
    rc = L.hmfem_picard(solver.h, C.byref(ks), prob.nx, prob.ny, prob.nz, prob.hx,
                        prob.hy, prob.hz, prob.visc, _p(KX), _p(KY), _p(KZ),
                        _p(bct), _p(bcv), _p(WI), _p(pw), C.byref(o), _p(p), _p(pc),
                        0, C.byref(st))
    if rc not in (0, gpu.E_NOTCONV):
        raise gpu.HmfemError(rc, gpu.last_error())
    out = dict(p=p, pc=pc, stats=st.as_dict())
    if fluxes:
        ucl = np.zeros((k.mmax, k.nk))
        ucr = np.zeros((k.mmax, k.nk))
        qk = np.zeros((3, k.nk))
        rc2 = L.hmfem_picard_fluxes(solver.h, _p(ucl), _p(ucr), _p(qk), 0)
        if rc2 != 0:
            raise gpu.HmfemError(rc2, gpu.last_error())
        out.update(ucl=ucl, ucr=ucr, qk=qk, v=solver.fluxes(p, np.zeros((n, 7)))[0])
    return out


def conduit_step(k: Karst, prob, p_old, pc_old, ucR, ucL, rho=1000.0):
    """One conduit() call (karst.c:8-40) on the GPU from given state; returns
    pc, kl, kr, kc (mmax x nk) and the updated ucR, ucL (max_brechas x nk)."""
    L = _lib()
    ks = k.struct()
    mm = (k.mmax, k.nk)
    pc = np.zeros(mm)
    kl, kr, kc = np.zeros(mm), np.zeros(mm), np.zeros(mm)
    uR = np.ascontiguousarray(ucR, dtype=np.float64).copy()
    uL = np.ascontiguousarray(ucL, dtype=np.float64).copy()
    KX = np.ascontiguousarray(prob.KX, dtype=np.float64)
    KY = np.ascontiguousarray(prob.KY, dtype=np.float64)
    KZ = np.ascontiguousarray(prob.KZ, dtype=np.float64)
    po = np.ascontiguousarray(p_old, dtype=np.float64)
    pco = np.ascontiguousarray(pc_old, dtype=np.float64)
    rc = L.hmfem_conduit_step(C.byref(ks), prob.nx, prob.ny, prob.nz, prob.hx,
                              prob.hy, prob.hz, prob.visc, rho, _p(KX), _p(KY),
                              _p(KZ), _p(po), _p(pco), _p(uR), _p(uL), _p(pc),
                              _p(kl), _p(kr), _p(kc), 0)
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())
    return dict(pc=pc, kl=kl, kr=kr, kc=kc, ucR=uR, ucL=uL)
