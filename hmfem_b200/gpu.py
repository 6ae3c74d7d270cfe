"""Python front-end of libhmfem_gpu.so (ctypes over the C-ABI in
include/hmfem_gpu.h).

Mirrors the reference's bridge -- ``compute`` (compute.cpp:7-51) and
``solve_linsys`` (solve_linearsystem_AMG.c:37-157) with the same argument
meaning -- plus the status-returning ``Solver`` object.  Arrays may be numpy
(host memory) or CUDA torch tensors (device memory, used in place).

There is no CPU fallback: if the library cannot be loaded (or built in-tree
with nvcc) every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

OK, E_NOTCONV, E_BREAKDOWN, E_CUDA, E_ARG, E_TIMEOUT, E_CAPACITY = range(7)
STATUS = {0: "ok", 1: "not converged", 2: "breakdown", 3: "cuda error",
          4: "bad argument", 5: "device wait timed out", 6: "capacity"}


class HmfemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hmfem status {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class Ele(C.Structure):  # structs.h:7-17
    _fields_ = [(f, C.c_double) for f in ("u", "d", "l", "r", "c", "t", "b")]


class Ind(C.Structure):  # structs.h:38-48
    _fields_ = [(f, C.c_int) for f in ("c", "u", "d", "l", "r", "t", "b")]


class Dim(C.Structure):  # structs.h:84-95
    _fields_ = [(f, C.c_int) for f in ("x", "y", "z", "xy", "t", "px", "pz", "py")]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("bf16_from", C.c_int),
                ("smoother", C.c_int), ("gs_from", C.c_int),
                ("omega", C.c_double),
                ("tol", C.c_double), ("stop_rule", C.c_int),
                ("max_iter", C.c_int), ("max_levels", C.c_int),
                ("min_coarse", C.c_int), ("coarse_direct", C.c_int),
                ("check_every", C.c_int), ("generic_setup", C.c_int),
                ("gs_fused", C.c_int), ("cheb_from", C.c_int),
                ("cheb_degree", C.c_int), ("reuse_setup", C.c_int),
                ("schur0", C.c_int), ("verbose", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("levels", C.c_int),
                ("status", C.c_int), ("relres", C.c_double),
                ("t_assemble_ms", C.c_double), ("t_setup_ms", C.c_double),
                ("t_solve_ms", C.c_double), ("t_flux_ms", C.c_double),
                ("divmin", C.c_double), ("divmax", C.c_double),
                ("setup_reused", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

EXPORTS = [
    "compute", "solve_linsys", "iter_amg",
    "_device_add_scale", "_device_sub_scale", "_device_scale_add",
    "_device_vector_product", "_device_linear_operator", "_device_jacobi",
    "_device_set_mul", "_device_add_mul", "_device_diagonal_solver",
    "_device_com_snd", "_device_com_rcv", "_device_sub", "_device_add",
    "_device_rsb", "_device_matrix_conversion",
    "hmfem_default_options", "hmfem_create", "hmfem_destroy",
    "hmfem_set_stream", "hmfem_get_stream", "hmfem_last_error",
    "hmfem_assemble", "hmfem_set_matrix", "hmfem_set_stencil", "hmfem_setup",
    "hmfem_solve", "hmfem_fluxes", "hmfem_num_levels", "hmfem_level_info",
    "hmfem_level_copy", "hmfem_vcycle", "hmfem_spmv", "hmfem_rhs",
    "hmfem_last_stats", "hmfem_time_kernel", "hmfem_fluxes_noalloc",
    "hmfem_launch_count", "hmfem_profile_iteration", "hmfem_batch_solve",
]


class KernelTime(C.Structure):
    """hmfem_kernel_time"""
    _fields_ = [("name", C.c_char * 96), ("level", C.c_int), ("launches", C.c_int),
                ("ms", C.c_double)]

NOALLOC_MAX_FACE = 262144  # HMFEM_NOALLOC_MAX_FACE in include/hmfem_gpu.h


def lib():
    """Load the in-tree library, building it with nvcc if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            _build.build()
        L = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        L.hmfem_last_error.restype = C.c_char_p
        L.hmfem_default_options.argtypes = [C.POINTER(Options)]
        L.hmfem_create.argtypes = [C.POINTER(vp), C.POINTER(Options)]
        L.hmfem_destroy.argtypes = [vp]
        L.hmfem_set_stream.argtypes = [vp, vp]
        L.hmfem_get_stream.argtypes = [vp]
        L.hmfem_get_stream.restype = vp
        L.hmfem_assemble.argtypes = [vp, ip, ip, ip, dp, dp, dp, dp, vp, vp, vp,
                                     vp, vp, vp, ip]
        L.hmfem_set_matrix.argtypes = [vp, ip, C.c_long, vp, vp, vp, vp, ip]
        L.hmfem_set_stencil.argtypes = [vp, ip, ip, ip, vp, vp, vp, ip]
        L.hmfem_setup.argtypes = [vp]
        L.hmfem_solve.argtypes = [vp, vp, vp, ip, C.POINTER(Stats)]
        L.hmfem_fluxes.argtypes = [vp, vp, vp, ip, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]
        L.hmfem_num_levels.argtypes = [vp]
        L.hmfem_level_info.argtypes = [vp, ip, C.POINTER(ip), C.POINTER(C.c_long),
                                       C.POINTER(C.c_long)]
        L.hmfem_level_copy.argtypes = [vp, ip] + [vp] * 7
        L.hmfem_vcycle.argtypes = [vp, vp, vp, ip]
        L.hmfem_spmv.argtypes = [vp, ip, vp, vp, ip]
        L.hmfem_rhs.argtypes = [vp, vp, ip]
        L.hmfem_last_stats.argtypes = [vp, C.POINTER(Stats)]
        L.hmfem_time_kernel.argtypes = [vp, ip, ip, ip, C.POINTER(C.c_float),
                                        C.POINTER(C.c_double)]
        L.hmfem_fluxes_noalloc.argtypes = [ip, ip, ip, dp, dp, dp, dp, vp, vp,
                                           vp, vp, vp, vp, vp,
                                           C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), vp]
        L.hmfem_launch_count.restype = C.c_ulonglong
        L.hmfem_profile_iteration.argtypes = [vp, ip, C.POINTER(KernelTime), ip,
                                              C.POINTER(ip)]
        L.hmfem_batch_solve.argtypes = [C.POINTER(vp), ip, C.POINTER(vp), ip,
                                        C.POINTER(Stats)]
        L.compute.argtypes = [vp] * 6
        L.solve_linsys.argtypes = [vp, vp, vp, vp, Dim]
        L.solve_linsys.restype = None
        _lib = L
    return _lib


def missing_exports():
    L = lib()
    return [s for s in EXPORTS if not hasattr(L, s)]


def last_error() -> str:
    return lib().hmfem_last_error().decode(errors="replace")


def _check(rc, allow=(OK,)):
    if rc not in allow:
        raise HmfemError(rc, last_error())
    return rc


def _ptr(a):
    """(pointer, mem) for a numpy array (host) or a CUDA tensor (device)."""
    if a is None:
        return None, 0
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data, 0
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr(), 1 if a.is_cuda else 0
    raise TypeError(f"unsupported array type {type(a)}")


def default_options(**kw) -> Options:
    o = Options()
    lib().hmfem_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Solver:
    """One pressure-solve pipeline on the current CUDA device."""

    def __init__(self, **options):
        self.L = lib()
        self.opt = default_options(**options)
        h = C.c_void_p()
        _check(self.L.hmfem_create(C.byref(h), C.byref(self.opt)))
        self.h = h
        self.n = 0
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.L.hmfem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _after_torch(self, *arrays):
        """Orders the solver's stream after torch's current stream when a
        CUDA tensor is passed (the solver works on its own non-blocking
        stream; a tensor just written on torch's stream must be complete
        before the solver reads it).  An event wait, no host synchronisation."""
        if not any(getattr(a, "is_cuda", False) for a in arrays):
            return
        import torch
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream())
        torch.cuda.ExternalStream(self.stream).wait_event(ev)

    def set_stream(self, stream_handle):
        _check(self.L.hmfem_set_stream(self.h, C.c_void_p(stream_handle)))

    @property
    def stream(self):
        return self.L.hmfem_get_stream(self.h)

    # -- problem ---------------------------------------------------------
    def assemble(self, prob, KX=None, KY=None, KZ=None, face_vals=None):
        """TPFA assembly of a problem.Problem on the device; K arrays default
        to the problem's (host) arrays, or pass CUDA tensors."""
        KX = prob.KX if KX is None else KX
        KY = prob.KY if KY is None else KY
        KZ = prob.KZ if KZ is None else KZ
        px, mem = _ptr(KX)
        py, _ = _ptr(KY)
        pz, _ = _ptr(KZ)
        bc = (C.c_int * 6)(*prob.bc_type)
        bv = (C.c_double * 6)(*prob.bc_value)
        fv = None
        if face_vals is not None:
            arr = (C.c_void_p * 6)(*[_ptr(f)[0] for f in face_vals])
            fv = arr
        self._keep = [KX, KY, KZ, face_vals]
        self._after_torch(KX, KY, KZ, *(face_vals or ()))
        _check(self.L.hmfem_assemble(self.h, prob.nx, prob.ny, prob.nz, prob.hx,
                                     prob.hy, prob.hz, prob.visc, px, py, pz,
                                     bc, bv, fv, mem))
        self.n = prob.n

    def set_matrix(self, cnt, col, ele, b=None):
        self._after_torch(cnt, col, ele, b)
        pc, mem = _ptr(cnt)
        _check(self.L.hmfem_set_matrix(self.h, len(cnt), len(col), pc,
                                       _ptr(col)[0], _ptr(ele)[0], _ptr(b)[0],
                                       mem))
        self.n = len(cnt)

    def set_stencil(self, nx, ny, nz, perm, indcol, b=None):
        self._after_torch(perm, indcol, b)
        pp, mem = _ptr(perm)
        _check(self.L.hmfem_set_stencil(self.h, nx, ny, nz, pp, _ptr(indcol)[0],
                                        _ptr(b)[0], mem))
        self.n = nx * ny * nz

    def setup(self):
        _check(self.L.hmfem_setup(self.h))

    def solve(self, b=None, x=None, allow_notconv=False):
        """Solves in place into x (initial guess in); returns Stats dict."""
        if x is None:
            x = np.zeros(self.n)
        self._after_torch(b, x)
        pb, _ = _ptr(b)
        px, mem = _ptr(x)
        st = Stats()
        rc = self.L.hmfem_solve(self.h, pb, px, mem, C.byref(st))
        _check(rc, (OK, E_NOTCONV) if allow_notconv else (OK,))
        return x, st.as_dict()

    def fluxes(self, p, v=None):
        if v is None:
            v = np.zeros((self.n, 7))
        self._after_torch(p, v)
        pp, mem = _ptr(p)
        dmin, dmax = C.c_double(), C.c_double()
        _check(self.L.hmfem_fluxes(self.h, pp, _ptr(v)[0], mem, C.byref(dmin),
                                   C.byref(dmax)))
        return v, dmin.value, dmax.value

    def stats(self):
        st = Stats()
        _check(self.L.hmfem_last_stats(self.h, C.byref(st)))
        return st.as_dict()

    def profile_iteration(self, iters=3):
        """Per (kernel, level) launches and summed milliseconds of `iters`
        CG iterations launched one kernel at a time (hmfem_profile_iteration;
        level -1 = the CG's level-0 vector work)."""
        cap = 512
        buf = (KernelTime * cap)()
        cnt = C.c_int()
        _check(self.L.hmfem_profile_iteration(self.h, iters, buf, cap, C.byref(cnt)))
        return [dict(kernel=buf[i].name.decode(), level=buf[i].level,
                     launches=buf[i].launches, ms=buf[i].ms)
                for i in range(min(cnt.value, cap))]

    # -- inspection ------------------------------------------------------
    def num_levels(self):
        return self.L.hmfem_num_levels(self.h)

    def level_info(self, l):
        """(rows, nonzeros, P nonzeros) of level l, without copying it."""
        n, nnz, pnnz = C.c_int(), C.c_long(), C.c_long()
        _check(self.L.hmfem_level_info(self.h, l, C.byref(n), C.byref(nnz),
                                       C.byref(pnnz)))
        return n.value, nnz.value, pnnz.value

    def level(self, l):
        n, nnz, pnnz = C.c_int(), C.c_long(), C.c_long()
        _check(self.L.hmfem_level_info(self.h, l, C.byref(n), C.byref(nnz),
                                       C.byref(pnnz)))
        last = l == self.num_levels() - 1
        d = dict(n=n.value, cnt=np.zeros(n.value, np.int32),
                 col=np.zeros(nnz.value, np.int32), ele=np.zeros(nnz.value),
                 dinv=np.zeros(n.value),
                 sel=np.zeros(0 if last else n.value, np.int8),
                 pcnt=np.zeros(0 if last else n.value, np.int32),
                 pcol=np.zeros(pnnz.value, np.int32))
        _check(self.L.hmfem_level_copy(self.h, l, *[
            d[k].ctypes.data for k in ("cnt", "col", "ele", "dinv", "sel",
                                       "pcnt", "pcol")]))
        return d

    def vcycle(self, f):
        u = np.zeros(len(f)) if isinstance(f, np.ndarray) else f.clone()
        self._after_torch(f, u)
        pf, mem = _ptr(f)
        _check(self.L.hmfem_vcycle(self.h, pf, _ptr(u)[0], mem))
        return u

    def spmv(self, level, x):
        y = np.zeros(len(x)) if isinstance(x, np.ndarray) else x.clone()
        self._after_torch(x, y)
        px, mem = _ptr(x)
        _check(self.L.hmfem_spmv(self.h, level, px, _ptr(y)[0], mem))
        return y

    def time_kernel(self, which, level, reps=20):
        """(mean ms, algorithmic bytes) of one solve-phase kernel."""
        ms, by = C.c_float(), C.c_double()
        _check(self.L.hmfem_time_kernel(self.h, which, level, reps, C.byref(ms),
                                        C.byref(by)))
        return ms.value, by.value

    def rhs(self):
        b = np.zeros(self.n)
        _check(self.L.hmfem_rhs(self.h, b.ctypes.data, 0))
        return b


# ---- the reference bridge ---------------------------------------------------

def compute(hdr, cnt, col, ele, b, x):
    """compute.cpp:7-51 -- same arrays and meaning (x in/out); returns 0."""
    L = lib()
    for a, dt in ((hdr, np.int32), (cnt, np.int32), (col, np.int32),
                  (ele, np.float64), (b, np.float64), (x, np.float64)):
        if a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
            raise TypeError("compute expects contiguous int32/float64 arrays")
    return L.compute(hdr.ctypes.data, cnt.ctypes.data, col.ctypes.data,
                     ele.ctypes.data, b.ctypes.data, x.ctypes.data)


def solve_linsys(perm, indcol, b, x, nx, ny, nz):
    """solve_linearsystem_AMG.c:37-157 -- perm (n,7) float64 in ELE field
    order u,d,l,r,c,t,b; indcol (n,7) int32 in IND order c,u,d,l,r,t,b."""
    L = lib()
    N = Dim(nx, ny, nz, nx * ny, nx * ny * nz, 0, 0, 0)
    L.solve_linsys(perm.ctypes.data, indcol.ctypes.data, b.ctypes.data,
                   x.ctypes.data, N)


def launch_count() -> int:
    """Kernels of this library launched so far (graph replays included)."""
    return int(lib().hmfem_launch_count())


def iter_amg() -> int:
    return C.c_int.in_dll(lib(), "iter_amg").value


def batch_solve(solvers, xs=None, allow_notconv=False):
    """hmfem_batch_solve: set-up solvers solved together (one CUDA graph with
    a branch per solver, replayed until all converged).  xs: per solver the
    initial guess in / solution out (numpy arrays, or CUDA tensors), or None
    (zero guesses, nothing returned).  Returns the stats dicts."""
    L = lib()
    m = len(solvers)
    hs = (C.c_void_p * m)(*[s.h for s in solvers])
    xp, mem = None, 0
    if xs is not None:
        ptrs = []
        for s, x in zip(solvers, xs):
            s._after_torch(x)
            pa, mem = _ptr(x)
            ptrs.append(pa)
        xp = (C.c_void_p * m)(*ptrs)
    st = (Stats * m)()
    rc = L.hmfem_batch_solve(hs, m, xp, mem, st)
    _check(rc, (OK, E_NOTCONV) if allow_notconv else (OK,))
    return [st[i].as_dict() for i in range(m)]


def fluxes_noalloc(prob, KX, KY, KZ, p, v, stream=None):
    """hmfem_fluxes_noalloc: fluxes of device pressure p into device v
    (n x 7 float64, c untouched) with no device allocation by the library;
    returns (divmin, divmax).  For callers that cannot let the library
    allocate (see include/hmfem_gpu.h)."""
    import torch
    L = lib()
    bc = (C.c_int * 6)(*prob.bc_type)
    bv = (C.c_double * 6)(*prob.bc_value)
    dmin, dmax = C.c_double(), C.c_double()
    dev = torch.cuda.current_device()
    ptrs = []
    for name, a, numel in (("KX", KX, prob.n), ("KY", KY, prob.n), ("KZ", KZ, prob.n),
                           ("p", p, prob.n), ("v", v, 7 * prob.n)):
        if not (hasattr(a, "is_cuda") and a.is_cuda):
            raise ValueError(f"fluxes_noalloc: {name} must be a CUDA tensor")
        if a.dtype != torch.float64:
            raise ValueError(f"fluxes_noalloc: {name} must be float64, not {a.dtype}")
        if a.numel() != numel:
            raise ValueError(f"fluxes_noalloc: {name} has {a.numel()} elements, "
                             f"the grid needs {numel}")
        if a.device.index != dev:
            raise ValueError(f"fluxes_noalloc: {name} is on cuda:{a.device.index}, "
                             f"the current device is cuda:{dev}")
        pa, _ = _ptr(a)
        ptrs.append(pa)
    _check(L.hmfem_fluxes_noalloc(prob.nx, prob.ny, prob.nz, prob.hx, prob.hy,
                                  prob.hz, prob.visc, ptrs[0], ptrs[1], ptrs[2],
                                  bc, bv, ptrs[3], ptrs[4], C.byref(dmin),
                                  C.byref(dmax), C.c_void_p(stream)))
    return dmin.value, dmax.value
