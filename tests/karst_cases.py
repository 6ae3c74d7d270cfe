"""Seeded coupled reservoir / conduit problems shared by the conduit-model
tests and their golden-fixture generator (tests/golden/make_golden_karst.py).

Units and constants follow the reference application (main.c:118-152):
viscosity 1e-3, density 1000, Dirichlet 60 MPa on the four lateral faces and
no flow through top and bottom, a well column at 10 MPa, conduits at
Kc = 1e-11 with karst index 1.0169e-12 and section 3.1415.
"""
import numpy as np

from hmfem_b200.karst import Karst
from hmfem_b200.problem import Problem

VISC, RHO = 1e-3, 1000.0
BC_TYPE = (0, 0, 0, 0, 1, 1)                   # l, r, u, d Dirichlet; t, b no flow
BC_VALUE = (60e6, 60e6, 60e6, 60e6, 0.0, 0.0)  # main.c:140-145
WELL_INDEX, WELL_P = 7.64352339e-13, 10e6      # main.c:128-129


def reservoir(nx, ny, nz, hx, hy, hz, seed=None, kbg=1e-13):
    """Homogeneous K (seed None, perm_homogeneous) or a seeded lognormal
    field around kbg."""
    n = nx * ny * nz
    if seed is None:
        K = np.full(n, kbg)
    else:
        g = np.random.default_rng(seed).standard_normal(n)
        K = kbg * 10.0 ** (0.5 * g)
    return Problem(nx, ny, nz, hx, hy, hz, K, K, K, bc_type=BC_TYPE,
                   bc_value=BC_VALUE, visc=VISC)


def well(prob, px, py, pz):
    """WI / pw of main.c:458-462 / 302-306: the column (px, py, z >= pz)."""
    WI = np.zeros(prob.n)
    pw = np.zeros(prob.n)
    for z in range(pz, prob.nz):
        c = px + prob.nx * (py + prob.ny * z)
        WI[c] = WELL_INDEX
        pw[c] = WELL_P
    return WI, pw


def _karst(rows, max_b):
    """rows: dicts with len, start (x, y, z), pos, bl, br, cont (l, r),
    ccont (l, r), fractures [(element, R^4, C)]."""
    nk = len(rows)
    beta = np.zeros((max_b, nk))
    cb = np.zeros((max_b, nk))
    br = np.zeros((max_b, nk), np.int32)
    for j, r in enumerate(rows):
        for b, (el, r4, c) in enumerate(r.get("fractures", [])):
            beta[b, j] = r4 - 1.0
            cb[b, j] = c
            br[b, j] = el
    return Karst([r["len"] for r in rows], [r["start"][0] for r in rows],
                 [r["start"][1] for r in rows], [r["start"][2] for r in rows],
                 [r["pos"] for r in rows], [r.get("Kc", 1e-11) for r in rows],
                 [r["bl"] for r in rows], [r["br"] for r in rows],
                 np.array([r["cont"] for r in rows]).T.copy(),
                 np.array([r.get("ccont", (1.0, 1.0)) for r in rows]).T.copy(),
                 [r.get("kindex", 1.01686094e-12) for r in rows],
                 [r.get("area", 3.1415) for r in rows],
                 [len(r.get("fractures", [])) for r in rows], beta, cb, br)


def case_single():
    """The reference run's layout scaled down: one x conduit with nonlinear
    Robin ends and two fractures, a well column beside it."""
    prob = reservoir(40, 10, 8, 1.0, 5.0, 5.0)
    k = _karst([dict(len=30, start=(5, 5, 3), pos=1, bl=3, br=3, cont=(1.0, 1.0),
                     fractures=[(8, 1e8, 1.0), (20, 1e8, 1.0)])], 2)
    WI, pw = well(prob, 20, 5, 4)
    return prob, k, WI, pw


def case_multi():
    """Four conduits on a heterogeneous field: along x, y and z; Dirichlet,
    Neumann and nonlinear Robin ends with active Robin terms (cont != 1);
    fractures; the last conduit overlaps the first one's cells (the later
    conduit owns them, as main.c:416-448 and reservoir.c:19-46 fill KI and
    pc_aux)."""
    prob = reservoir(24, 20, 16, 2.0, 2.0, 2.5, seed=11)
    rows = [
        dict(len=12, start=(2, 3, 4), pos=1, bl=0, br=1, cont=(5.0e7, 1e-6),
             fractures=[(5, 1e6, 1.0)]),
        dict(len=10, start=(10, 4, 8), pos=2, bl=3, br=3, cont=(1.2, 0.9),
             ccont=(0.5, 2.0), fractures=[(2, 1e5, 2.0), (7, 1e6, 0.5)]),
        dict(len=9, start=(15, 15, 3), pos=3, bl=3, br=0, cont=(0.8, 5.5e7),
             ccont=(2.0, 1.0), Kc=3e-11),
        dict(len=6, start=(8, 3, 4), pos=1, bl=1, br=3, cont=(-2e-6, 1.1),
             ccont=(1.0, 1.5), kindex=2e-12, area=1.5),
    ]
    k = _karst(rows, 2)
    WI, pw = well(prob, 12, 10, 6)
    return prob, k, WI, pw


CASES = {"single": case_single, "multi": case_multi}


def step_state(prob, k, seed):
    """A conduit() input state: a smooth reservoir pressure, conduit
    pressures near it and fracture velocities of both signs."""
    rng = np.random.default_rng(seed)
    x = np.arange(prob.n) % prob.nx
    p_old = 55e6 + 3e6 * np.cos(x / prob.nx * 3.0) + 1e5 * rng.standard_normal(prob.n)
    pc_old = np.zeros((k.mmax, k.nk))
    for j, c in enumerate(k.cells(prob.nx, prob.ny)):
        pc_old[:len(c), j] = p_old[c] + 2e4 * rng.standard_normal(len(c))
    ucR = 1e-4 * rng.standard_normal((k.max_brechas, k.nk))
    ucL = 1e-4 * rng.standard_normal((k.max_brechas, k.nk))
    return p_old, pc_old, ucR, ucL
