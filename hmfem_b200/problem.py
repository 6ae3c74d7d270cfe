"""Seeded synthetic Darcy problems (permeability fields, conduits, boundary
conditions) with the shapes of hmfem's pressure-solve workloads.

Grid convention is the reference's: cell ``s = i + j*nx + k*nx*ny``
(``pindex``, solve_linearsystem_AMG.c:15-20), so a field is stored as a
C-ordered ``(nz, ny, nx)`` array flattened to length ``n``.

Face order for boundary descriptions (``bc_type`` / ``bc_value``) is
``l, r, u, d, t, b`` = x-, x+, y+, y-, z+, z- -- the order of
``val_bound[1..6]`` in main.c:140-152.  ``bc_type`` 0 is Dirichlet, 1 is
Neumann (main.c:347-350).

Nothing here comes from a public dataset: the reference ships none for this
path, and every field is generated from numpy's PCG64 (``default_rng``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

FACES = ("l", "r", "u", "d", "t", "b")
DIRICHLET, NEUMANN = 0, 1


@dataclass
class Problem:
    nx: int
    ny: int
    nz: int
    hx: float
    hy: float
    hz: float
    KX: np.ndarray
    KY: np.ndarray
    KZ: np.ndarray
    bc_type: tuple = (DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, NEUMANN)
    bc_value: tuple = (1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    visc: float = 1.0
    name: str = ""
    conduit_mask: np.ndarray | None = field(default=None, repr=False)

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    def face_arrays(self):
        """Per-face value arrays in the reference's Bound layout
        (set_boundaries.c:42-125): l/r indexed k*ny+j, u/d k*nx+i,
        t/b j*nx+i."""
        sizes = (self.ny * self.nz, self.ny * self.nz, self.nx * self.nz,
                 self.nx * self.nz, self.nx * self.ny, self.nx * self.ny)
        return [np.full(sz, float(v)) for sz, v in zip(sizes, self.bc_value)]


def random_walk_conduit(rng: np.random.Generator, nx: int, ny: int, nz: int):
    """One 6-connected, 1-cell-wide random-walk conduit.

    Starts at a uniform cell of the x=0 face; each step moves +x with
    probability 1/2 and +y, -y, +z, -z with 1/8 each (one uniform draw u per
    step: u<.5 +x, <.625 +y, <.75 -y, <.875 +z, else -z).  A lateral step that
    would leave the domain is rejected and the walker stays put.  The walk
    stops when x reaches nx.  Returns the visited cell indices."""
    x = 0
    y = int(rng.integers(0, ny))
    z = int(rng.integers(0, nz))
    cells = [x + y * nx + z * nx * ny]
    while True:
        u = rng.random()
        if u < 0.5:
            x += 1
            if x >= nx:
                break
        elif u < 0.625:
            if y + 1 < ny:
                y += 1
        elif u < 0.75:
            if y > 0:
                y -= 1
        elif u < 0.875:
            if z + 1 < nz:
                z += 1
        else:
            if z > 0:
                z -= 1
        cells.append(x + y * nx + z * nx * ny)
    return np.unique(np.asarray(cells, dtype=np.int64))


def gaussian_field(rng: np.random.Generator, nx: int, ny: int, nz: int,
                   corr: float) -> np.ndarray:
    """Unit-variance Gaussian random field: white noise N(0,1) convolved
    (periodically, by FFT) with a normalised isotropic Gaussian kernel of
    standard deviation ``corr`` cells, then standardised to zero sample mean
    and unit sample variance.  Returns a flat array of n cells."""
    g = rng.standard_normal((nz, ny, nx))
    if corr > 0:
        kz = np.fft.fftfreq(nz)[:, None, None]
        ky = np.fft.fftfreq(ny)[None, :, None]
        kx = np.fft.rfftfreq(nx)[None, None, :]
        # Fourier transform of a unit-mass Gaussian of std `corr` cells
        ker = np.exp(-2.0 * (np.pi * corr) ** 2 * (kx**2 + ky**2 + kz**2))
        g = np.fft.irfftn(np.fft.rfftn(g) * ker, s=(nz, ny, nx), axes=(0, 1, 2))
    g = g - g.mean()
    sd = g.std()
    if sd > 0:
        g = g / sd
    return g.reshape(-1)


def make_problem(nx, ny, nz, log10k=None, kbg=1e-14, n_conduits=0,
                 k_conduit=1e-10, seed=0, lengths=(1.0, 1.0, 1.0),
                 name="", bc_type=None, bc_value=None) -> Problem:
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    if log10k is not None:
        mean, std, corr = log10k
        K = 10.0 ** (mean + std * gaussian_field(rng, nx, ny, nz, corr))
    else:
        K = np.full(n, float(kbg))
    mask = np.zeros(n, dtype=np.uint8)
    for _ in range(n_conduits):
        c = random_walk_conduit(rng, nx, ny, nz)
        K[c] = k_conduit
        mask[c] = 1
    K = np.ascontiguousarray(K, dtype=np.float64)
    p = Problem(nx, ny, nz, lengths[0] / nx, lengths[1] / ny, lengths[2] / nz,
                K, K, K, name=name, conduit_mask=mask)
    if bc_type is not None:
        p.bc_type = tuple(bc_type)
    if bc_value is not None:
        p.bc_value = tuple(bc_value)
    return p


def config_problem(config: int, realisation: int = 0, size=None) -> Problem:
    """The synthetic workloads: seed = 1000 + 100*config + realisation.

    0: 32^3, K = 1e-14 homogeneous.
    1: 128^3, K = 1e-14 + 4 conduits at 1e-10.
    2: 256^3, log10 K = -14 + 1.5 g (correlation 8 cells) + 8 conduits at 1e-9.
    3: one uneven instance: n_x,n_y,n_z ~ U{24..96}, lengths n/64 m,
       log10 std ~ U[1,2], correlation 4 cells, 0-4 conduits at 1e-10.
    4: 128^3 lognormal (std 1.5, correlation 8) with 0-6 conduits at 1e-10.
    ``size`` overrides the cube edge (for scaled-down parity cases)."""
    seed = 1000 + 100 * config + realisation
    if config == 0:
        s = size or 32
        return make_problem(s, s, s, kbg=1e-14, seed=seed, name=f"homog{s}")
    if config == 1:
        s = size or 128
        return make_problem(s, s, s, kbg=1e-14, n_conduits=4, k_conduit=1e-10,
                            seed=seed, name=f"conduit{s}")
    if config == 2:
        s = size or 256
        return make_problem(s, s, s, log10k=(-14.0, 1.5, 8.0), n_conduits=8,
                            k_conduit=1e-9, seed=seed, name=f"lognormal{s}")
    if config == 3:
        rng = np.random.default_rng(seed)
        nx, ny, nz = (int(v) for v in rng.integers(24, 97, size=3))
        std = float(rng.uniform(1.0, 2.0))
        nc = int(rng.integers(0, 5))
        return make_problem(nx, ny, nz, log10k=(-14.0, std, 4.0),
                            n_conduits=nc, k_conduit=1e-10, seed=seed + 50000,
                            lengths=(nx / 64, ny / 64, nz / 64),
                            name=f"batch{realisation}")
    if config == 4:
        s = size or 128
        rng = np.random.default_rng(seed)
        nc = int(rng.integers(0, 7))
        return make_problem(s, s, s, log10k=(-14.0, 1.5, 8.0), n_conduits=nc,
                            k_conduit=1e-10, seed=seed + 50000,
                            name=f"learned{s}")
    raise ValueError(f"unknown config {config}")
