"""numpy restatement of the reference's permeability readers (TEST
INFRASTRUCTURE ONLY: the checker for include/hmfem_permio.h).

read_set_perm_field (permeabilities.c:494-668), read_layer_perm_field
(:57-186), gaussian_permfield (:673-772): the file parse and the resample
onto the simulation grid, every floating-point operation as the reference
evaluates it (numpy float64 arithmetic is IEEE, no contraction).
"""
import numpy as np

SPE_DIMS = (60, 220, 85)   # permeabilities.c:518-523


def _numbers(path, want):
    with open(path) as f:
        v = np.array(f.read().split()[:want], dtype=np.float64)
    if v.size < want:
        raise ValueError("too few values")
    return v


def read_spe(path, nxg, nyg, nzg, layer=-1):
    """Three blocks, layers k = nzg-1 .. 0, rows j, columns i ascending, into
    ind(nxg-1-i, nyg-1-j, k); layer >= 0 keeps one layer (K_z = 1e-8)."""
    v = _numbers(path, 3 * nxg * nyg * nzg).reshape(3, nzg, nyg, nxg)
    v = v[:, ::-1, ::-1, ::-1]          # -> [c, k, nyg-1-j, nxg-1-i] ascending
    if layer < 0:
        return [np.ascontiguousarray(v[c]).reshape(-1) for c in range(3)]
    out = [np.ascontiguousarray(v[c, layer]).reshape(-1) for c in range(2)]
    out.append(np.full(nxg * nyg, 1e-8))
    return out


def read_gaussian(path, nxg, nyg, nzg):
    """i, j, k loops (k fastest), three columns, the first used."""
    v = _numbers(path, 3 * nxg * nyg * nzg)[0::3].reshape(nxg, nyg, nzg)
    return np.ascontiguousarray(v.transpose(2, 1, 0)).reshape(-1)


def _geo(n, I, ng):
    h = I / n
    hg = I / ng
    return np.floor(((np.arange(n) + 0.5) * h) / hg).astype(np.int64)


def resample(variant, KXg, KYg, KZg, nxg, nyg, nzg, Ix, Iy, Iz, nx, ny, nz, K0=None):
    """variant 0: 3-D; 1: one layer into the k = 0 plane (other planes from
    K0, default zero); 2: gaussian_permfield (z cell size Iz / nxg)."""
    gi, gj = _geo(nx, Ix, nxg), _geo(ny, Iy, nyg)
    if variant == 2:
        gk = np.floor(((np.arange(nz) + 0.5) * (Iz / nz)) / (Iz / nxg)).astype(np.int64)
    else:
        gk = _geo(nz, Iz, nzg)
    out = []
    for c, G in enumerate((KXg, KYg, KZg)):
        K = np.zeros(nx * ny * nz) if K0 is None else np.array(K0[c], dtype=np.float64)
        if variant == 1:
            g = gi[None, :] + nxg * gj[:, None]
            K[:nx * ny] = G[g].reshape(-1)
        else:
            g = gi[None, None, :] + nxg * (gj[None, :, None] + nyg * gk[:, None, None])
            K[:] = G[g].reshape(-1)
        out.append(K)
    return out


def write_synthetic(path, nvals, seed=0, gaussian=False):
    """A seeded lognormal field in the file layout (SPE blocks, or three
    columns per cell), "%.6e" text."""
    rng = np.random.default_rng(seed)
    v = 1e-13 * 10.0 ** rng.standard_normal(nvals)
    with open(path, "w") as f:
        f.write("\n".join("%.6e" % x for x in v))
        f.write("\n")
    return v
