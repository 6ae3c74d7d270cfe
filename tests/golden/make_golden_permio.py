"""Digests of the REFERENCE's permeability readers (read_set_perm_field,
read_layer_perm_field, gaussian_permfield from permeabilities.c, compiled
into oracle/_ref/libhmfem_ref.so by oracle/Makefile) on seeded synthetic
files in their formats (oracle/permio.py write_synthetic).

    python tests/golden/make_golden_permio.py
"""
import ctypes as C
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import permio  # noqa: E402

# name: (variant, file seed, layer, geological n (gaussian) / SPE dims, grid, domain)
CASES = {
    "spe_30x50x17": (0, 1, -1, None, (30, 50, 17), (1200.0, 2200.0, 170.0)),
    "spe_75x300x100": (0, 1, -1, None, (75, 300, 100), (1200.0, 2200.0, 170.0)),
    "spe_layer37_45x110x1": (1, 1, 37, None, (45, 110, 1), (1200.0, 2200.0, 170.0)),
    "gaussian24_20x28x36": (2, 2, -1, 24, (20, 28, 36), (1.0, 2.0, 3.0)),
}


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def file_for(variant, seed, ng, d):
    path = os.path.join(d, f"perm_{variant}_{seed}_{ng}.txt")
    if not os.path.exists(path):
        n = 3 * (ng ** 3 if variant == 2 else int(np.prod(permio.SPE_DIMS)))
        permio.write_synthetic(path, n, seed=seed)
    return path


def main():
    from oracle.oracle import REF_SO
    L = C.CDLL(REF_SO)
    L.ref_read_perm.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                C.c_void_p, C.c_void_p]
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (variant, seed, layer, ng, (nx, ny, nz), (Ix, Iy, Iz)) in CASES.items():
            path = file_for(variant, seed, ng, d)
            K = [np.zeros(nx * ny * nz) for _ in range(3)]
            L.ref_read_perm(variant, path.encode(), layer, ng or 0, nx, ny, nz, Ix, Iy, Iz,
                            *[k.ctypes.data for k in K])
            out[name] = digest(*K)
            print(name, out[name][:16])
    np.savez(os.path.join(HERE, "permio.npz"), **out)


if __name__ == "__main__":
    main()
