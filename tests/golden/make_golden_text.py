"""Generates the result-file fixtures under tests/golden/ with the
REFERENCE's own writers (posprocessing_output.c save_pressure / save_flux /
save_pressure_1d / save_flux_1d and vtk.c vts_StructuredGrid_file, compiled
from the hmfem tree into oracle/_ref/libhmfem_ref.so by oracle/Makefile).

    python tests/golden/make_golden_text.py

Inputs are seeded (text_case() below) and include the cases a formatter
gets wrong first: exact ties at the last printed digit (cell centres of
h = 1/64 under %.6f, of h = 1/16 under %.4f, x.5 integers under %1.9e),
signed zeros, a value that rounds up to the next power of ten, magnitudes
far outside the device's exact range, infinities and NaN.  The writers run
in a child process: save_pressure_1d closes only its last file, so the
others are flushed when the process exits.
"""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

GRID = (5, 4, 3, 1.0 / 64, 0.37, 1.0 / 16)


def text_case():
    """(p, v, karst set, pc, ucl, ucr) of the fixtures."""
    from hmfem_b200.karst import Karst
    nx, ny, nz = GRID[:3]
    n = nx * ny * nz
    rng = np.random.default_rng(2024)
    p = 6e7 * (1 + 0.1 * rng.standard_normal(n))
    special = [0.0, -0.0, 1234567890.5, 1234567891.5, 9.9999999995e5, 2.5e-7, -3.0e-12,
               1e-19, 1e36, 4.2e40, float("inf"), float("-inf"), float("nan"),
               5e-324, -1.0, 123.456]
    p[:len(special)] = special
    v = rng.standard_normal((n, 7)) * 1e-6
    v[0, :] = 0.0
    v[1, 3], v[1, 2] = 1e-30, -1e-30
    k = Karst([4, 3, 3], [0, 2, 1], [1, 0, 3], [1, 0, 2], [1, 2, 5], [1e-11] * 3, [1] * 3,
              [1] * 3, np.zeros((2, 3)), np.ones((2, 3)), [1e-12] * 3, [1.0] * 3, [0, 0, 0],
              np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)))
    pc = 6e7 + 1e5 * rng.standard_normal((k.mmax, k.nk))
    ucl = 1e-5 * rng.standard_normal((k.mmax, k.nk))
    ucr = 1e-5 * rng.standard_normal((k.mmax, k.nk))
    return p, v, k, pc, ucl, ucr


def _child(out_dir):
    from oracle.oracle import REF_SO
    L = C.CDLL(REF_SO)
    p, v, k, pc, ucl, ucr = text_case()
    nx, ny, nz, hx, hy, hz = GRID
    L.ref_save_grid.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_void_p, C.c_void_p]
    L.ref_save_karst.argtypes = [C.c_char_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    pp = np.ascontiguousarray(p)
    vv = np.ascontiguousarray(v)
    L.ref_save_grid(out_dir.encode(), nx, ny, nz, hx, hy, hz, pp.ctypes.data, vv.ctypes.data)
    ks = k.struct()
    arrs = [np.ascontiguousarray(a) for a in (pc, ucl, ucr)]
    L.ref_save_karst(out_dir.encode(), C.addressof(ks), hx, hy, hz, *[a.ctypes.data for a in arrs])


def main():
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([sys.executable, __file__, "--child", d], check=True,
                       stdout=subprocess.DEVNULL)
        for f in sorted(os.listdir(d)):
            shutil.copyfile(os.path.join(d, f), os.path.join(HERE, "text_" + f))
            print("text_" + f, os.path.getsize(os.path.join(d, f)))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--child":
        _child(sys.argv[2])
    else:
        main()
