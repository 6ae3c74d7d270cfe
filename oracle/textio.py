"""Python restatement of the reference's result writers (TEST
INFRASTRUCTURE ONLY: the checker for the GPU text writers).

Python's %-formatting of floats is correctly rounded (exact decimal value,
ties to even), as glibc's printf is, so these strings equal the bytes the
reference's fprintf calls write; tests/test_textio.py pins that against
files written by the reference's own writers (tests/golden/text_*).
"""
import numpy as np

ELE = ("u", "d", "l", "r", "c", "t", "b")   # structs.h:7-17 field order


def _co(h, i):
    return h * (i + 0.5)


def pressure_text(nx, ny, nz, hx, hy, hz, p):
    """posprocessing_output.c:200-234 (save_pressure)."""
    out = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                s = i + nx * (j + ny * k)
                out.append("%.6f %.6f %.6f %1.9e\n" % (_co(hx, i), _co(hy, j), _co(hz, k), p[s]))
            out.append(" \n")
        out.append(" \n")
    return "".join(out)


def _half_diffs(v):
    v = np.asarray(v).reshape(-1, 7)
    return (0.5 * (v[:, 3] - v[:, 2]), 0.5 * (v[:, 0] - v[:, 1]), 0.5 * (v[:, 5] - v[:, 6]))


def flux_text(nx, ny, nz, hx, hy, hz, v):
    """posprocessing_output.c:236-296 (save_flux)."""
    vx, vy, vz = _half_diffs(v)
    out = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                s = i + nx * (j + ny * k)
                out.append("%.6f %.6f %.6f %1.9e %1.9e %1.9e \n"
                           % (_co(hx, i), _co(hy, j), _co(hz, k), vx[s], vy[s], vz[s]))
    return "".join(out)


def vts_text(nx, ny, nz, hx, hy, hz, v, p):
    """vtk.c:8-76 (vts_StructuredGrid_file)."""
    vx, vy, vz = _half_diffs(v)
    n = nx * ny * nz
    out = ['<?xml version="1.0"?>\n', '<VTKFile type="StructuredGrid" version="0.1">\n',
           '<StructuredGrid WholeExtent="0 %d 0 %d 0 %d">\n' % (nx - 1, ny - 1, nz - 1),
           '<Piece Extent="0 %d 0 %d 0 %d">\n' % (nx - 1, ny - 1, nz - 1),
           '<PointData  Vectors="Velocity" Scalars="pressure">\n',
           '<DataArray type="Float32" Name="Velocity" NumberOfComponents="3" format="ascii">\n']
    out += ["%1.8e %1.8e %1.8e\n" % (vx[s], vy[s], vz[s]) for s in range(n)]
    out += ['</DataArray>\n',
            '<DataArray type="Float32" Name="pressure" NumberOfComponents="1" format="ascii">\n']
    out += ["%1.8e\n" % p[s] for s in range(n)]
    out += ['</DataArray>\n', '</PointData>\n', '<CellData>\n', '</CellData>\n', '<Points>\n',
            '<DataArray type="Float32" NumberOfComponents="3">\n']
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                out.append("%.4f %.4f %.4f \n" % (_co(hx, i), _co(hy, j), _co(hz, k)))
    out += ['</DataArray>\n', '</Points>\n', '</Piece>\n', '</StructuredGrid>\n', '</VTKFile>\n']
    return "".join(out)


_DIR = {1: (1, 0, 0), 2: (0, 1, 0), 3: (0, 0, 1), 4: (1, 1, 0), 5: (1, -1, 0),
        6: (-1, 1, 0), 7: (-1, -1, 0)}


def karst_texts(k, hx, hy, hz, pc, ucl, ucr):
    """posprocessing_output.c:437-661 (save_pressure_1d, save_flux_1d):
    {file name: text}."""
    files = {}
    for j in range(k.nk):
        dx, dy, dz = _DIR[int(k.pos[j])]
        pl, fl = [], []
        for i in range(int(k.len[j])):
            x, y, z = k.sxi[j] + i * dx, k.syi[j] + i * dy, k.szi[j] + i * dz
            c = "%.6f %.6f %.6f " % (_co(hx, x), _co(hy, y), _co(hz, z))
            pl.append(c + "%1.9e\n" % pc[i, j])
            fl.append(c + "%1.9e\n" % (0.5 * (ucr[i, j] - ucl[i, j])))
        files["pressure_karst_%d.dat" % j] = "".join(pl)
        files["flux_karst_%d.dat" % j] = "".join(fl)
    return files


def number_text(x, conv, prec):
    """hmfem_format_numbers: one "%.<prec><conv>\\n" per value."""
    f = "%." + str(prec) + conv + "\n"
    return "".join(f % float(v) for v in x)
