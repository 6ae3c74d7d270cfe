"""The reference's result files (pressure_reservoir.dat, flux_reservoir.dat,
campos.vts, pressure_karst_<j>.dat, flux_karst_<j>.dat): the Python
restatement against files the reference's own writers produced
(tests/golden/make_golden_text.py), then the GPU writers (include/
hmfem_textio.h) byte for byte against both."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from oracle import textio as T

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
_spec = importlib.util.spec_from_file_location(
    "make_golden_text", os.path.join(GOLD, "make_golden_text.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)

KARST_FILES = ["pressure_karst_%d.dat" % j for j in range(3)] + \
    ["flux_karst_%d.dat" % j for j in range(3)]


def gold(name):
    with open(os.path.join(GOLD, "text_" + name), "rb") as f:
        return f.read()


@pytest.fixture(scope="module")
def case():
    return MG.text_case()


def test_python_restatement_equals_reference_writers(case):
    p, v, k, pc, ucl, ucr = case
    nx, ny, nz, hx, hy, hz = MG.GRID
    assert T.pressure_text(nx, ny, nz, hx, hy, hz, p).encode() == gold("pressure_reservoir.dat")
    assert T.flux_text(nx, ny, nz, hx, hy, hz, v).encode() == gold("flux_reservoir.dat")
    assert T.vts_text(nx, ny, nz, hx, hy, hz, v, p).encode() == gold("campos.vts")
    files = T.karst_texts(k, hx, hy, hz, pc, ucl, ucr)
    for name in KARST_FILES:
        assert files[name].encode() == gold(name), name


# ---- GPU writers ------------------------------------------------------------------

def _lib():
    from hmfem_b200 import gpu, karst
    L = gpu.lib()
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.hmfem_save_pressure.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, i]
    L.hmfem_save_flux.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, i]
    L.hmfem_save_vts.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, vp, i]
    L.hmfem_save_karst.argtypes = [C.c_char_p, C.POINTER(karst.KarstStruct), d, d, d, vp, vp,
                                   vp, i]
    L.hmfem_format_numbers.argtypes = [vp, C.c_long, C.c_char, i, C.c_char_p, C.c_long,
                                       C.POINTER(C.c_long), i]
    return L


def _p(a):
    return C.c_void_p(a.ctypes.data)


def gpu_files(tmp, nx, ny, nz, hx, hy, hz, p, v):
    L = _lib()
    p = np.ascontiguousarray(p, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = {}
    for name, call in (("pressure_reservoir.dat",
                        lambda f: L.hmfem_save_pressure(f, nx, ny, nz, hx, hy, hz, _p(p), 0)),
                       ("flux_reservoir.dat",
                        lambda f: L.hmfem_save_flux(f, nx, ny, nz, hx, hy, hz, _p(v), 0)),
                       ("campos.vts",
                        lambda f: L.hmfem_save_vts(f, nx, ny, nz, hx, hy, hz, _p(v), _p(p), 0))):
        path = os.path.join(tmp, name)
        rc = call(path.encode())
        assert rc == 0, name
        with open(path, "rb") as fh:
            out[name] = fh.read()
    return out


@pytest.mark.gpu
def test_gpu_writers_equal_reference_files(case, tmp_path):
    p, v, k, pc, ucl, ucr = case
    out = gpu_files(str(tmp_path), *MG.GRID, p, v)
    for name, data in out.items():
        assert data == gold(name), name
    L = _lib()
    arrs = [np.ascontiguousarray(a) for a in (pc, ucl, ucr)]
    ks = k.struct()
    nx, ny, nz, hx, hy, hz = MG.GRID
    assert L.hmfem_save_karst(str(tmp_path).encode(), C.byref(ks), hx, hy, hz,
                              *[_p(a) for a in arrs], 0) == 0
    for name in KARST_FILES:
        with open(os.path.join(str(tmp_path), name), "rb") as fh:
            assert fh.read() == gold(name), name


@pytest.mark.gpu
def test_gpu_writers_on_a_larger_grid(tmp_path):
    """40 x 30 x 20 (24k lines, several kernel chunks' worth of work per
    file) of lognormal pressures and fluxes against the Python writers."""
    nx, ny, nz, hx, hy, hz = 40, 30, 20, 0.013, 7.0 / 3.0, 0.1
    rng = np.random.default_rng(8)
    p = np.exp(rng.standard_normal(nx * ny * nz) * 8) * rng.choice([-1, 1], nx * ny * nz)
    v = rng.standard_normal((nx * ny * nz, 7)) * 10.0 ** rng.integers(-15, 3, (nx * ny * nz, 1))
    out = gpu_files(str(tmp_path), nx, ny, nz, hx, hy, hz, p, v)
    assert out["pressure_reservoir.dat"] == T.pressure_text(nx, ny, nz, hx, hy, hz, p).encode()
    assert out["flux_reservoir.dat"] == T.flux_text(nx, ny, nz, hx, hy, hz, v).encode()
    assert out["campos.vts"] == T.vts_text(nx, ny, nz, hx, hy, hz, v, p).encode()


def adversarial_values(seed=1):
    """Values at every decimal magnitude the exact path covers and beyond,
    exact ties at several digit positions, the neighbours of powers of ten,
    signed zeros, subnormals, infinities and NaN."""
    rng = np.random.default_rng(seed)
    vals = [0.0, -0.0, 5e-324, -5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
            float("inf"), float("-inf"), float("nan")]
    for e in range(-40, 45):
        b = 10.0 ** e
        vals += [b, np.nextafter(b, 0), np.nextafter(b, np.inf), -b, 9.99999999995 * b,
                 9.9999999995 * b, 1.2345678905 * b, 5.0 * b, 0.5 * b]
    # exact binary ties: k/2^q at various q
    for q in range(1, 30):
        for kk in (1, 3, 5, 7, 123, 1001):
            vals.append(kk / 2.0 ** q)
            vals.append(-kk / 2.0 ** q)
    vals += [1234567890.5, 1234567891.5, 0.0078125, 0.0234375, 0.03125, 0.09375]
    # the edge of the device's 256-bit range for tiny magnitudes (5^86)
    for e in range(-90, -40):
        vals += [1.2345678905 * 10.0 ** e, -7.0 * 10.0 ** e, 2.0 ** (3.32 * e)]
    x = rng.standard_normal(20000) * 10.0 ** rng.integers(-25, 40, 20000)
    return np.concatenate([np.array(vals, dtype=np.float64), x])


@pytest.mark.gpu
@pytest.mark.parametrize("conv,prec", [("e", 9), ("e", 8), ("e", 0), ("e", 3), ("e", 17),
                                       ("f", 6), ("f", 4), ("f", 0), ("f", 12)])
def test_gpu_number_conversion(conv, prec):
    x = adversarial_values()
    if conv == "f":
        x = x[np.abs(np.nan_to_num(x, posinf=0, neginf=0)) < 1e30]  # keep %f lines short
    want = T.number_text(x, conv, prec).encode()
    L = _lib()
    buf = C.create_string_buffer(len(want) + 64)
    used = C.c_long()
    rc = L.hmfem_format_numbers(_p(x), len(x), conv.encode(), prec, buf, len(buf),
                                C.byref(used), 0)
    assert rc == 0
    got = buf.raw[:used.value]
    if got != want:
        g, w = got.split(b"\n"), want.split(b"\n")
        bad = [(float(x[i]), g[i], w[i]) for i in range(min(len(g), len(w))) if g[i] != w[i]]
        raise AssertionError(f"{len(bad)} differ, first: {bad[:5]}")
