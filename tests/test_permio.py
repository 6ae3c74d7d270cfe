"""Permeability from geological files: the numpy restatement
(oracle/permio.py) against digests of the reference's own readers
(tests/golden/make_golden_permio.py), then the library's host parse +
device resample (include/hmfem_permio.h) against both, bit for bit."""
import ctypes as C
import hashlib
import importlib.util
import os

import numpy as np
import pytest

from oracle import permio as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
_spec = importlib.util.spec_from_file_location(
    "make_golden_permio", os.path.join(GOLD, "make_golden_permio.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("perm"))
    return lambda variant, seed, ng: MG.file_for(variant, seed, ng, d)


def oracle_fields(case, path):
    variant, seed, layer, ng, (nx, ny, nz), (Ix, Iy, Iz) = case
    if variant == 2:
        G = O.read_gaussian(path, ng, ng, ng)
        return O.resample(2, G, G, G, ng, ng, ng, Ix, Iy, Iz, nx, ny, nz)
    nxg, nyg, nzg = O.SPE_DIMS
    G = O.read_spe(path, nxg, nyg, nzg, layer)
    return O.resample(variant, *G, nxg, nyg, nzg, Ix, Iy, Iz, nx, ny, nz)


@pytest.mark.parametrize("name", sorted(MG.CASES))
def test_restatement_equals_reference(name, files):
    case = MG.CASES[name]
    path = files(case[0], case[1], case[3])
    K = oracle_fields(case, path)
    assert digest(*K) == str(np.load(os.path.join(GOLD, "permio.npz"))[name])


def _lib():
    from hmfem_b200 import gpu
    L = gpu.lib()
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.hmfem_read_spe.argtypes = [C.c_char_p, i, i, i, i, vp, vp, vp]
    L.hmfem_read_gaussian.argtypes = [C.c_char_p, i, i, i, vp]
    L.hmfem_resample_perm.argtypes = [i, vp, vp, vp, i, i, i, d, d, d, i, i, i, vp, vp, vp, i]
    return L


def _p(a):
    return C.c_void_p(a.ctypes.data)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(MG.CASES))
def test_gpu_reader_and_resample(name, files):
    case = MG.CASES[name]
    variant, seed, layer, ng, (nx, ny, nz), (Ix, Iy, Iz) = case
    path = files(variant, seed, ng)
    L = _lib()
    if variant == 2:
        G = np.zeros(ng ** 3)
        assert L.hmfem_read_gaussian(path.encode(), ng, ng, ng, _p(G)) == 0
        Gs, dims = [G, G, G], (ng, ng, ng)
        assert np.array_equal(G, O.read_gaussian(path, ng, ng, ng))
    else:
        nxg, nyg, nzg = O.SPE_DIMS
        m = nxg * nyg * (nzg if layer < 0 else 1)
        Gs = [np.zeros(m) for _ in range(3)]
        assert L.hmfem_read_spe(path.encode(), nxg, nyg, nzg, layer, *[_p(g) for g in Gs]) == 0
        for a, b in zip(Gs, O.read_spe(path, nxg, nyg, nzg, layer)):
            assert np.array_equal(a, b)
        dims = (nxg, nyg, nzg)
    K = [np.zeros(nx * ny * nz) for _ in range(3)]
    assert L.hmfem_resample_perm(variant, *[_p(g) for g in Gs], *dims, Ix, Iy, Iz, nx, ny, nz,
                                 *[_p(k) for k in K], 0) == 0
    assert digest(*K) == str(np.load(os.path.join(GOLD, "permio.npz"))[name])


@pytest.mark.gpu
def test_gpu_resample_device_arrays(files):
    torch = pytest.importorskip("torch")
    variant, seed, layer, ng, (nx, ny, nz), (Ix, Iy, Iz) = MG.CASES["spe_75x300x100"]
    nxg, nyg, nzg = O.SPE_DIMS
    Gs = O.read_spe(files(variant, seed, ng), nxg, nyg, nzg, layer)
    dG = [torch.as_tensor(g, device="cuda") for g in Gs]
    dK = [torch.zeros(nx * ny * nz, dtype=torch.float64, device="cuda") for _ in range(3)]
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert _lib().hmfem_resample_perm(0, *[vp(g) for g in dG], nxg, nyg, nzg, Ix, Iy, Iz,
                                      nx, ny, nz, *[vp(k) for k in dK], 1) == 0
    torch.cuda.synchronize()
    K = [k.cpu().numpy() for k in dK]
    assert digest(*K) == str(np.load(os.path.join(GOLD, "permio.npz"))["spe_75x300x100"])


def test_short_file_is_rejected(tmp_path):
    p = tmp_path / "short.txt"
    p.write_text("1e-13 2e-13\n")
    G = np.zeros(8)
    assert _lib().hmfem_read_spe(str(p).encode(), 2, 2, 2, -1, _p(G), _p(G), _p(G)) != 0
