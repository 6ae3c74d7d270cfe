"""hmfem_fluxes_noalloc: the flux entry point for callers that cannot let
the library allocate device memory (for example an application whose GPU
memory is already reserved by its own or a framework's caching allocator).

Collected last (file name) so that a first-failure run has already run every
other test.  Works both alone in a fresh process and after the other tests:
the first call on the device sets up the scratch address itself.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import config_problem, make_problem  # noqa: E402

FACES = [0, 1, 2, 3, 5, 6]  # u, d, l, r, t, b (c is left untouched)


def _reference_fluxes(prob):
    """Pressure and fluxes through the existing solver entry points."""
    s = gpu.Solver(tol=1e-12)
    s.assemble(prob)
    x, _ = s.solve()
    v, dmin, dmax = s.fluxes(x)
    s.close()
    return x, v, dmin, dmax


def _noalloc(prob, x):
    dev = torch.device("cuda")
    K = [torch.tensor(a, device=dev) for a in (prob.KX, prob.KY, prob.KZ)]
    p = torch.tensor(x, device=dev)
    v = torch.full((prob.n, 7), 7.0, dtype=torch.float64, device=dev)
    dmin, dmax = gpu.fluxes_noalloc(prob, K[0], K[1], K[2], p, v)
    out = v.cpu().numpy()
    assert np.all(out[:, 4] == 7.0)  # the c field is not written
    return out, dmin, dmax


def test_noalloc_matches_existing_entry_point_twice_in_a_row():
    a = config_problem(2, size=24)
    b = make_problem(9, 6, 7, log10k=(-13.0, 1.0, 2.0), n_conduits=1, seed=4,
                     bc_type=(0, 1, 0, 1, 0, 1),
                     bc_value=(2.0, 0.5, 1.0, -0.3, 0.25, 0.7))
    for prob in (a, b):  # two calls in a row share (and reuse) the scratch
        x, v, dmin, dmax = _reference_fluxes(prob)
        vn, nmin, nmax = _noalloc(prob, x)
        np.testing.assert_array_equal(vn[:, FACES], v[:, FACES])
        assert nmin == dmin and nmax == dmax


def test_noalloc_rejects_faces_beyond_the_scratch():
    side = int(np.sqrt(gpu.NOALLOC_MAX_FACE)) + 1
    prob = make_problem(side, side, 1)
    dev = torch.device("cuda")
    K = torch.zeros(1, dtype=torch.float64, device=dev)
    with pytest.raises(gpu.HmfemError) as e:
        gpu.fluxes_noalloc(prob, K, K, K, K, K)
    assert e.value.code == gpu.E_CAPACITY
    assert "HMFEM_NOALLOC_MAX_FACE" in str(e.value)
