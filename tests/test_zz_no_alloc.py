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
    # no Dirichlet face at all: the reference pins one cell's left face
    # (permeabilities.c), a branch of its own in the face coefficients
    c = make_problem(6, 4, 5, log10k=(-13.0, 0.5, 1.0), seed=5, bc_type=(1,) * 6,
                     bc_value=(0.1, 0.1, 0.0, 0.0, 0.0, 0.0))
    for prob in (a, b, c):  # calls in a row share (and reuse) the scratch
        x, v, dmin, dmax = _reference_fluxes(prob)
        vn, nmin, nmax = _noalloc(prob, x)
        np.testing.assert_array_equal(vn[:, FACES], v[:, FACES])
        assert nmin == dmin and nmax == dmax


def test_noalloc_rejects_faces_beyond_the_scratch():
    side = int(np.sqrt(gpu.NOALLOC_MAX_FACE)) + 1
    prob = make_problem(side, side, 1)
    dev = torch.device("cuda")
    # arrays of the grid's full size: were the capacity check ever to let the
    # call through, it would compute on valid memory and fail the assertions
    K = torch.full((prob.n,), 1e-14, dtype=torch.float64, device=dev)
    p = torch.zeros(prob.n, dtype=torch.float64, device=dev)
    v = torch.zeros((prob.n, 7), dtype=torch.float64, device=dev)
    with pytest.raises(gpu.HmfemError) as e:
        gpu.fluxes_noalloc(prob, K, K, K, p, v)
    assert e.value.code == gpu.E_CAPACITY
    assert "HMFEM_NOALLOC_MAX_FACE" in str(e.value)


def test_noalloc_python_front_end_rejects_mismatched_arrays():
    prob = make_problem(4, 3, 2)
    dev = torch.device("cuda")
    K = torch.full((prob.n,), 1e-14, dtype=torch.float64, device=dev)
    p = torch.zeros(prob.n, dtype=torch.float64, device=dev)
    v = torch.zeros((prob.n, 7), dtype=torch.float64, device=dev)
    for bad in (dict(p=p.float()), dict(p=p[:-1]), dict(v=v[:, :6].contiguous()),
                dict(KX=K.cpu())):
        args = dict(KX=K, KY=K, KZ=K, p=p, v=v)
        args.update(bad)
        with pytest.raises(ValueError):
            gpu.fluxes_noalloc(prob, **args)
