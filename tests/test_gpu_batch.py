"""Batched uneven solves (config 3 shape): several solvers on their own
streams, driven from worker threads, give exactly the results of one solver
run alone."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import batch, gpu  # noqa: E402
from hmfem_b200.problem import make_problem  # noqa: E402

SHAPES = [(12, 9, 15), (20, 8, 6), (16, 16, 16), (7, 11, 5), (24, 10, 9), (9, 9, 30)]


def _problems():
    return [make_problem(nx, ny, nz, log10k=(-14.0, 1.0 + 0.2 * i, 2.0),
                         n_conduits=i % 3, k_conduit=1e-10, seed=40 + i,
                         lengths=(nx / 64, ny / 64, nz / 64))
            for i, (nx, ny, nz) in enumerate(SHAPES)]


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_one_solver(precision):
    probs = _problems()
    res = batch.solve_batch(probs, precision=precision, tol=1e-10, workers=3)
    for p, (x, st, sec) in zip(probs, res):
        assert st["status"] == 0 and st["relres"] <= 1e-10
        assert sec > 0
        s = gpu.Solver(precision=precision, tol=1e-10)
        s.assemble(p)
        s.setup()
        xs, sts = s.solve()
        s.close()
        np.testing.assert_array_equal(x, xs)
        assert st["iterations"] == sts["iterations"]


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_graph_equals_one_solver(precision):
    """All instances solved by one batched graph (hmfem_batch_solve): each
    gives bit for bit the pressure and the iteration count of its own
    solve, though the instances converge after different iteration counts."""
    probs = _problems()
    opts = dict(schur0=1, bf16_from=1) if precision == 1 else {}
    res = batch.solve_batch_graph(probs, precision=precision, tol=1e-10, workers=3,
                                  options=opts)
    its = set()
    for p, (x, st, sec) in zip(probs, res):
        assert st["status"] == 0 and st["relres"] <= 1e-10
        assert sec > 0
        s = gpu.Solver(precision=precision, tol=1e-10, **opts)
        s.assemble(p)
        s.setup()
        xs, sts = s.solve()
        s.close()
        np.testing.assert_array_equal(x, xs)
        assert st["iterations"] == sts["iterations"]
        its.add(st["iterations"])
    assert len(its) > 1   # a mask of converged instances was needed


def test_batch_graph_rejects_a_solver_twice():
    p = _problems()[0]
    s = gpu.Solver()
    s.assemble(p)
    s.setup()
    with pytest.raises(gpu.HmfemError) as e:
        gpu.batch_solve([s, s])
    assert e.value.code == gpu.E_ARG
    s.close()


def test_tune_picks_a_driver_and_worker_count(tmp_path):
    probs = _problems()
    d, w, entry = batch.tune(probs, precision=1, candidates=(1, 2),
                             cache=str(tmp_path / "t.json"))
    assert d in ("graph", "threads") and w in (1, 2)
    assert len(entry["instances_per_s"]) == 4
    d2, w2, _ = batch.tune(probs, precision=1, candidates=(1, 2),
                           cache=str(tmp_path / "t.json"))
    assert (d2, w2) == (d, w)  # read back from the cache


def test_tune_workers_picks_a_candidate(tmp_path):
    probs = _problems()
    w, entry = batch.tune_workers(probs, precision=1, candidates=(1, 2),
                                  cache=str(tmp_path / "t.json"))
    assert w in (1, 2)
    w2, _ = batch.tune_workers(probs, precision=1, candidates=(1, 2),
                               cache=str(tmp_path / "t.json"))
    assert w2 == w  # read back from the cache
