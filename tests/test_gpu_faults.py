"""Failure paths of the solver, provoked from the host without faulting the
GPU: invalid inputs, a matrix that is not SPD, a right-hand side with NaN,
and a bounded device wait made to run out.  Each case checks the status
code, the message, and that the same solver object (and the process) keeps
working afterwards.

The reference has no status codes: it prints CUDA errors and continues
(toolbox/toolbox.h:21-26), flips a negative sigma silently
(toolbox/inverse_operator/pcg.h:47) and reads indices unchecked.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import config_problem, make_problem  # noqa: E402
from oracle.oracle import Port  # noqa: E402


def _solve_ok(s, prob):
    s.assemble(prob)
    s.setup()
    x, st = s.solve()
    assert st["status"] == gpu.OK and st["relres"] <= 1e-10, st
    return x


@pytest.mark.parametrize("bad", [np.nan, np.inf, -1e-14])
@pytest.mark.parametrize("axis", ["KX", "KZ"])
def test_invalid_permeability_is_rejected_and_solver_recovers(bad, axis):
    prob = config_problem(2, size=12)
    good = make_problem(12, 12, 12, log10k=(-14.0, 1.0, 2.0), seed=3)
    s = gpu.Solver(tol=1e-10)
    K = {a: getattr(prob, a).copy() for a in ("KX", "KY", "KZ")}
    K[axis][777] = bad
    with pytest.raises(gpu.HmfemError) as e:
        s.assemble(prob, **K)
    assert e.value.code == gpu.E_ARG
    assert "cell 777" in str(e.value)
    for call in (s.setup, s.solve):  # the rejected matrix is never used
        with pytest.raises(gpu.HmfemError) as e:
            call()
        assert e.value.code == gpu.E_ARG
    _solve_ok(s, good)
    s.close()


def test_invalid_permeability_on_device_arrays():
    prob = config_problem(2, size=10)
    K = torch.tensor(prob.KX, device="cuda")
    K[5] = float("nan")
    s = gpu.Solver()
    with pytest.raises(gpu.HmfemError) as e:
        s.assemble(prob, KX=K, KY=K, KZ=K)
    assert e.value.code == gpu.E_ARG
    s.close()


def _laplace_1d(n, diag=2.0, off=-1.0):
    cnt = np.full(n, 3, np.int32)
    cnt[0] = cnt[-1] = 2
    col, ele = [], []
    for i in range(n):
        for j in (i - 1, i, i + 1):
            if 0 <= j < n:
                col.append(j)
                ele.append(diag if j == i else off)
    return cnt, np.array(col, np.int32), np.array(ele)


@pytest.mark.parametrize("diag,off", [(-2.0, 1.0), (0.0, -1.0)])
def test_matrix_with_nonpositive_diagonal_gives_breakdown(diag, off):
    """Negative definite (-L) and zero-diagonal (indefinite) matrices: a
    diagonal entry <= 0 proves the matrix is not SPD."""
    cnt, col, ele = _laplace_1d(500, diag, off)
    s = gpu.Solver(tol=1e-10)
    s.set_matrix(cnt, col, ele, np.ones(500))
    with pytest.raises(gpu.HmfemError) as e:
        s.setup()
    assert e.value.code == gpu.E_BREAKDOWN
    assert "not SPD" in str(e.value)
    # the same object takes a valid matrix afterwards
    cnt, col, ele = _laplace_1d(500)
    s.set_matrix(cnt, col, ele, np.ones(500))
    s.setup()
    x, st = s.solve()
    assert st["status"] == gpu.OK
    s.close()


@pytest.mark.parametrize("where", ["b", "x0"])
@pytest.mark.parametrize("precision", [0, 1])
def test_nan_in_right_hand_side_or_guess_gives_breakdown(where, precision):
    prob = config_problem(2, size=16)
    s = gpu.Solver(tol=1e-10, precision=precision)
    s.assemble(prob)
    s.setup()
    _, _, b = Port().assemble(prob)   # the assembled right-hand side
    x = np.zeros(prob.n)
    if where == "x0":
        x[100] = np.nan
        with pytest.raises(gpu.HmfemError) as e:
            s.solve(x=x)
    else:
        bb = b.copy()
        bb[100] = np.nan
        with pytest.raises(gpu.HmfemError) as e:
            s.solve(b=bb, x=x)   # replaces the solver's right-hand side
    assert e.value.code == gpu.E_BREAKDOWN
    assert "breakdown" in str(e.value)
    # the hierarchy is intact: the next solve converges
    x, st = s.solve(b=b, x=np.zeros(prob.n))
    assert st["status"] == gpu.OK and st["relres"] <= 1e-10
    s.close()


@pytest.mark.parametrize("bad", ["col", "cnt"])
def test_out_of_range_indices_are_rejected(bad):
    cnt, col, ele = _laplace_1d(300)
    if bad == "col":
        col = col.copy()
        col[17] = 300
    else:
        cnt = cnt.copy()
        cnt[0], cnt[1] = 6, -1
    s = gpu.Solver()
    with pytest.raises(gpu.HmfemError) as e:
        s.set_matrix(cnt, col, ele, np.ones(300))
    assert e.value.code == gpu.E_ARG
    with pytest.raises(gpu.HmfemError):
        s.setup()
    s.close()


def test_out_of_range_stencil_index_is_rejected():
    prob = make_problem(5, 4, 3)
    port = Port()
    perm, ind, b = port.assemble(prob)
    ind = ind.copy()
    ind[7, 2] = prob.n + 3
    s = gpu.Solver()
    with pytest.raises(gpu.HmfemError) as e:
        s.set_stencil(prob.nx, prob.ny, prob.nz, perm, ind, b)
    assert e.value.code == gpu.E_ARG
    s.close()


def test_split_wait_that_runs_out_returns_timeout(monkeypatch):
    """The greedy C/F split waits (bounded) on the decisions of lower rows.
    HMFEM_TEST_POLL_LIMIT=0 lets a row give up at its first wait: the kernel
    flags the error, every row leaves, and setup returns HMFEM_E_TIMEOUT.
    With the limit back, the same solver sets up and solves."""
    prob = config_problem(2, size=24)
    port = Port()
    perm, ind, b = port.assemble(prob)
    cnt, col, ele = port.pack(perm, ind)
    s = gpu.Solver(tol=1e-10)
    s.set_matrix(cnt, col, ele, b)          # general matrix: wavefront split
    monkeypatch.setenv("HMFEM_TEST_POLL_LIMIT", "0")
    with pytest.raises(gpu.HmfemError) as e:
        s.setup()
    assert e.value.code == gpu.E_TIMEOUT
    assert "gave up" in str(e.value)
    monkeypatch.delenv("HMFEM_TEST_POLL_LIMIT")
    s.setup()
    x, st = s.solve()
    assert st["status"] == gpu.OK and st["relres"] <= 1e-10
    H = port.amg(cnt, col, ele)  # and the split is the reference's again
    np.testing.assert_array_equal(s.level(0)["sel"], H.level(0)["sel"])
    s.close()
