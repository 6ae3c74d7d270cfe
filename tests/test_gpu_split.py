"""The greedy C/F split of level 1 (the 19-offset structure of a parity-split
7-point grid), formed by one launch that walks the x-row wavefront with
bounded waits between rows, against the oracle's split of the same level
(node_selection in natural order, amg.h:1-32).

Shapes with x-rows of several 32-cell chunks (nx > 64, and nx > 256 so a row
takes more than one group of four chunks), thin and tall planes, and the
plain FP64 as well as the reduced-precision setup (whose level 1 is the
exact red-black reduction with the same structure).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import make_problem  # noqa: E402

SHAPES = [(6, 4, 5), (130, 7, 5), (258, 4, 9), (64, 33, 3), (96, 5, 40), (520, 4, 4),
          (40, 40, 12)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_level1_split_matches_the_oracle(shape, port):
    nx, ny, nz = shape
    p = make_problem(nx, ny, nz, log10k=(-14.0, 1.0, 1.5), seed=nx + ny + nz)
    perm, ind, b = port.assemble(p)
    H = port.amg(*port.pack(perm, ind))
    for precision, schur0 in ((0, 0), (1, 1)):
        s = gpu.Solver(precision=precision, schur0=schur0)
        s.assemble(p)
        s.setup()
        g = s.level(1)
        assert g["n"] == H.level(1)["n"]
        np.testing.assert_array_equal(g["sel"], H.level(1)["sel"],
                                      err_msg=f"precision {precision}")
        s.close()


def test_level1_split_wait_that_runs_out_returns_timeout(monkeypatch, port):
    """HMFEM_TEST_POLL_LIMIT=0 lets an x-row give up at its first wait for
    the rows below it: the kernel flags the error, every warp leaves, and
    setup returns HMFEM_E_TIMEOUT.  With the limit back, the same solver
    sets up, its split is the oracle's and it solves."""
    p = make_problem(48, 40, 24, log10k=(-14.0, 1.0, 1.5), seed=5)
    s = gpu.Solver(tol=1e-10)
    s.assemble(p)                         # assembled grid: the wavefront split
    monkeypatch.setenv("HMFEM_TEST_POLL_LIMIT", "0")
    with pytest.raises(gpu.HmfemError) as e:
        s.setup()
    assert e.value.code == gpu.E_TIMEOUT
    assert "gave up" in str(e.value)
    monkeypatch.delenv("HMFEM_TEST_POLL_LIMIT")
    s.setup()
    x, st = s.solve()
    assert st["status"] == gpu.OK and st["relres"] <= 1e-10
    perm, ind, b = port.assemble(p)
    H = port.amg(*port.pack(perm, ind))
    np.testing.assert_array_equal(s.level(1)["sel"], H.level(1)["sel"])
    s.close()
