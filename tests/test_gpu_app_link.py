"""The drop-in claim, end to end: the reference application's unmodified
sources (reservoir.c, permeabilities.c, set_boundaries.c,
set_source_term.c, solve_linearsystem_AMG.c, create_variables.c), built by
tests/link/Makefile and linked against libhmfem_gpu.so in place of
compute.cpp, run reservoir() (reservoir.c:8-57) -> solve_linsys
(solve_linearsystem_AMG.c:37-157) -> compute() on the GPU.

The pressure must agree with the oracle's (the reference algorithm solved
tightly) within 1e-6 relative at the reference's own stopping rule
(compute.cpp:41: preconditioned residual 1e-8), and the application's
iter_amg (variables.h:63, defined in the executable) must be set by the
library.
"""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200.problem import config_problem  # noqa: E402
from oracle.oracle import Port  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
APP = os.path.join(HERE, "link", "_build", "app_link")


@pytest.mark.skipif(not os.path.exists(APP), reason="app_link not built (needs the hmfem tree)")
@pytest.mark.parametrize("size", [16, 20])
def test_unmodified_application_solves_through_the_gpu_library(tmp_path, size):
    prob = config_problem(1, size=size)   # background 1e-14 + conduits at 1e-10
    kfile, pfile = tmp_path / "K.bin", tmp_path / "p.bin"
    prob.KX.astype(np.float64).tofile(kfile)
    env = dict(os.environ)
    env.pop("HMFEM_TOL", None)
    env.pop("HMFEM_STOP", None)
    out = subprocess.run([APP, str(prob.nx), str(prob.ny), str(prob.nz), str(kfile),
                          str(pfile)], capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 0, out.stderr
    iters = int(out.stdout.split("iter_amg")[1].split()[0])
    assert iters > 0
    p = np.fromfile(pfile, dtype=np.float64)
    port = Port()
    perm, ind, b = port.assemble(prob)
    cnt, col, ele = port.pack(perm, ind)
    H = port.amg(cnt, col, ele)
    po, _, rel = H.pcg(b, eps=1e-12, stop=1)   # true residual <= 1e-12
    err = np.linalg.norm(p - po) / np.linalg.norm(po)
    print(f"{size}^3: iter_amg={iters} |p - p_oracle|/|p_oracle| = {err:.2e}")
    assert err <= 1e-6
