"""The timed reference arm of bench.py on the host: the reference's own
path (oracle/_ref) split into steps gives ref_solve_all's result bit for
bit, every step plan is one complete solve, and `--impl reference` prints
one JSON line on the bench's own configuration."""
import io
import json
import os
import sys
from contextlib import redirect_stdout
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")
sys.path.insert(0, ROOT)

from hmfem_b200.problem import config_problem  # noqa: E402
from oracle.oracle import REF_SO  # noqa: E402

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("steps", [1, 2, 3, 4, 7])
def test_stepped_reference_job_equals_the_whole_path(steps):
    import bench
    from oracle.oracle import Ref
    p = config_problem(2, size=20)
    R = Ref()
    with bench._QuietStdout():
        x, v, it, rel, _ = R.solve_all(p, eps=1e-10)
    job = R.job(p, eps=1e-10)
    for part in bench.ref_plan(steps, est_iters=12):
        for op in part:
            if op == "assemble":
                job.assemble()
            elif op == "setup":
                job.setup()
            else:
                job.iterate(op[1])
    vj = np.zeros((p.n, 7))
    with bench._QuietStdout():
        job.flux(vj)
    xj, itj, relj, _ = job.result()
    job.close()
    np.testing.assert_array_equal(xj, x)
    np.testing.assert_array_equal(vj, v)
    assert relj == rel <= 1e-10
    assert itj == it - 1   # compute()'s count is loop bodies + 1 (pcg.h:57)


def test_every_plan_is_one_complete_solve():
    import bench
    for steps in range(1, 30):
        plan = bench.ref_plan(steps)
        assert len(plan) == steps
        ops = [op for part in plan for op in part]
        assert ops[0] == "assemble" and ops[1] == "setup"
        assert ops[-1] == ("iterate", -1)        # runs to the tolerance
        assert all(isinstance(op, tuple) for op in ops[2:])


@needs_ref
def test_reference_arm_prints_one_line_on_the_bench_configuration():
    import bench
    args = SimpleNamespace(size=16, steps=4, warmup=1, tol=1e-10)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    lines = [ln for ln in buf.getvalue().splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 4 and d["warmup"] == 1
    assert d["config"]["workload"] == "config2 16^3 lognormal+8 conduits"
    assert d["value"] > 0 and d["cpu_baseline"]["max_relres"] <= 1e-10
    assert d["e2e"]["value"] == d["value"]


def test_kernel_byte_models_of_the_level0_kernels():
    """The bench's algorithmic bytes of the CG's pair SpMV and of the
    level-0 prolongation that also forms the CG's dots, from their
    demangled names."""
    import bench
    n0 = 1000
    info = [(n0, 7 * n0, 0), (n0 // 2, 19 * n0 // 2, n0)]
    assert bench.kernel_bytes("void (anonymous namespace)::k_g7_spmv_dot2<true>(...)", -1,
                              info, 1) == 48 * n0
    assert bench.kernel_bytes("void (anonymous namespace)::k_g7_sprol2_zd<float, float>(...)",
                              0, info, 1) == 38 * n0
