"""The coarse tail of the V-cycle (k_tail: every small Chebyshev level and
the coarse solve in one cluster launch) against the same cycle launched
level by level (HMFEM_TAIL=0, in a separate process): bit-identical
solutions and iteration counts, both precisions.  The per-level path itself
is pinned to the oracle by the V-cycle parity tests."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")

CHILD = r"""
import sys, json
sys.path.insert(0, {root!r})
import numpy as np
from hmfem_b200 import gpu
from hmfem_b200.problem import config_problem
out = {{}}
for cfg, size in ((2, 40), (1, 48)):
    p = config_problem(cfg, size=size)
    for prec in (0, 1):
        s = gpu.Solver(precision=prec, tol=1e-10, bf16_from=1 if prec else -1, schur0=prec)
        s.assemble(p); s.setup()
        x, st = s.solve()
        u = s.vcycle(np.linspace(0.0, 1.0, p.n))
        names = [r["kernel"] for r in s.profile_iteration(1)]
        out[f"{{cfg}}_{{prec}}"] = dict(x=x.tobytes().hex(), u=u.tobytes().hex(),
                                        it=st["iterations"],
                                        tail=any("k_tail" in k for k in names))
        s.close()
print(json.dumps(out))
"""


def _run(tail):
    env = dict(os.environ, HMFEM_TAIL=str(tail))
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], capture_output=True,
                       text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tail_launch_is_bit_identical_to_per_level_launches():
    a, b = _run(1), _run(0)
    for key in a:
        assert a[key]["tail"] and not b[key]["tail"], key
        assert a[key]["it"] == b[key]["it"], key
        assert a[key]["u"] == b[key]["u"], key     # one V-cycle, bit for bit
        assert a[key]["x"] == b[key]["x"], key     # whole solve, bit for bit
