"""Error against the FP64 oracle at a headline size: 128^3 (config 1, and
the config-2 field at 128^3).  The oracle is the reference algorithm's
AMG-PCG (the C restatement, pinned bit for bit to the reference's own
sources) solved to a true residual of 1e-13.

Both GPU arms -- the plain FP64 drop-in and the chosen FP32 V-cycle (exact
level-0 reduction, BF16 levels >= 1) in FP64 flexible CG -- are solved to
the bench tolerance 1e-10 and to 1e-12.  Bars: at 1e-10, pressures and
the six face fluxes within 1e-8 relative (a solution at residual 1e-10 is
itself ~2e-9 from the tight one on these fields); at 1e-12, within 1e-9.
The divvel_pontual maximum |div u| is the largest row residual, so it
scales with the tolerance: within 1e3 * tol of the flux scale max|v|/h (the
oracle's own solutions reach 1.6-4.3e-8 at 1e-10 and 3-5e-10 at 1e-12)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import config_problem  # noqa: E402
from oracle.oracle import Port  # noqa: E402

FACES = [0, 1, 2, 3, 5, 6]


@pytest.fixture(scope="module", params=[1, 2], ids=["config1_128", "config2_128"])
def oracle_case(request):
    prob = config_problem(request.param, size=128)
    port = Port()
    perm, ind, b = port.assemble(prob)
    cnt, col, ele = port.pack(perm, ind)
    H = port.amg(cnt, col, ele)
    po, it, rel = H.pcg(b, eps=1e-13, stop=1)
    assert rel <= 1e-13
    vo, _, _ = port.fluxes(prob, perm, po)
    return prob, po, vo[:, FACES]


@pytest.mark.parametrize("arm", ["plain_fp64", "fp32_chosen"])
@pytest.mark.parametrize("tol,bar", [(1e-10, 1e-8), (1e-12, 1e-9)])
def test_pressure_and_fluxes_against_the_fp64_oracle(oracle_case, arm, tol, bar):
    prob, po, vo = oracle_case
    opts = dict(precision=1, bf16_from=1, schur0=1) if arm == "fp32_chosen" else {}
    s = gpu.Solver(tol=tol, **opts)
    K = torch.tensor(prob.KX, device="cuda")
    s.assemble(prob, KX=K, KY=K, KZ=K)
    s.setup()
    x = torch.zeros(prob.n, dtype=torch.float64, device="cuda")
    _, st = s.solve(x=x)
    assert st["status"] == gpu.OK and st["relres"] <= tol
    v = torch.zeros((prob.n, 7), dtype=torch.float64, device="cuda")
    _, dmin, dmax = s.fluxes(x, v)
    p = x.cpu().numpy()
    vf = v[:, FACES].cpu().numpy()
    s.close()
    p_rel = np.linalg.norm(p - po) / np.linalg.norm(po)
    f_rel = np.linalg.norm(vf - vo) / np.linalg.norm(vo)
    div_rel = dmax / (np.abs(vo).max() / prob.hx)
    print(f"{prob.name} {arm} tol={tol:g}: iters={st['iterations']} relres={st['relres']:.2e} "
          f"|p-p_o|/|p_o|={p_rel:.2e} |v-v_o|/|v_o|={f_rel:.2e} max|div|/(|v|/h)={div_rel:.2e}")
    assert p_rel <= bar
    assert f_rel <= bar
    assert div_rel <= 1e3 * tol
