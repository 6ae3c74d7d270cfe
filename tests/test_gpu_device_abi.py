"""The reference's device layer: all fifteen ``_device_*`` entry points of
toolbox/lib/toolbox.cu, called through the C-ABI on device data and checked
against the reference's formulas (bit for bit, FP64 without contraction)
and, for the sparse ones, against the oracle's CSR product.

The SELL-32 operands are laid out exactly as device_matrix_conversion
builds them (toolbox/inverse_operator/device_amg.h:60-126, the ``#if 1``
branch): ``tdsp`` = the CSR row offsets (bucket_sort_offset, an exclusive
prefix sum, toolbox/vector/sort.h:415-428); ``dsp[i]`` counts rows one by
one and, at the start of every slice of L = 32 rows (toolbox/toolbox.h:67),
skips L times the previous slice's longest row; element k of row i sits at
``dsp[i] + L*k``.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from hmfem_b200 import gpu  # noqa: E402
from hmfem_b200.problem import config_problem, make_problem  # noqa: E402
from oracle.oracle import Port  # noqa: E402

L_SLICE = 32
vp, ui, dd, ii = C.c_void_p, C.c_uint, C.c_double, C.c_int


def _lib():
    L = gpu.lib()
    for name in ("_device_add_scale", "_device_sub_scale", "_device_scale_add"):
        getattr(L, name).argtypes = [vp, vp, dd, ui]
    L._device_vector_product.argtypes = [vp, vp, vp, ui, ui]
    L._device_linear_operator.argtypes = [vp, vp, vp, vp, ii, ii, ii, vp, vp]
    L._device_jacobi.argtypes = [vp, vp, vp, vp, ii, ii, vp, vp, vp]
    L._device_set_mul.argtypes = [vp, vp, vp, dd, ui]
    L._device_add_mul.argtypes = [vp, vp, vp, dd, ui]
    L._device_diagonal_solver.argtypes = [vp, vp, vp, ui]
    L._device_com_snd.argtypes = [vp, vp, vp, ui]
    L._device_com_rcv.argtypes = [vp, vp, vp, ui]
    for name in ("_device_sub", "_device_add", "_device_rsb"):
        getattr(L, name).argtypes = [vp, vp, ui]
    L._device_matrix_conversion.argtypes = [vp, vp, vp, vp, vp, vp, vp, ii]
    return L


def _d(a):
    return torch.tensor(np.ascontiguousarray(a), device="cuda")


def _p(t):
    return t.data_ptr()


def sell_layout(cnt):
    """dsp and the padded size m of device_matrix_conversion
    (device_amg.h:72-83)."""
    n = len(cnt)
    dsp = np.zeros(n, np.int32)
    m = mx = 0
    for i in range(n):
        if i % L_SLICE == 0:
            m += mx * L_SLICE
            mx = 0
        dsp[i] = m
        m += 1
        mx = max(mx, int(cnt[i]))
    m += mx * L_SLICE
    return dsp, m


def to_sell(cnt, col, ele):
    """Host build of the SELL-32 arrays (the layout of device_amg.h:72-91):
    the arrays _device_matrix_conversion must produce."""
    dsp, m = sell_layout(cnt)
    tdsp = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.int32)
    acol = np.full(m, -7, np.int32)
    aele = np.full(m, np.nan)
    used = np.zeros(m, bool)
    for i in range(len(cnt)):
        k = dsp[i] + L_SLICE * np.arange(cnt[i])
        acol[k] = col[tdsp[i]:tdsp[i] + cnt[i]]
        aele[k] = ele[tdsp[i]:tdsp[i] + cnt[i]]
        used[k] = True
    return dsp, tdsp, m, acol, aele, used


@pytest.fixture(scope="module")
def levels():
    """CSR levels 0 and 1 of the oracle's hierarchy (7-point rows in the
    reference's d,l,c,r,u,t,b order; column-sorted Galerkin rows) and a
    ragged one-row-per-slice-boundary case."""
    port = Port()
    out = []
    for prob in (config_problem(1, size=24),
                 make_problem(5, 3, 7, log10k=(-14.0, 1.0, 1.5), n_conduits=1, seed=9)):
        perm, ind, _ = port.assemble(prob)
        cnt, col, ele = port.pack(perm, ind)
        H = port.amg(cnt, col, ele)
        out.append((cnt, col, ele))
        lv = H.level(1)
        out.append((lv["cnt"], lv["col"], lv["ele"]))
    return port, out


def test_matrix_conversion_builds_the_reference_sell32_layout(levels):
    L = _lib()
    _, mats = levels
    for cnt, col, ele in mats:
        dsp, tdsp, m, acol_h, aele_h, used = to_sell(cnt, col, ele)
        acol = torch.full((m,), -7, dtype=torch.int32, device="cuda")
        aele = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
        dc, dds, dtd, dtc, dte = _d(cnt), _d(dsp), _d(tdsp), _d(col), _d(ele)
        L._device_matrix_conversion(_p(dc), _p(dds), _p(acol), _p(aele), _p(dtd),
                                    _p(dtc), _p(dte), len(cnt))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(acol.cpu().numpy(), acol_h)
        g = aele.cpu().numpy()
        np.testing.assert_array_equal(g[used], aele_h[used])
        assert np.all(np.isnan(g[~used]))  # padding is left alone


def test_sell32_linear_operator_and_jacobi_match_the_oracle(levels):
    L = _lib()
    port, mats = levels
    rng = np.random.default_rng(11)
    for cnt, col, ele in mats:
        n = len(cnt)
        dsp, tdsp, m, acol_h, aele_h, used = to_sell(cnt, col, ele)
        aele_h[~used] = 0.0
        acol_h[~used] = 0
        u = rng.standard_normal(n)
        f = rng.standard_normal(n)
        dc, dds, dac, dae = _d(cnt), _d(dsp), _d(acol_h), _d(aele_h)
        du, df = _d(u), _d(f)
        v = torch.zeros(n, dtype=torch.float64, device="cuda")
        # l = SELL size, m = length of u, n = rows (toolbox.cu:221)
        L._device_linear_operator(_p(dc), _p(dds), _p(dac), _p(dae), m, n, n, _p(du), _p(v))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(v.cpu().numpy(), port.spmv(cnt, col, ele, u))
        # jacobi residual v = f - A u, subtracting row entries in order
        # (toolbox.cu:269-281)
        r = f.copy()
        for k in range(int(cnt.max())):
            on = cnt > k
            idx = tdsp[on] + k
            r[on] = r[on] - ele[idx] * u[col[idx]]
        L._device_jacobi(_p(dc), _p(dds), _p(dac), _p(dae), m, n, _p(df), _p(du), _p(v))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(v.cpu().numpy(), r)


def test_device_jacobi_smoother_steps(levels):
    """device_jacobi (device_amg.h:26-42): the pre-smoother from zero
    (u = w D^-1 f, r = f - A u) and a smoothing step (v = f - A u,
    u += w v D^-1), composed from the entry points as the class does."""
    L = _lib()
    _, mats = levels
    cnt, col, ele = mats[0]
    n = len(cnt)
    dsp, tdsp, m, acol_h, aele_h, used = to_sell(cnt, col, ele)
    aele_h[~used] = 0.0
    acol_h[~used] = 0
    diag = np.array([ele[tdsp[i]:tdsp[i] + cnt[i]][col[tdsp[i]:tdsp[i] + cnt[i]] == i][0]
                     for i in range(n)])
    dia = 1.0 / diag
    w = 0.8
    f = np.random.default_rng(2).standard_normal(n)
    dc, dds, dac, dae, ddia, df = (_d(a) for a in (cnt, dsp, acol_h, aele_h, dia, f))
    du = torch.zeros(n, dtype=torch.float64, device="cuda")
    dr = torch.zeros(n, dtype=torch.float64, device="cuda")
    L._device_set_mul(_p(du), _p(df), _p(ddia), w, n)
    L._device_jacobi(_p(dc), _p(dds), _p(dac), _p(dae), m, n, _p(df), _p(du), _p(dr))
    torch.cuda.synchronize()
    u = (w * f) * dia
    np.testing.assert_array_equal(du.cpu().numpy(), u)

    def resid(u):
        r = f.copy()
        for k in range(int(cnt.max())):
            on = cnt > k
            idx = tdsp[on] + k
            r[on] = r[on] - ele[idx] * u[col[idx]]
        return r
    np.testing.assert_array_equal(dr.cpu().numpy(), resid(u))
    dv = torch.zeros(n, dtype=torch.float64, device="cuda")
    L._device_jacobi(_p(dc), _p(dds), _p(dac), _p(dae), m, n, _p(df), _p(du), _p(dv))
    L._device_add_mul(_p(du), _p(dv), _p(ddia), w, n)
    torch.cuda.synchronize()
    v = resid(u)
    np.testing.assert_array_equal(du.cpu().numpy(), u + (w * v) * dia)


def test_vector_entry_points_match_reference_formulas():
    """toolbox.cu:12-63 (add/sub/scale), :356-435 (set_mul, add_mul,
    diagonal solver), :513-583 (sub, add, rsb): same operations in the same
    order, FP64 without contraction."""
    L = _lib()
    rng = np.random.default_rng(7)
    for n in (1, 31, 1000, 70001):
        x, y, z = (rng.standard_normal(n) for _ in range(3))
        s = float(rng.standard_normal())

        def run(name, *args):
            dev = [_d(a) for a in args[:-1]] if isinstance(args[-1], float) else [
                _d(a) for a in args]
            extra = [args[-1]] if isinstance(args[-1], float) else []
            getattr(L, name)(*[_p(t) for t in dev], *extra, n)
            torch.cuda.synchronize()
            return [t.cpu().numpy() for t in dev]

        np.testing.assert_array_equal(run("_device_add_scale", x, y, s)[0], x + y * s)
        np.testing.assert_array_equal(run("_device_sub_scale", x, y, s)[0], x - y * s)
        np.testing.assert_array_equal(run("_device_scale_add", x, y, s)[0], x * s + y)
        np.testing.assert_array_equal(run("_device_set_mul", x, y, z, s)[0], s * y * z)
        np.testing.assert_array_equal(run("_device_add_mul", x, y, z, s)[0], x + s * y * z)
        np.testing.assert_array_equal(run("_device_diagonal_solver", x, y, z)[0], y * z)
        np.testing.assert_array_equal(run("_device_sub", x, y)[1], y - x)
        np.testing.assert_array_equal(run("_device_add", x, y)[1], y + x)
        np.testing.assert_array_equal(run("_device_rsb", x, y)[1], x - y)
        # per-block partial products; the caller sums the m partials
        # (device_binary_operator.h:29-49)
        for m in (1, 7, 64):
            w = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
            dx, dy = _d(x), _d(y)
            L._device_vector_product(_p(dx), _p(dy), _p(w), n, m)
            torch.cuda.synchronize()
            assert not torch.isnan(w).any()
            assert w.sum().item() == pytest.approx(float(x @ y), rel=1e-12, abs=1e-12)


def test_communicator_gather_and_scatter_add():
    """_device_com_snd / _device_com_rcv (toolbox.cu:443-506): gather the
    send list, scatter-add the receive list (several entries may hit one
    index, the adds are atomic)."""
    L = _lib()
    rng = np.random.default_rng(3)
    n, k = 5000, 3001
    x = rng.standard_normal(n)
    rcom = rng.integers(0, n, k).astype(np.int32)
    dx, dr = _d(x), _d(rcom)
    sv = torch.zeros(k, dtype=torch.float64, device="cuda")
    L._device_com_snd(_p(dx), _p(sv), _p(dr), k)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sv.cpu().numpy(), x[rcom])
    rv = rng.standard_normal(k)
    drv = _d(rv)
    L._device_com_rcv(_p(dx), _p(drv), _p(dr), k)
    torch.cuda.synchronize()
    want = x.copy()
    np.add.at(want, rcom, rv)
    np.testing.assert_allclose(dx.cpu().numpy(), want, rtol=1e-13, atol=1e-13)
    # distinct targets: one add per entry, bit-exact
    uniq = rng.permutation(n)[:k].astype(np.int32)
    dx, du = _d(x), _d(uniq)
    L._device_com_rcv(_p(dx), _p(drv), _p(du), k)
    torch.cuda.synchronize()
    want = x.copy()
    want[uniq] += rv
    np.testing.assert_array_equal(dx.cpu().numpy(), want)


def test_zero_sizes_launch_nothing():
    L = _lib()
    c0 = gpu.launch_count()
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    L._device_add_scale(_p(z), _p(z), 1.0, 0)
    L._device_rsb(_p(z), _p(z), 0)
    L._device_matrix_conversion(*([_p(z)] * 7), 0)
    L._device_linear_operator(*([_p(z)] * 4), 0, 0, 0, _p(z), _p(z))
    torch.cuda.synchronize()
    assert gpu.launch_count() == c0
    L._device_add_scale(_p(z), _p(z), 1.0, 1)   # one launch, counted once
    torch.cuda.synchronize()
    assert gpu.launch_count() == c0 + 1
