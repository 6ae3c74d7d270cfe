"""The learned guess's tcgen05 convolution kernels against torch's conv3d in
float64 on the CPU (the reference for these kernels; inputs rounded to BF16
first, as the kernels see them)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import torch.nn.functional as F  # noqa: E402

from hmfem_b200 import guess  # noqa: E402

DIMS = [(9, 7, 5), (20, 16, 12)]
# x rows of 128 cells and more: row mode (one MMA run per x row, x tiles,
# the last ragged) or plane mode over the whole x extent, as the planner picks
ROW_DIMS = [(130, 5, 3), (128, 4, 5), (256, 3, 2)]
SHAPES = [(16, 16), (16, 32), (32, 64), (64, 64), (96, 32), (48, 16), (32, 96)]


def _to_ncdhw(x, dims):
    nx, ny, nz = dims
    return x.view(nz, ny, nx, -1).permute(3, 0, 1, 2)[None]


def _from_ncdhw(t):
    c = t.shape[1]
    return t[0].permute(1, 2, 3, 0).reshape(-1, c)


def _w_torch(w):  # (27, cout, cin) -> (cout, cin, kz, ky, kx)
    return w.view(3, 3, 3, w.shape[1], w.shape[2]).permute(3, 4, 0, 1, 2)


def _fwd(x, w, b, dims, relu):
    """The kernel on channels-last (n, C) tensors (it takes channel-blocked ones)."""
    out = guess.conv3d_raw(guess.blocked(x.cuda()), w.cuda(),
                           None if b is None else b.cuda(), dims, relu)
    return guess.unblocked(out).cpu().double()


def _rel(a, b):
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


@pytest.mark.parametrize("dims", DIMS + ROW_DIMS)
@pytest.mark.parametrize("cin,cout", SHAPES)
def test_forward_matches_conv3d(cin, cout, dims):
    g = torch.Generator().manual_seed(cin * 100 + cout)
    n = dims[0] * dims[1] * dims[2]
    x = torch.randn(n, cin, generator=g).bfloat16()
    w = (torch.randn(27, cout, cin, generator=g) * 0.1).bfloat16()
    b = torch.randn(cout, generator=g)
    ours = _fwd(x, w, b, dims, False)
    ref = _from_ncdhw(F.conv3d(_to_ncdhw(x.double(), dims), _w_torch(w.double()),
                               b.double(), padding=1))
    assert _rel(ours, ref) < 6e-3   # BF16 output rounding
    relu = _fwd(x, w, b, dims, True)
    assert _rel(relu, ref.clamp(min=0)) < 6e-3
    guess.check_errors()


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("cin,cout", SHAPES)
def test_weight_gradient_matches_conv3d(cin, cout, dims):
    g = torch.Generator().manual_seed(cin * 7 + cout)
    n = dims[0] * dims[1] * dims[2]
    x = torch.randn(n, cin, generator=g).bfloat16()
    dy = torch.randn(n, cout, generator=g).bfloat16()
    ours = guess.conv3d_wgrad_raw(guess.blocked(x.cuda()), guess.blocked(dy.cuda()),
                                  dims).cpu().double()
    ref = torch.nn.grad.conv3d_weight(_to_ncdhw(x.double(), dims), (cout, cin, 3, 3, 3),
                                      _to_ncdhw(dy.double(), dims), padding=1)
    ref = ref.permute(2, 3, 4, 0, 1).reshape(27, cout, cin)
    assert _rel(ours, ref) < 1e-5   # exact BF16 products, FP32 sums
    guess.check_errors()


@pytest.mark.parametrize("cin,cout", [(16, 32), (64, 64), (32, 96)])
def test_data_gradient_is_flipped_forward(cin, cout):
    dims = (11, 6, 7)
    g = torch.Generator().manual_seed(5)
    n = dims[0] * dims[1] * dims[2]
    w = (torch.randn(27, cout, cin, generator=g) * 0.1).bfloat16()
    dy = torch.randn(n, cout, generator=g).bfloat16()
    ours = _fwd(dy, guess.flip_transpose(w), None, dims, False)
    ref = torch.nn.grad.conv3d_input((1, cin, dims[2], dims[1], dims[0]), _w_torch(w.double()),
                                     _to_ncdhw(dy.double(), dims), padding=1)
    assert _rel(ours, _from_ncdhw(ref)) < 6e-3


@pytest.mark.parametrize("cin,cout", [(48, 16), (32, 16)])
def test_wide_plane_grouped_forward(cin, cout):
    """A 256-wide grid the planner tiles in plane mode with grouped x taps
    (the form 48 -> 16 takes at 256^3): against torch's conv3d."""
    dims = (256, 6, 16)
    p = guess.conv_plan(dims, cin, cout)
    assert p["row_mode"] == 0 and p["xg"] == 1 and p["bx"] == 256
    g = torch.Generator().manual_seed(cin + 7)
    n = dims[0] * dims[1] * dims[2]
    x = torch.randn(n, cin, generator=g).bfloat16()
    w = (torch.randn(27, cout, cin, generator=g) * 0.1).bfloat16()
    b = torch.randn(cout, generator=g)
    ours = _fwd(x, w, b, dims, False)
    ref = _from_ncdhw(F.conv3d(_to_ncdhw(x.double(), dims), _w_torch(w.double()),
                               b.double(), padding=1))
    assert _rel(ours, ref) < 6e-3
    guess.check_errors()
