"""The learned initial guess: a 3-level 3-D U-Net (16/32/64 channels, 3x3x3
kernels) that maps log K, the conduit mask and the Dirichlet mask of a grid
to a pressure guess for the CG.  No counterpart in the reference.

Every 3x3x3 convolution -- forward, data gradient and weight gradient --
runs on this library's tcgen05 tensor-core kernels (`hmfem_conv3d_fwd`,
`hmfem_conv3d_wgrad`: BF16 operands, FP32 accumulation), and so do the
features, the 2x average pooling and the nearest upsampling fused with the
skip concatenation (`hmfem_guess_*`, one HBM pass each) and, at inference,
the 1x1 head fused with the linear profile.  PyTorch is the training driver
around them: autograd bookkeeping, the head while training and the Adam
update of the FP32 master weights.

Activations are channel-blocked: a grid of n = nx*ny*nz cells with C
channels is a (C/8, n, 8) BF16 tensor -- slab k holds channels 8k..8k+7 of
every cell, cell s = x + nx (y + ny z) -- so a halo row of one slab is
contiguous for the kernels' bulk copies, channel concatenation is
concatenation of slabs, and pooling and upsampling are views over the
cells.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import gpu

CH = (16, 32, 64)
IN_CH = 16          # 3 input features, zero-padded to the kernels' K step
_SHAPES = {(16, 16), (16, 32), (32, 16), (32, 32), (32, 64), (64, 32), (64, 64),
           (96, 32), (32, 96), (48, 16), (16, 48)}


def _lib():
    L = gpu.lib()
    if not getattr(L, "_guess_bound", False):
        vp, i = C.c_void_p, C.c_int
        L.hmfem_conv3d_fwd.argtypes = [vp, vp, vp, vp, i, i, i, i, i, i, vp, vp]
        L.hmfem_conv3d_wgrad.argtypes = [vp, vp, vp, i, i, i, i, i, vp, vp]
        L.hmfem_conv3d_plan.argtypes = [i, i, i, i, i, i, i, vp]
        L.hmfem_guess_features.argtypes = [vp, vp, i, i, i, vp, vp]
        L.hmfem_guess_pool2.argtypes = [vp, i, i, i, i, vp, vp]
        L.hmfem_guess_up2_cat.argtypes = [vp, i, vp, i, i, i, i, vp, vp]
        L.hmfem_guess_up2_grad.argtypes = [vp, i, i, i, i, vp, vp]
        L.hmfem_guess_head_profile.argtypes = [vp, i, vp, vp, i, i, i, vp, vp]
        L._guess_bound = True
    return L


PLAN_FIELDS = ("bx", "by", "bz", "W", "H", "hc", "hcp", "runs", "rp", "row_mode",
               "ntx", "nty", "ntz", "ns", "nb", "wres", "tmem_cols", "stage_bytes",
               "wbytes", "smem_bytes", "xg")


def conv_plan(dims, cin, cout, nsm=148, smem_max=232448):
    """The tiling `hmfem_conv3d_fwd` launches for this grid (host only)."""
    out = (C.c_int * len(PLAN_FIELDS))()
    rc = _lib().hmfem_conv3d_plan(dims[0], dims[1], dims[2], cin, cout, nsm, smem_max,
                                  C.addressof(out))
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())
    return dict(zip(PLAN_FIELDS, list(out)))


_ERR = {}


def _err_buf(dev):
    if dev not in _ERR:
        _ERR[dev] = torch.zeros(1, dtype=torch.int32, device=dev)
    return _ERR[dev]


def check_errors(dev=None):
    """Raises if a tensor-core kernel reported a timed-out wait."""
    dev = dev or torch.device("cuda", torch.cuda.current_device())
    e = _err_buf(dev)
    if int(e.item()) != 0:
        e.zero_()
        raise RuntimeError("conv3d: a bounded tensor-core wait gave up")


def blocked(x):
    """(n, C) channels-last -> (C/8, n, 8) channel-blocked."""
    n, c = x.shape
    return x.reshape(n, c // 8, 8).permute(1, 0, 2).contiguous()


def unblocked(x):
    """(C/8, n, 8) channel-blocked -> (n, C) channels-last."""
    s, n, _ = x.shape
    return x.permute(1, 0, 2).reshape(n, 8 * s)


def conv3d_raw(x, w, bias, dims, relu):
    """out = relu?(conv(x, w) + bias): x (cin/8, n, 8) bf16, w (27, cout, cin)
    bf16; out (cout/8, n, 8)."""
    nx, ny, nz = dims
    n, cin = x.shape[1], 8 * x.shape[0]
    cout = w.shape[1]
    assert (cin, cout) in _SHAPES, (cin, cout)
    assert x.dtype == torch.bfloat16 and w.dtype == torch.bfloat16
    x = x.contiguous()
    w = w.contiguous()
    out = torch.empty(cout // 8, n, 8, dtype=torch.bfloat16, device=x.device)
    st = torch.cuda.current_stream(x.device).cuda_stream
    rc = _lib().hmfem_conv3d_fwd(x.data_ptr(), w.data_ptr(),
                                 bias.data_ptr() if bias is not None else None,
                                 out.data_ptr(), nx, ny, nz, cin, cout, int(relu),
                                 _err_buf(x.device).data_ptr(), st)
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())
    return out


def conv3d_wgrad_raw(x, dy, dims):
    """dw (27, cout, cin) fp32 = sum over cells dy[cell][co] x[cell + tap][ci];
    x (cin/8, n, 8), dy (cout/8, n, 8)."""
    nx, ny, nz = dims
    cin, cout = 8 * x.shape[0], 8 * dy.shape[0]
    dw = torch.zeros(27, cout, cin, dtype=torch.float32, device=x.device)
    st = torch.cuda.current_stream(x.device).cuda_stream
    rc = _lib().hmfem_conv3d_wgrad(x.contiguous().data_ptr(), dy.contiguous().data_ptr(),
                                   dw.data_ptr(), nx, ny, nz, cin, cout,
                                   _err_buf(x.device).data_ptr(), st)
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())
    return dw


def flip_transpose(w):
    """Weights of the data gradient: w_t[t][ci][co] = w[26 - t][co][ci]."""
    return w.flip(0).transpose(1, 2).contiguous()


class Conv3x3x3(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w, bias, dims, relu):
        wb = w.to(torch.bfloat16)
        out = conv3d_raw(x, wb, bias, dims, relu)
        ctx.save_for_backward(x, wb, out)
        ctx.dims, ctx.relu = dims, relu
        return out

    @staticmethod
    def backward(ctx, gout):
        x, wb, out = ctx.saved_tensors
        g = gout.to(torch.bfloat16)
        if ctx.relu:
            g = g * (out > 0).to(g.dtype)
        gx = conv3d_raw(g, flip_transpose(wb), None, ctx.dims, False)
        gw = conv3d_wgrad_raw(x, g, ctx.dims)
        gb = g.float().sum(1).reshape(-1)
        return gx, gw, gb, None, None


def conv(x, w, b, dims, relu=True):
    return Conv3x3x3.apply(x, w, b, dims, relu)


# ---- grid data movement (channel-blocked, dims (nx, ny, nz)) ---------------

def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


def _rc(rc):
    if rc != 0:
        raise gpu.HmfemError(rc, gpu.last_error())


class _Pool2(torch.autograd.Function):
    """2x2x2 average pooling; the gradient spreads 1/8 to each fine cell."""

    @staticmethod
    def forward(ctx, x, dims):
        nx, ny, nz = dims
        x = x.contiguous()
        out = torch.empty(x.shape[0], x.shape[1] // 8, 8, dtype=x.dtype, device=x.device)
        _rc(_lib().hmfem_guess_pool2(x.data_ptr(), x.shape[0], nx, ny, nz, out.data_ptr(),
                                     _stream(x)))
        ctx.dims = dims
        return out

    @staticmethod
    def backward(ctx, g):
        nx, ny, nz = ctx.dims
        g = g.contiguous()
        out = torch.empty(g.shape[0], 8 * g.shape[1], 8, dtype=g.dtype, device=g.device)
        _rc(_lib().hmfem_guess_up2_cat(g.data_ptr(), g.shape[0], None, 0, nx, ny, nz,
                                       out.data_ptr(), _stream(g)))
        return out * 0.125, None


class _Up2Cat(torch.autograd.Function):
    """[nearest-upsampled coarse | skip] on the fine grid; the coarse
    gradient sums the 8 fine cells', the skip's is its slabs."""

    @staticmethod
    def forward(ctx, coarse, skip, dims):
        nx, ny, nz = dims
        coarse, skip = coarse.contiguous(), skip.contiguous()
        sa, sb = coarse.shape[0], skip.shape[0]
        out = torch.empty(sa + sb, skip.shape[1], 8, dtype=skip.dtype, device=skip.device)
        _rc(_lib().hmfem_guess_up2_cat(coarse.data_ptr(), sa, skip.data_ptr(), sb, nx, ny, nz,
                                       out.data_ptr(), _stream(skip)))
        ctx.dims, ctx.sa = dims, sa
        return out

    @staticmethod
    def backward(ctx, g):
        nx, ny, nz = ctx.dims
        g = g.contiguous()
        ga = torch.empty(ctx.sa, g.shape[1] // 8, 8, dtype=g.dtype, device=g.device)
        _rc(_lib().hmfem_guess_up2_grad(g.data_ptr(), ctx.sa, nx, ny, nz, ga.data_ptr(),
                                        _stream(g)))
        return ga, g[ctx.sa:], None


def pool2(x, dims):
    nx, ny, nz = dims
    return _Pool2.apply(x, dims), (nx // 2, ny // 2, nz // 2)


def up2_cat(coarse, skip, dims):
    """Upsample `coarse` to the fine grid `dims` and append `skip`'s slabs."""
    return _Up2Cat.apply(coarse, skip, dims)


class UNet(torch.nn.Module):
    """enc 16 -> pool -> enc 32 -> pool -> 64 -> up + skip -> 32 -> up + skip
    -> 16 -> 1x1 head; two 3x3x3 convolutions (ReLU) per stage."""

    SPEC = [("e0a", IN_CH, 16), ("e0b", 16, 16), ("e1a", 16, 32), ("e1b", 32, 32),
            ("bna", 32, 64), ("bnb", 64, 64), ("d1a", 96, 32), ("d1b", 32, 32),
            ("d0a", 48, 16), ("d0b", 16, 16)]

    def __init__(self, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.w = torch.nn.ParameterDict()
        self.b = torch.nn.ParameterDict()
        for name, cin, cout in self.SPEC:
            std = math.sqrt(2.0 / (27 * cin))
            self.w[name] = torch.nn.Parameter(torch.randn(27, cout, cin, generator=g) * std)
            self.b[name] = torch.nn.Parameter(torch.zeros(cout))
        self.head = torch.nn.Parameter(torch.randn(16, generator=g) * 0.01)
        self.head_b = torch.nn.Parameter(torch.zeros(1))

    def n_params(self):
        return sum(p.numel() for p in self.parameters())

    def trunk(self, feats, dims):
        """feats (IN_CH/8, n, 8) bf16 -> the last activation (2, n, 8) bf16."""
        def block(x, a, b_, d):
            x = conv(x, self.w[a], self.b[a], d)
            return conv(x, self.w[b_], self.b[b_], d)
        d0 = dims
        e0 = block(feats, "e0a", "e0b", d0)
        x, d1 = pool2(e0, d0)
        e1 = block(x, "e1a", "e1b", d1)
        x, d2 = pool2(e1, d1)
        x = block(x, "bna", "bnb", d2)
        x = block(up2_cat(x, e1, d1), "d1a", "d1b", d1)
        return block(up2_cat(x, e0, d0), "d0a", "d0b", d0)

    def forward(self, feats, dims):
        """feats (IN_CH/8, n, 8) bf16 -> (n,) fp32 pressure correction."""
        x = self.trunk(feats, dims)
        return torch.einsum("snc,sc->n", x.float(), self.head.view(-1, 8)) + self.head_b


# ---- inputs and targets ------------------------------------------------------

def features(K, mask, dims):
    """(IN_CH/8, n, 8) bf16 from device K (n,) and conduit mask (n,):
    (log10 K + 14) / 2, the mask, the Dirichlet face mask (+1 at x = 0,
    -1 at x = 1) and zero channels up to IN_CH."""
    nx, ny, nz = dims
    K = K.to(torch.float64).contiguous()
    m = None if mask is None else mask.to(torch.uint8).contiguous()
    f = torch.empty(IN_CH // 8, K.numel(), 8, dtype=torch.bfloat16, device=K.device)
    _rc(_lib().hmfem_guess_features(K.data_ptr(), None if m is None else m.data_ptr(),
                                    nx, ny, nz, f.data_ptr(), _stream(K)))
    return f


def linear_profile(dims, device="cuda"):
    """The homogeneous solution p = 1 - (i + 1/2) / nx the net corrects."""
    nx, ny, nz = dims
    i = (torch.arange(nx * ny * nz, device=device) % nx).double()
    return 1.0 - (i + 0.5) / nx


def predict(model, K, mask, dims):
    """FP64 pressure guess on the device: the trunk, then the 1x1 head and
    the linear profile in one kernel."""
    nx, ny, nz = dims
    with torch.no_grad():
        x = model.trunk(features(K, mask, dims), dims).contiguous()
        p = torch.empty(K.numel(), dtype=torch.float64, device=K.device)
        w = model.head.detach().float().contiguous()
        b = model.head_b.detach().float().contiguous()
        _rc(_lib().hmfem_guess_head_profile(x.data_ptr(), x.shape[0], w.data_ptr(),
                                            b.data_ptr(), nx, ny, nz, p.data_ptr(), _stream(x)))
    return p


_SIDE = {}


def solve_from_guess(solver, prob, model, KX, KY=None, KZ=None, mask=None, x=None):
    """Assembly, AMG setup and the solve started from the learned guess.

    The guess depends on K alone, not on the hierarchy, so its inference
    runs on a side stream while the setup runs on the solver's stream, which
    waits for it before the solve.  K arrays and the conduit mask are CUDA
    tensors (the features use KX); x, a CUDA FP64 tensor (allocated when
    None), receives the pressure.  Every solve still runs to the solver's
    tolerance.  Returns (x, stats)."""
    KY = KX if KY is None else KY
    KZ = KX if KZ is None else KZ
    dims = (prob.nx, prob.ny, prob.nz)
    stream = torch.cuda.ExternalStream(solver.stream)
    dev = KX.device
    if dev not in _SIDE:
        _SIDE[dev] = torch.cuda.Stream(device=dev)
    side = _SIDE[dev]
    if x is None:
        x = torch.empty(prob.n, dtype=torch.float64, device=dev)
    solver.assemble(prob, KX=KX, KY=KY, KZ=KZ)
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        xg = predict(model, KX, mask, dims)
        done = torch.cuda.Event()
        done.record(side)
    solver.setup()
    with torch.cuda.stream(stream):
        stream.wait_event(done)
        xg.record_stream(stream)
        x.copy_(xg)
    del xg
    _, st = solver.solve(x=x)
    return x, st


def save(model, path):
    np.savez(path, **{k: v.detach().cpu().float().numpy() for k, v in model.state_dict().items()})


def load(path, device="cuda"):
    m = UNet()
    d = np.load(path)
    m.load_state_dict({k: torch.tensor(d[k]) for k in d.files})
    return m.to(device)
