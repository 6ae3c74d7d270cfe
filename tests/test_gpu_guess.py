"""The learned initial guess: the U-Net on this library's tensor-core
convolutions against the same network in float64 on the CPU (torch's
conv3d), the data-movement kernels against torch, a short A-norm training
run, and the shipped model's measured gain on held-out seeds."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import torch.nn.functional as F  # noqa: E402

from hmfem_b200 import gpu, guess, train_guess  # noqa: E402


def test_unet_matches_float64_network_and_gradients():
    dims = (8, 12, 8)
    n = dims[0] * dims[1] * dims[2]
    model = guess.UNet(seed=3).cuda()
    g = torch.Generator().manual_seed(1)
    feats = torch.zeros(n, guess.IN_CH)
    feats[:, :3] = torch.randn(n, 3, generator=g)
    feats = feats.bfloat16()
    target = torch.randn(n, generator=g)
    # the same network in float64 on the CPU, weights rounded to BF16
    ref_model = guess.UNet(seed=3)
    ref_model.load_state_dict({k: v.detach().cpu() for k, v in model.state_dict().items()})
    for p in ref_model.parameters():
        p.data = p.data.bfloat16().double()
    ref = _ref_forward_with_grad(ref_model, feats.double(), dims)
    out = model(guess.blocked(feats.cuda()), dims)   # the network takes channel-blocked input
    rel = float((out.detach().cpu().double() - ref.detach()).norm() / ref.detach().norm())
    assert rel < 5e-2  # BF16 activations between layers
    # gradients of a loss: tensor-core backward vs float64 autograd
    ((out - target.cuda()) ** 2).sum().backward()
    ((ref - target.double()) ** 2).sum().backward()
    guess.check_errors()
    for (name, p), (_, q) in zip(model.named_parameters(), ref_model.named_parameters()):
        a, b = p.grad.detach().cpu().double().reshape(-1), q.grad.reshape(-1)
        cos = float(a @ b / (a.norm() * b.norm() + 1e-30))
        assert cos > 0.98, (name, cos)


def _ref_forward_with_grad(model, feats, dims):
    """The network with torch's conv3d, autograd through the parameters."""
    def t5(x, d):
        return x.view(d[2], d[1], d[0], -1).permute(3, 0, 1, 2)[None]

    def back(t):
        return t[0].permute(1, 2, 3, 0).reshape(-1, t.shape[1])

    def conv(x, name, d):
        w = model.w[name]
        w = w.view(3, 3, 3, w.shape[1], w.shape[2]).permute(3, 4, 0, 1, 2)
        return back(F.relu(F.conv3d(t5(x, d), w, model.b[name], padding=1)))

    def block(x, a, b, d):
        return conv(conv(x, a, d), b, d)

    def pool(x, d):
        return back(F.avg_pool3d(t5(x, d), 2)), (d[0] // 2, d[1] // 2, d[2] // 2)

    def up(x, d):
        return back(t5(x, d).repeat_interleave(2, 2).repeat_interleave(2, 3)
                    .repeat_interleave(2, 4))

    d0 = dims
    e0 = block(feats, "e0a", "e0b", d0)
    x, d1 = pool(e0, d0)
    e1 = block(x, "e1a", "e1b", d1)
    x, d2 = pool(e1, d1)
    x = block(x, "bna", "bnb", d2)
    x = block(torch.cat([up(x, d2), e1], 1), "d1a", "d1b", d1)
    x = block(torch.cat([up(x, d1), e0], 1), "d0a", "d0b", d0)
    return x @ model.head + model.head_b


def test_short_energy_training_lowers_its_loss():
    """Six epochs on 16 grids at 32^3 with the A-norm loss: the loss over an
    epoch goes down and the guess leads the CG to the zero-guess solution."""
    size = 32
    data = train_guess.make_dataset(range(16), size)
    model = guess.UNet().cuda()
    hist = train_guess.train(model, data, size, epochs=6, log_every=1, loss_kind="energy")
    first = np.mean([h[1] for h in hist[:16]])
    last = np.mean([h[1] for h in hist[-16:]])
    assert last < first
    rows = train_guess.evaluate(model, range(32, 36), size)
    assert all(r["relres_net"] <= 1e-10 for r in rows)
    assert max(r["diff"] for r in rows) < 1e-7  # same solution either way


# Measured with the shipped model (hmfem_b200/models/unet_config4.npz, A-norm
# loss, 2048 training grids at 128^3, 4 epochs) on the bench's held-out
# seeds 2048-2055: 27.375 CG iterations against 28.75 from the zero guess
# (-1.375; 256 held-out seeds: 24.84 against 26.18), the guess's A-norm error
# 0.049 and its initial residual 0.24 of the linear profile's.
GAIN_ITERATIONS = 1.0
MAX_ENERGY_RATIO = 0.08
MAX_RESIDUAL_RATIO = 0.35


def test_shipped_guess_cuts_iterations_on_held_out_seeds():
    model = guess.load(train_guess.MODEL_PATH)
    rows = train_guess.evaluate(model, range(2048, 2056), 128)
    it_zero = np.mean([r["it_zero"] for r in rows])
    it_net = np.mean([r["it_net"] for r in rows])
    assert it_zero - it_net >= GAIN_ITERATIONS, (it_zero, it_net)
    assert all(r["it_net"] <= r["it_zero"] for r in rows)
    assert np.mean([r["energy_ratio"] for r in rows]) <= MAX_ENERGY_RATIO
    assert np.mean([r["resid_ratio"] for r in rows]) <= MAX_RESIDUAL_RATIO
    assert all(r["relres_net"] <= 1e-10 for r in rows)
    assert max(r["diff"] for r in rows) < 1e-7


def test_data_movement_kernels_match_torch():
    """Features, pooling (and its gradient), upsampling fused with the skip
    concatenation (and its gradients) and the fused head/profile against
    the same operations written with torch on channels-last tensors."""
    dims = (12, 8, 4)   # two 2x levels: divisible by 4
    nx, ny, nz = dims
    n = nx * ny * nz
    g = torch.Generator(device="cuda").manual_seed(2)
    K = 10.0 ** (-14.0 + torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
    mask = (torch.rand(n, generator=g, device="cuda") < 0.1).to(torch.uint8)
    f = guess.unblocked(guess.features(K, mask, dims)).float()
    i = torch.arange(n, device="cuda") % nx
    ref = torch.zeros(n, 16, device="cuda")
    ref[:, 0] = ((torch.log10(K) + 14.0) / 2.0).float().bfloat16().float()
    ref[:, 1] = mask.float()
    ref[:, 2] = (i == 0).float() - (i == nx - 1).float()
    assert torch.equal(f, ref)

    def t5(x, d):  # channels-last (n, C) -> (1, C, nz, ny, nx)
        return x.view(d[2], d[1], d[0], -1).permute(3, 0, 1, 2)[None]

    def back(t):
        return t[0].permute(1, 2, 3, 0).reshape(-1, t.shape[1])

    x = torch.randn(n, 32, generator=g, device="cuda").bfloat16().requires_grad_()
    xb = guess.blocked(x.detach()).requires_grad_()
    pooled, cd = guess.pool2(xb, dims)
    pref = back(F.avg_pool3d(t5(x.float(), dims), 2))
    assert torch.allclose(guess.unblocked(pooled).float(), pref, rtol=1e-2, atol=1e-2)
    w = torch.randn(pooled.shape, generator=g, device="cuda").bfloat16()
    (pooled.float() * w.float()).sum().backward()
    (pref * guess.unblocked(w).float()).sum().backward()
    assert torch.allclose(guess.unblocked(xb.grad).float(), x.grad.float(), rtol=1e-2, atol=1e-3)

    c = torch.randn(n // 8, 16, generator=g, device="cuda").bfloat16().requires_grad_()
    s = torch.randn(n, 8, generator=g, device="cuda").bfloat16().requires_grad_()
    cb, sb = guess.blocked(c.detach()).requires_grad_(), guess.blocked(s.detach()).requires_grad_()
    out = guess.up2_cat(cb, sb, dims)
    up = back(t5(c.float(), cd).repeat_interleave(2, 2).repeat_interleave(2, 3)
              .repeat_interleave(2, 4))
    oref = torch.cat([up, s.float()], 1)
    assert torch.equal(guess.unblocked(out).float(), oref)
    w = torch.randn(out.shape, generator=g, device="cuda").bfloat16()
    (out.float() * w.float()).sum().backward()
    (oref * guess.unblocked(w).float()).sum().backward()
    assert torch.allclose(guess.unblocked(cb.grad).float(), c.grad.float(), rtol=1e-2, atol=1e-2)
    assert torch.equal(guess.unblocked(sb.grad).float(), s.grad.float())

    model = guess.UNet(seed=4).cuda()
    p = guess.predict(model, K, mask, dims)
    with torch.no_grad():
        corr = model(guess.features(K, mask, dims), dims)
    assert torch.allclose(p, guess.linear_profile(dims) + corr.double(), rtol=0, atol=1e-5)
    guess.check_errors()


def test_solve_from_guess_equals_the_sequential_solve():
    """The overlapped call (inference beside the setup) starts the CG from
    the same guess as predict-then-solve: the same iterations and pressure."""
    size = 32
    model = guess.UNet(seed=5).cuda()
    prob, K, mask = train_guess.sample(7, size)
    s = gpu.Solver(precision=1, tol=1e-10)
    x1, st1 = guess.solve_from_guess(s, prob, model, K, mask=mask)
    s.assemble(prob, KX=K, KY=K, KZ=K)
    s.setup()
    x2 = guess.predict(model, K, mask, (size, size, size))
    _, st2 = s.solve(x=x2)
    assert st1["iterations"] == st2["iterations"] and st1["relres"] <= 1e-10
    assert torch.equal(x1, x2)
    s.close()
