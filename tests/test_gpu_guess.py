"""The learned initial guess: the U-Net on this library's tensor-core
convolutions against the same network in float64 on the CPU (torch's
conv3d), and a short training run whose guess the solver then starts from."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import torch.nn.functional as F  # noqa: E402

from hmfem_b200 import guess, train_guess  # noqa: E402


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


def test_short_training_guess_beats_zero_guess():
    size = 32
    data = train_guess.make_dataset(range(16), size)
    model = guess.UNet().cuda()
    hist = train_guess.train(model, data, size, epochs=6, log_every=1)
    first = np.mean([h[1] for h in hist[:16]])
    last = np.mean([h[1] for h in hist[-16:]])
    assert last < first  # the mean loss over an epoch went down
    rows = train_guess.evaluate(model, range(32, 36), size)
    assert all(r["relres_net"] <= 1e-10 for r in rows)
    assert np.mean([r["it_net"] for r in rows]) <= np.mean([r["it_zero"] for r in rows])
    assert max(r["diff"] for r in rows) < 1e-7  # same solution either way
