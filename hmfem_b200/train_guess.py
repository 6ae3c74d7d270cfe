"""Trains and evaluates the learned initial guess on solver-generated data.

    python -m hmfem_b200.train_guess --size 128 --train 2048 --eval 256 \\
        --epochs 4 --out unet_guess.npz

Data: log10 K = -14 + 1.5 g with g a unit-variance Gaussian field of
correlation length 8 cells (seeded white noise, FFT filtered on the GPU)
and random-walk conduits, Dirichlet 1/0 on the x faces, no flow elsewhere
(--dist): config4 = 0-6 conduits at K = 1e-10, config2 = 0-8 at 1e-9 (the
256^3 headline problem's kind), mixed = the two alternately by seed parity;
seeds 0..train-1 train, the next `eval` seeds (config-4 kind) evaluate.  Targets are this solver's FP64 pressures (relres 1e-8);
the net learns the correction to the linear profile 1 - (i + 1/2)/nx.  The
loss (--loss) measures the guess's error e = p_guess - p the way the CG
sees it, relative to the linear profile's error e_lin:
  energy    e^T A e / e_lin^T A e_lin   (A-norm; gradient 2 A e)
  residual  |A e|^2 / |A e_lin|^2       (the initial residual; 2 A A e)
  l2        |e| / |p|                   (plain pressure error)
with A this sample's TPFA matrix (FP64 SpMV of the solver) and the head's
output in FP32.  Evaluation solves every held-out grid to
||b - A x|| / ||b|| <= 1e-10 from the zero guess and from the net's guess
(inference included in the timed path) and prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np
import torch

from . import gpu, guess
from .problem import Problem, random_walk_conduit

# the shipped model: A-norm loss, seeds 0-2047 at 128^3, 4 epochs
MODEL_PATH = os.path.join(os.path.dirname(__file__), "models", "unet_config4.npz")


def gaussian_field_gpu(gen, n, corr, device="cuda"):
    """Unit-variance Gaussian random field on an n^3 grid: white noise
    convolved (periodically, by FFT) with a normalised Gaussian of std
    `corr` cells."""
    g = torch.randn(n, n, n, generator=gen, device=device, dtype=torch.float64)
    k = torch.fft.fftfreq(n, device=device, dtype=torch.float64)
    kr = torch.fft.rfftfreq(n, device=device, dtype=torch.float64)
    ker = torch.exp(-2.0 * (math.pi * corr) ** 2 *
                    (k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2))
    g = torch.fft.irfftn(torch.fft.rfftn(g) * ker, s=(n, n, n))
    g = g - g.mean()
    return (g / g.std()).reshape(-1)


DISTS = {"config4": (7, 1e-10), "config2": (9, 1e-9)}  # (conduits < n, K of a conduit)


def dist_of(seed, dist):
    """The distribution of a seed: `dist`, or for "mixed" config4 on even
    seeds and config2 on odd ones."""
    return ("config2" if seed % 2 else "config4") if dist == "mixed" else dist


def sample(seed, size, device="cuda", dist="config4"):
    """(Problem without host K, device K, device conduit mask) of one seed."""
    n_max, k_conduit = DISTS[dist_of(seed, dist)]
    rng = np.random.default_rng(1400 + seed)
    gen = torch.Generator(device=device).manual_seed(77_000 + seed)
    K = 10.0 ** (-14.0 + 1.5 * gaussian_field_gpu(gen, size, 8.0, device))
    mask = torch.zeros(size ** 3, dtype=torch.uint8, device=device)
    for _ in range(int(rng.integers(0, n_max))):
        c = torch.as_tensor(random_walk_conduit(rng, size, size, size), device=device)
        K[c] = k_conduit
        mask[c] = 1
    dummy = np.zeros(1)
    p = Problem(size, size, size, 1.0 / size, 1.0 / size, 1.0 / size, dummy, dummy, dummy)
    return p, K.contiguous(), mask


def solve(solver, prob, K, x=None):
    """Assembly + setup + solve on the device; x (device FP64) is the
    initial guess in and the pressure out."""
    solver.assemble(prob, KX=K, KY=K, KZ=K)
    solver.setup()
    if x is None:
        x = torch.zeros(prob.n, dtype=torch.float64, device=K.device)
    _, st = solver.solve(x=x)
    return x, st


class Sample:
    """One training grid: input features, K (FP32; the matrix is assembled
    again from it for the A-norm and residual losses), the target correction
    p - p_lin (FP64) and the loss normalisers."""

    def __init__(self, f3, K32, target, pnorm, e_energy, e_resid):
        self.f3, self.K32, self.target = f3, K32, target
        self.pnorm, self.e_energy, self.e_resid = pnorm, e_energy, e_resid


def make_dataset(seeds, size, device="cuda", dist="config4"):
    s = gpu.Solver(precision=1, tol=1e-8)
    data = []
    dims = (size, size, size)
    for sd in seeds:
        prob, K, mask = sample(sd, size, device, dist)
        p, _ = solve(s, prob, K)
        f3 = guess.features(K, mask, dims)[0, :, :3].contiguous()
        target = p - guess.linear_profile(dims, device)        # -e_lin
        K32 = K.float()
        s.assemble(prob, KX=K32.double(), KY=K32.double(), KZ=K32.double())
        At = s.spmv(0, target)
        data.append(Sample(f3, K32, target, float(p.norm()), float(target @ At),
                           float(At @ At)))
    s.close()
    return data


class GuessLoss(torch.autograd.Function):
    """energy: e^T A e / E0 (d/de = 2 A e / E0); residual: |A e|^2 / R0
    (d/de = 2 A A e / R0); e = corr - target in FP64."""

    @staticmethod
    def forward(ctx, corr, target, solver, norm, kind):
        e = corr.double() - target
        Ae = solver.spmv(0, e)
        if kind == "energy":
            ctx.save_for_backward(Ae)
            val = (e @ Ae) / norm
        else:
            ctx.save_for_backward(solver.spmv(0, Ae))
            val = (Ae @ Ae) / norm
        ctx.norm = norm
        return val.float()

    @staticmethod
    def backward(ctx, g):
        (v,) = ctx.saved_tensors
        return (2.0 * g.double() * v / ctx.norm).float(), None, None, None, None


def _feats(f3):
    f = torch.zeros(guess.IN_CH // 8, f3.shape[0], 8, dtype=torch.bfloat16, device=f3.device)
    f[0, :, :3] = f3
    return f


def train(model, data, size, epochs, lr=1e-3, log_every=0, loss_kind="l2"):
    dims = (size, size, size)
    solver = gpu.Solver(precision=1) if loss_kind != "l2" else None
    prob = sample_problem(size)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    steps = epochs * len(data)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=max(1, steps))
    order = np.random.default_rng(0)
    hist = []
    k = 0
    for ep in range(epochs):
        for i in order.permutation(len(data)):
            d = data[i]
            pred = model(_feats(d.f3), dims)
            if loss_kind == "l2":
                loss = (pred.double() - d.target).norm() / d.pnorm
            else:
                K = d.K32.double()
                solver.assemble(prob, KX=K, KY=K, KZ=K)
                norm = d.e_energy if loss_kind == "energy" else d.e_resid
                loss = GuessLoss.apply(pred, d.target, solver, norm, loss_kind)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            torch.nn.utils.clip_grad_norm_(model.parameters(), 1.0)
            opt.step()
            sched.step()
            k += 1
            if log_every and k % log_every == 0:
                hist.append((k, float(loss.detach())))
    guess.check_errors()
    if solver is not None:
        solver.close()
    return hist


def sample_problem(size):
    """The Problem (dims, spacing, boundary conditions) of a training grid."""
    dummy = np.zeros(1)
    return Problem(size, size, size, 1.0 / size, 1.0 / size, 1.0 / size, dummy, dummy, dummy)


def evaluate(model, seeds, size, device="cuda", tol=1e-10):
    dims = (size, size, size)
    s = gpu.Solver(precision=1, tol=tol)
    rows = []
    for sd in seeds:
        prob, K, mask = sample(sd, size, device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x0, st0 = solve(s, prob, K)
        torch.cuda.synchronize()
        t_zero = time.perf_counter() - t0
        t0 = time.perf_counter()
        xg = guess.predict(model, K, mask, dims)
        x1, st1 = solve(s, prob, K, xg.clone())   # the solve overwrites its guess
        torch.cuda.synchronize()
        t_net = time.perf_counter() - t0
        e_guess = float((xg - x0).norm() / x0.norm())
        xl = guess.linear_profile(dims, device)
        e_lin = float((xl - x0).norm() / x0.norm())
        # the guesses' errors as the CG sees them, relative to the profile's
        # (A of this grid is assembled: the last solve)
        en, rn = [], []
        for xx in (xg, xl):
            e = xx - x0
            Ae = s.spmv(0, e)
            en.append(float(e @ Ae))
            rn.append(float(Ae.norm()))
        xl, stl = solve(s, prob, K, xl)
        rows.append(dict(seed=sd, it_zero=st0["iterations"], it_net=st1["iterations"],
                         it_linear=stl["iterations"], t_zero=t_zero, t_net=t_net,
                         err_guess=e_guess, err_linear=e_lin,
                         energy_ratio=en[0] / en[1], resid_ratio=rn[0] / rn[1],
                         relres_net=st1["relres"], diff=float((x1 - x0).norm() / x0.norm())))
    s.close()
    return rows


def infer_once(size=128, seed=5000, path=None):
    """One guess inference on a config-4 grid (the command the conv3d ncu
    summary profiles); returns its wall time in ms."""
    model = guess.load(path) if path else guess.UNet().cuda()
    prob, K, mask = sample(seed, size)
    dims = (size, size, size)
    guess.predict(model, K, mask, dims)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    guess.predict(model, K, mask, dims)
    torch.cuda.synchronize()
    guess.check_errors()
    return 1e3 * (time.perf_counter() - t0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--train", type=int, default=2048)
    ap.add_argument("--eval", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default="unet_guess.npz")
    ap.add_argument("--loss", default="energy", choices=("energy", "residual", "l2"))
    ap.add_argument("--dist", default="config4", choices=("config4", "config2", "mixed"))
    ap.add_argument("--infer-only", action="store_true",
                    help="time one inference at --size (no training) and exit")
    args = ap.parse_args()
    if args.infer_only:
        print(json.dumps({"size": args.size, "inference_ms": infer_once(args.size)}))
        return
    torch.manual_seed(0)
    t0 = time.perf_counter()
    data = make_dataset(range(args.train), args.size, dist=args.dist)
    t_data = time.perf_counter() - t0
    model = guess.UNet().cuda()
    t0 = time.perf_counter()
    hist = train(model, data, args.size, args.epochs, args.lr, log_every=256,
                 loss_kind=args.loss)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del data
    guess.save(model, args.out)
    rows = evaluate(model, range(args.train, args.train + args.eval), args.size)
    mean = lambda k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    print(json.dumps({
        "workload": f"config4 {args.size}^3 lognormal (std 1.5, corr 8) + 0-6 conduits",
        "params": model.n_params(), "train_samples": args.train, "epochs": args.epochs,
        "eval_samples": args.eval, "data_s": t_data, "train_s": t_train,
        "loss_history": hist,
        "iterations_zero_guess": mean("it_zero"), "iterations_net_guess": mean("it_net"),
        "iterations_linear_guess": mean("it_linear"),
        "time_zero_guess_ms": 1e3 * mean("t_zero"), "time_net_guess_ms": 1e3 * mean("t_net"),
        "guess_rel_error": mean("err_guess"), "linear_rel_error": mean("err_linear"),
        "loss": args.loss, "dist": args.dist, "guess_energy_vs_linear": mean("energy_ratio"),
        "guess_residual_vs_linear": mean("resid_ratio"),
        "max_relres_net": max(r["relres_net"] for r in rows),
        "max_pressure_diff_vs_zero_guess": max(r["diff"] for r in rows),
        "out": args.out}), flush=True)


if __name__ == "__main__":
    main()
