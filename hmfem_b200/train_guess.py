"""Trains and evaluates the learned initial guess on solver-generated data.

    python -m hmfem_b200.train_guess --size 128 --train 2048 --eval 256 \\
        --epochs 4 --out unet_guess.npz

Data (config 4 distribution): log10 K = -14 + 1.5 g with g a unit-variance
Gaussian field of correlation length 8 cells (seeded white noise, FFT
filtered on the GPU), 0-6 random-walk conduits at K = 1e-10, Dirichlet 1/0
on the x faces, no flow elsewhere; seeds 0..train-1 train, the next `eval`
seeds evaluate.  Targets are this solver's FP64 pressures (relres 1e-8);
the net learns the correction to the linear profile 1 - (i + 1/2)/nx with a
relative-L2 pressure loss.  Evaluation solves every held-out grid to
||b - A x|| / ||b|| <= 1e-10 from the zero guess and from the net's guess
(inference included in the timed path) and prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import gpu, guess
from .problem import Problem, random_walk_conduit


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


def sample(seed, size, device="cuda"):
    """(Problem without host K, device K, device conduit mask) of one seed."""
    rng = np.random.default_rng(1400 + seed)
    gen = torch.Generator(device=device).manual_seed(77_000 + seed)
    K = 10.0 ** (-14.0 + 1.5 * gaussian_field_gpu(gen, size, 8.0, device))
    mask = torch.zeros(size ** 3, dtype=torch.uint8, device=device)
    for _ in range(int(rng.integers(0, 7))):
        c = torch.as_tensor(random_walk_conduit(rng, size, size, size), device=device)
        K[c] = 1e-10
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


def make_dataset(seeds, size, device="cuda"):
    s = gpu.Solver(precision=1, tol=1e-8)
    data = []
    for sd in seeds:
        prob, K, mask = sample(sd, size, device)
        p, _ = solve(s, prob, K)
        dims = (size, size, size)
        f3 = guess.features(K, mask, dims)[0, :, :3].contiguous()
        target = (p - guess.linear_profile(dims, device)).float()
        pnorm = float(p.norm())
        data.append((f3, target, pnorm))
    s.close()
    return data


def _feats(f3):
    f = torch.zeros(guess.IN_CH // 8, f3.shape[0], 8, dtype=torch.bfloat16, device=f3.device)
    f[0, :, :3] = f3
    return f


def train(model, data, size, epochs, lr=1e-3, log_every=0):
    dims = (size, size, size)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    steps = epochs * len(data)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=max(1, steps))
    order = np.random.default_rng(0)
    hist = []
    k = 0
    for ep in range(epochs):
        for i in order.permutation(len(data)):
            f3, target, pnorm = data[i]
            pred = model(_feats(f3), dims)
            loss = (pred - target).norm() / pnorm
            opt.zero_grad(set_to_none=True)
            loss.backward()
            torch.nn.utils.clip_grad_norm_(model.parameters(), 1.0)
            opt.step()
            sched.step()
            k += 1
            if log_every and k % log_every == 0:
                hist.append((k, float(loss.detach())))
    guess.check_errors()
    return hist


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
        e_guess = float((xg - x0).norm() / x0.norm())
        x1, st1 = solve(s, prob, K, xg)
        torch.cuda.synchronize()
        t_net = time.perf_counter() - t0
        xl = guess.linear_profile(dims, device)
        e_lin = float((xl - x0).norm() / x0.norm())
        xl, stl = solve(s, prob, K, xl)
        rows.append(dict(seed=sd, it_zero=st0["iterations"], it_net=st1["iterations"],
                         it_linear=stl["iterations"], t_zero=t_zero, t_net=t_net,
                         err_guess=e_guess, err_linear=e_lin,
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
    ap.add_argument("--infer-only", action="store_true",
                    help="time one inference at --size (no training) and exit")
    args = ap.parse_args()
    if args.infer_only:
        print(json.dumps({"size": args.size, "inference_ms": infer_once(args.size)}))
        return
    torch.manual_seed(0)
    t0 = time.perf_counter()
    data = make_dataset(range(args.train), args.size)
    t_data = time.perf_counter() - t0
    model = guess.UNet().cuda()
    t0 = time.perf_counter()
    hist = train(model, data, args.size, args.epochs, args.lr, log_every=256)
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
        "max_relres_net": max(r["relres_net"] for r in rows),
        "max_pressure_diff_vs_zero_guess": max(r["diff"] for r in rows),
        "out": args.out}), flush=True)


if __name__ == "__main__":
    main()
