"""Benchmark: cells/s of hmfem's pressure solve on B200 to ||r||/||b|| <= 1e-10.

One step = the hot path over one synthetic problem with the permeability
field already resident in HBM: TPFA assembly -> AMG setup (C/F split,
interpolation, Galerkin products, all on the device) -> CG to a true FP64
relative residual <= 1e-10.  Workload: 256^3 cells, log10 K = -14 + 1.5 g
(Gaussian field, correlation 8 cells) + 8 random-walk conduits at K = 1e-9,
Dirichlet p=1 / p=0 on the x faces, no-flow elsewhere.

The headline variant ("chosen") is the FP32 V-cycle inside FP64 flexible CG
started from the learned initial guess (U-Net on the tensor-core conv3d
kernels, hmfem_b200/models/unet_config4.npz, its inference inside the timed
step); measured in the same run: the same solve from the zero guess (the
fallback and the judge of the guess; --zero-guess-chosen makes it the
headline, and it is the headline when the model is absent or --no-guess)
and the plain FP64 AMG-PCG drop-in.  `e2e` is the chosen solve from pinned
host buffers (K and the conduit mask uploaded, the guess inferred on the
device, the pressure downloaded, all inside the timed region).  `--impl reference` times the
reference's own CPU path (oracle/_ref, compiled from the hmfem sources) on
all host cores over a bounded sample of the same workload.

Multi-GPU: the path does not shard; --gpus N runs N independent replicas,
one per rank (weak scaling), and value is the sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (read + write) per cell of one k_g7_spmv_dot2 launch, from an
# ncu --set full capture of the same kernel on config 2 at 192^3 (7.08M
# cells, 328 MB): the launch is linear in cells, so bench scales it.
SPMV_TRAFFIC_B_PER_CELL = 46.4

METRIC = ("cells/s to ||r||/||b||<=1e-10 (256^3 lognormal+conduits), "
          "chosen=FP32 V-cycle in FP64 FCG from the learned initial guess")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-guess", action="store_true",
                    help="skip the learned-guess variant")
    ap.add_argument("--zero-guess-chosen", action="store_true",
                    help="report the zero-guess FP32 variant as the headline")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched uneven-instance measurement (config 3)")
    ap.add_argument("--no-coupled", action="store_true",
                    help="skip the coupled reservoir/conduit (Picard) workload")
    ap.add_argument("--no-output", action="store_true",
                    help="skip the result-file writers")
    ap.add_argument("--cpu-sample", type=int, default=96)
    ap.add_argument("--no-config1", action="store_true",
                    help="skip the 128^3 plain-vs-chosen comparison (config 1)")
    ap.add_argument("--profile-step", type=int, default=-1, metavar="PRECISION",
                    help="run one untimed step (assembly + setup + solve) of "
                         "the plain FP64 (0), the FP32 zero-guess (1) or the "
                         "FP32 learned-guess (2) variant and exit: the command "
                         "the ncu summaries under profiles/ profile")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers --

def _split_kernel(name):
    """('k_cheb_step', ['float', 'Pk16', '2']) from a demangled kernel name
    such as 'void hm::(anonymous namespace)::k_cheb_step<float, hm::Pk16, 2>(...)'."""
    import re
    m = re.search(r"\b(k_\w+)", name)
    if not m:
        return name, []
    base, i = m.group(1), m.end()
    args = []
    if i < len(name) and name[i] == "<":
        depth, cur = 0, ""
        for ch in name[i:]:
            if ch == "<":
                depth += 1
                if depth == 1:
                    continue
            elif ch == ">":
                depth -= 1
                if depth == 0:
                    args.append(cur.strip())
                    break
            elif ch == "," and depth == 1:
                args.append(cur.strip())
                cur = ""
                continue
            cur += ch
    return base, [a.split("::")[-1] for a in args]


def _tbytes(t):
    return {"double": 8, "float": 4, "__nv_bfloat16": 2}.get(t, 4)


def kernel_bytes(name, level, info, precision):
    """Algorithmic bytes of one launch (no padding; every vector element and
    every stored matrix entry once).  `info[l]` = (rows, nonzeros, P
    nonzeros) of level l; level -1 = the CG's level-0 vectors.  T = vector
    bytes, vb = matrix value bytes, es = SELL entry bytes (value + 4-byte
    column; 4 for the packed BF16 word).  Returns None for kernels without
    a bandwidth model (latency-bound setup work)."""
    base, targs = _split_kernel(name)
    l = max(level, 0)
    n, nnz, pn = info[l]
    nc = info[l + 1][0] if l + 1 < len(info) else 0
    T = _tbytes(targs[0]) if targs else 8
    vb = _tbytes(targs[1]) if len(targs) > 1 else T
    es = 4 if (len(targs) > 1 and targs[1] == "Pk16") else vb + 4
    mode = targs[2] if len(targs) > 2 else ""
    n0 = info[0][0]
    table = {
        "k_g7_spmv_dot": 48 * n0,                       # 4 coefficients + s + v
        "k_g7_spmv_dot2": 48 * n0,                      # the same on x-adjacent cell pairs
        "k_update": 48 * n0 + (4 if precision == 1 else 16) * n0,  # x, r, s, v + FP32 r / FP64 seed
        "k_g7_resid": (56 + (4 if precision == 1 else 16)) * n0,   # runs on check iterations
        "k_finish_z": (T + 16) * n0,                    # z, r, v
        "k_sdir": (T + 16) * n0,                        # z, s in/out
        "k_g7_sred": (T + 3 * vb + T // 2 + T) * n,     # f, couplings, F-half D^-1, fc + seed
        "k_g7_sprol2": (3 * vb + T + T // 2 + T) * n,   # couplings, F-half f/D^-1, uc, z
        "k_g7_sprol2_zd": (3 * vb + T + T // 2 + T + 16) * n,  # the same + the CG's r, v for the dots
        "k_g7_pre": (4 * vb + 3 * T) * n,
        "k_g7_post": (4 * vb + 4 * T) * n,
        "k_g7_restrict": T * n + 3 * T * nc,
        "k_g7_prolong": T * nc + 2 * T * n,
        "k_g19_pre": nnz * vb + (3 * T + 4) * n,
        "k_g19_post": nnz * vb + 4 * T * n,
        "k_pre": nnz * es + (3 * T + 4) * n,
        "k_post": nnz * es + 4 * T * n,
        "k_cheb0": nnz * es + 5 * T * n,
        "k_cheb_step": nnz * es + {"0": 6, "1": 7}.get(mode, 6) * T * n,
        "k_restrict": 4 * pn + T * n + (4 + 3 * T) * nc,
        "k_prolong_add": 4 * n + 4 * pn + T * nc + 2 * T * n,
        "k_dense_solve": 8 * n * n + 2 * T * n,
        "k_diag_solve": 3 * T * n,
    }
    return table.get(base)


def kernel_table(solver, precision, iters, peak):
    """Every kernel of `iters` CG iterations, timed one launch at a time with
    CUDA events on the solver stream (hmfem_profile_iteration), with its
    algorithmic bytes, GB/s and fraction of the HBM peak; sorted by time."""
    info = []
    for l in range(solver.num_levels()):
        info.append(solver.level_info(l))
    rows = solver.profile_iteration(iters)
    tot = sum(r["ms"] for r in rows)
    out = []
    for r in sorted(rows, key=lambda r: -r["ms"]):
        base, targs = _split_kernel(r["kernel"])
        label = base + ("<" + ",".join(targs) + ">" if targs else "")
        b = kernel_bytes(r["kernel"], r["level"], info, precision)
        us = 1e3 * r["ms"] / r["launches"]
        e = {"kernel": label, "level": r["level"], "launches_per_iteration": r["launches"] / iters,
             "us_per_launch": round(us, 2), "share": round(r["ms"] / tot, 4)}
        if b is not None:
            gbs = b / (us * 1e-6) / 1e9
            e.update(bytes_per_launch=int(b), GBps=round(gbs, 1), frac=round(gbs / peak, 3))
        out.append(e)
    return {"iterations_profiled": iters, "sum_ms_per_iteration": round(tot / iters, 4),
            "kernels": out,
            "timing": "CUDA events around each launch on the solver stream, launches "
                      "one at a time (no graph, no programmatic overlap)"}


class Clocks:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev, self.rows, self.proc = dev, [], None
        self.t0, self.t1 = None, None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(),
                              [c.strip() for c in line.split(",")]))

    def window(self, t0, t1):
        """Samples taken while [t0, t1] (the timed region) was running."""
        self.t0, self.t1 = t0, t1

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = [r for t, r in self.rows
                if self.t0 is None or self.t0 <= t <= self.t1 + 0.15]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 2 + i and r[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def dist_init(args):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK); NCCL
    on GPUs, gloo where there is none (the host-side tests of this path)."""
    import torch
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime
        import torch.distributed as dist
        timeout = datetime.timedelta(seconds=600)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timeout,
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timeout)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world):
    """The max of v over the ranks (times are taken as the slowest rank's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------- our arm -----

def run_ours(args):
    import torch

    from hmfem_b200 import gpu
    from hmfem_b200.problem import config_problem

    rank, world, local = dist_init(args)
    # the reference's own CPU path on this exact problem, on one host core
    # in a process of its own while the GPU arms run: the CPU baseline at the
    # bench's configuration and the FP64 oracle the pressures are checked
    # against
    ref_full = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref_full = start_reference_full(args.size, args.tol)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prob = config_problem(2, size=args.size)  # same field on every replica
    n = prob.n
    K = torch.tensor(prob.KX, device=dev)     # resident in HBM (> L2)

    def make(precision):
        # the FP32 cycle keeps levels >= 1 in BF16 (same iterations, less
        # traffic); the plain drop-in stays FP64 throughout
        # the FP32 cycle also reduces level 0 exactly (schur0: level 1 is the
        # Schur complement of the red-black split, same structure as the
        # reference's level 1)
        s = gpu.Solver(precision=precision, tol=args.tol,
                       bf16_from=1 if precision == 1 else -1, check_every=2,
                       schur0=1 if precision == 1 else 0)
        stream = torch.cuda.ExternalStream(s.stream)
        return s, stream

    # learned initial guess (trained by hmfem_b200.train_guess on config-4
    # data and kept with the package): its inference is part of the step
    model = None
    model_path = os.path.join(ROOT, "hmfem_b200", "models", "unet_config4.npz")
    if os.path.exists(model_path) and not args.no_guess:
        from hmfem_b200 import guess
        model = guess.load(model_path, dev)
        mask = torch.as_tensor(prob.conduit_mask, device=dev)
        dims = (prob.nx, prob.ny, prob.nz)

    def step(s, x, stream=None, learned=False):
        if learned:  # inference beside the setup (guess.solve_from_guess)
            _, st = guess.solve_from_guess(s, prob, model, K, mask=mask, x=x)
            return st
        s.assemble(prob, KX=K, KY=K, KZ=K)
        s.setup()
        with torch.cuda.stream(stream):  # the solver's stream: ordered
            x.zero_()
        _, st = s.solve(x=x)
        return st

    variants = [("plain_fp64", 0, False), ("fp32_zero_guess", 1, False)]
    if model is not None:
        variants.append(("fp32_learned_guess", 1, True))
    results = {}
    launches = {}
    for name, precision, learned in variants:
        s, stream = make(precision)
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        # the clock sampler starts before the warm-up (its start-up stalls
        # the driver) and only its samples from the timed region are kept
        with Clocks(local) as ck:
            for _ in range(args.warmup):
                st = step(s, x, stream, learned)
            torch.cuda.synchronize()
            barrier(world)
            times, stats = [], []
            c0 = gpu.launch_count()
            tw0 = time.perf_counter()
            for _ in range(args.steps):
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st = step(s, x, stream, learned)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                stats.append(st)
            ck.window(tw0, time.perf_counter())
        torch.cuda.synchronize()
        launches[name] = gpu.launch_count() - c0
        barrier(world)
        total_ms = max_over_ranks(sum(times), world)
        results[name] = dict(ms_per_step=total_ms / args.steps,
                             value=world * n * args.steps / (total_ms / 1e3),
                             iterations=stats[-1]["iterations"],
                             relres=stats[-1]["relres"],
                             levels=stats[-1]["levels"],
                             setup_ms=stats[-1]["t_setup_ms"],
                             solve_ms=stats[-1]["t_solve_ms"],
                             clocks=ck.summary(), solver=s, stream=stream, x=x)
    # "chosen": the FP32 V-cycle in FP64 flexible CG from the learned guess
    # (here 44 CG iterations against 50 from zero; the inference is part of
    # the step); the zero guess, measured beside it, is the fallback
    chosen_name = "fp32_zero_guess" if (model is None or args.zero_guess_chosen) \
        else "fp32_learned_guess"
    ch = results[chosen_name]
    launches["chosen"] = launches[chosen_name]

    # ---- roofline: the dominant kernel, timed live on the solver stream
    s0 = results["plain_fp64"]["solver"]
    s1 = ch["solver"]
    # L0 SpMV of the CG in its 7-point form: 4 coefficients + x + y per cell
    ms0, by0 = s1.time_kernel(5, 0, reps=20)
    peaks = {}
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    if "hbm_gbs" in peaks:
        peak, peak_src = float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = by0 / (ms0 / 1e3) / 1e9
    # every kernel of the chosen and the plain CG iteration, timed live
    kernels = {"chosen": kernel_table(s1, 1, 3, peak),
               "plain_fp64": kernel_table(s0, 0, 3, peak)}

    # ---- e2e through the public API with host buffers (pinned host memory,
    # as an application that streams fields to the GPU keeps them)
    s_e2e = gpu.Solver(precision=1, tol=args.tol, bf16_from=1, check_every=2, schur0=1)
    k_pin = torch.from_numpy(np.ascontiguousarray(prob.KX)).pin_memory()
    x_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    kh, xh = k_pin.numpy(), x_pin.numpy()
    learned_e2e = chosen_name == "fp32_learned_guess"
    if learned_e2e:
        # the guess needs K on the device: K and the conduit mask go up once
        # (pinned -> device on the solver's stream), the inference writes the
        # guess there, the solve starts from it, the pressure comes back
        m_pin = torch.as_tensor(prob.conduit_mask).pin_memory()
        Kd = torch.empty(n, dtype=torch.float64, device=dev)
        md = torch.empty(n, dtype=torch.uint8, device=dev)
        xd = torch.empty(n, dtype=torch.float64, device=dev)
        e2e_stream = torch.cuda.ExternalStream(s_e2e.stream)

    def e2e_step():
        if not learned_e2e:
            xh[:] = 0                     # the step's input: the initial guess
            s_e2e.assemble(prob, KX=kh, KY=kh, KZ=kh)  # K host -> device inside
            s_e2e.setup()
            s_e2e.solve(x=xh)             # x host -> device, pressure device -> host
            return
        # blocking copies (the step ends synchronised anyway): a non-blocking
        # copy would leave the pinned buffers an event on the solver's stream
        # to record when they are freed, after that stream is gone
        with torch.cuda.stream(e2e_stream):
            Kd.copy_(k_pin)
            md.copy_(m_pin)
        guess.solve_from_guess(s_e2e, prob, model, Kd, mask=md, x=xd)
        with torch.cuda.stream(e2e_stream):
            x_pin.copy_(xd)
        e2e_stream.synchronize()

    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    te = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        te.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(te), world)
    # K uploaded once per distinct host array (the field is isotropic: the
    # three directions share one array), plus the initial guess (zero-guess
    # path) or the conduit mask (learned path)
    e2e = {"value": world * n * args.steps / e2e_s, "unit": "cells/s",
           "h2d_bytes_per_step": n * 8 + (n if learned_e2e else n * 8),
           "d2h_bytes_per_step": n * 8, "variant": chosen_name}

    batched = None if args.no_batch else run_batch(args, world)

    # the chosen and plain pressures and fluxes against the reference's
    # own FP64 solution of the same problem (waits for its process; the
    # host-side baselines below run after it, so they do not share cores
    # with it)
    oracle_error, cpu_full = None, None
    if ref_full is not None:
        cpu_full, ref_p, ref_v = finish_reference_full(ref_full)
        if ref_p is not None:
            oracle_error = {}
            for name in dict.fromkeys(("plain_fp64", "fp32_zero_guess", chosen_name)):
                r = results[name]
                oracle_error[name] = pressure_flux_error(r["solver"], r["x"], prob, ref_p,
                                                         ref_v, dev)
                oracle_error[name]["relres"] = r["relres"]
            oracle_error["oracle"] = cpu_full.get("oracle")
            del ref_p, ref_v
    if batched is not None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        batched["cpu_reference"] = batch_cpu_baseline(args.tol)
        rate = batched["cpu_reference"].get("processes", {}).get("instances_per_s")
        if rate:
            batched["speedup_vs_reference_processes"] = batched["instances_per_s"] / rate
    config1 = None if args.no_config1 else run_config1(args, dev)
    config4 = None if (args.no_guess or model is None) else run_config4(args, dev, model)

    coupled = None if args.no_coupled else run_coupled(args, world, rank)
    output = None
    if not args.no_output and rank == 0:
        output = run_output(args, prob, s_e2e, xh, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_full if (cpu_full and cpu_full.get("value")) else \
            cpu_baseline_sample(args.cpu_sample, cores=1)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": ch["value"], "unit": "cells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ch["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 CG / f32 V-cycle",
            "data": "synthetic (seeded lognormal field + random-walk conduits)",
            "config": {"workload": f"config2 {args.size}^3 lognormal+8 conduits",
                       "cells": n, "tol": args.tol,
                       "l2": "inputs (K 3x8 B/cell, matrix, hierarchy) larger than L2",
                       "parallelism": f"replicas x{world}"},
            "chosen_variant": chosen_name,
            **{name: {k: v for k, v in r.items() if k not in ("solver", "stream", "x")}
               for name, r in results.items()},
            "speedup_chosen_vs_plain": ch["value"] / results["plain_fp64"]["value"],
            "e2e": e2e,
            "roofline": {"bound": "hbm",
                         "kernel": "k_g7_spmv_dot2 (L0 SpMV FP64 of the CG, 7-point form, "
                                   "two x-adjacent cells per thread; algorithmic bytes 48 "
                                   "per cell)",
                         "achieved": round(achieved, 1), "peak": peak,
                         "peak_source": peak_src, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "algorithmic_bytes": by0, "ms": ms0,
                         "traffic": round(SPMV_TRAFFIC_B_PER_CELL * n),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of one launch at 192^3, scaled by cells"},
            "kernels": kernels,
            "oracle_error": oracle_error,
            "config1": config1,
            "config4": config4,
            "gpu_launches": launches["chosen"],
            "gpu_launches_per_step": launches["chosen"] / args.steps,
            "batched": batched,
            "coupled": coupled,
            "output": output,
            "cpu_baseline": cpu,
            "clocks": ch["clocks"],
        }
        print(json.dumps(line), flush=True)
    for r in results.values():
        r["solver"].close()
    s_e2e.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------ reference (CPU) ----

def _ref_worker(args_tuple):
    size, seed_off, tol = args_tuple
    from hmfem_b200.problem import config_problem
    from oracle.oracle import Ref
    p = config_problem(2, realisation=seed_off, size=size)
    t0 = time.perf_counter()
    with _QuietStdout():
        x, v, it, rel, times = Ref().solve_all(p, eps=tol)
    dt = time.perf_counter() - t0
    return p.n, dt, it, rel, list(times)


def run_batch(args, world, n_inst=96):
    """Config 3: 96 uneven instances (n ~ U{24..96} per axis, lengths n/64,
    log10 std ~ U[1,2], correlation 4 cells, 0-4 conduits at 1e-10), FP32
    V-cycle with the exact level-0 reduction in FP64 flexible CG to 1e-10,
    several solvers on their own
    streams (worker count tuned once per GPU).  Every rank solves the same
    batch (replicas); one untimed pass, then wall clock around the whole
    batch, max over ranks."""
    import torch

    from hmfem_b200 import batch as hb
    from hmfem_b200.problem import config_problem
    probs = [config_problem(3, realisation=r) for r in range(n_inst)]
    # the level-0 reduction and BF16 levels, as the chosen 256^3 variant
    opts = dict(schur0=1, bf16_from=1)
    driver, workers, tune = hb.tune(probs[:16], precision=1, tol=args.tol, options=opts)
    run = hb.DRIVERS[driver]
    # warm-up: one untimed pass over the whole batch, so the device memory
    # pool has grown to the batch's working set before the timed pass
    run(probs, 1, args.tol, workers=workers, options=opts)
    torch.cuda.synchronize()
    walls = []
    for _ in range(2):  # the better of two timed passes (every rank runs both)
        barrier(world)
        t0 = time.perf_counter()
        r = run(probs, 1, args.tol, workers=workers, options=opts)
        torch.cuda.synchronize()
        w = max_over_ranks(time.perf_counter() - t0, world)
        if not walls or w < min(walls):
            res = r
        walls.append(w)
    wall = min(walls)
    secs = np.sort([r[2] for r in res])
    return {"workload": f"config3: {n_inst} uneven instances, n ~ U{{24..96}}^3",
            "cells": int(sum(p.n for p in probs)),
            "instances_per_s": world * n_inst / wall,
            "wall_s": wall, "driver": driver, "workers": workers,
            "p50_ms": 1e3 * float(np.percentile(secs, 50)),
            "p99_ms": 1e3 * float(np.percentile(secs, 99)),
            "iterations_mean": float(np.mean([r[1]["iterations"] for r in res])),
            "iterations_min_max": [int(min(r[1]["iterations"] for r in res)),
                                   int(max(r[1]["iterations"] for r in res))],
            "max_relres": float(max(r[1]["relres"] for r in res)),
            "timing": "host wall clock around the batch (host K in, pressure out), the "
                      "better of two passes after an untimed one; per instance: its "
                      "assembly + setup + the solve it waited for",
            "passes_s": walls,
            "tuning": tune}


def _ref_instance(args_tuple):
    """One config-3 instance through the reference's own path (oracle/_ref):
    assembly + CSR + AMG setup + PCG to the tolerance; its seconds."""
    r, tol = args_tuple
    from hmfem_b200.problem import config_problem
    from oracle.oracle import Ref
    p = config_problem(3, realisation=r)
    with _QuietStdout():
        job = Ref().job(p, eps=tol)
        t0 = time.perf_counter()
        job.assemble()
        job.setup()
        job.iterate(-1)
        dt = time.perf_counter() - t0
        _, it, rel, _ = job.result(want_p=False)
        job.close()
    return dt, it, rel


def batch_cpu_baseline(tol, n_inst=96, sample=8):
    """Config 3 on the host with the reference's own code: the first
    `sample` instances one after another on one core (instances/s, p50/p99
    of their times), and all n_inst instances on independent processes, one
    per core (instances/s, core count stated)."""
    import multiprocessing as mp
    try:
        t0 = time.perf_counter()
        seq = [_ref_instance((r, tol)) for r in range(sample)]
        t_seq = time.perf_counter() - t0
        cores = max(1, min(os.cpu_count() or 1, 16))
        with mp.get_context("spawn").Pool(cores) as pool:
            pool.map(_ref_instance, [(r, tol) for r in range(cores)])   # warm-up
            t0 = time.perf_counter()
            allr = pool.map(_ref_instance, [(r, tol) for r in range(n_inst)])
            t_par = time.perf_counter() - t0
    except Exception as e:  # reference build missing
        return {"unavailable": str(e)}
    d = np.sort([x[0] for x in seq])
    return {"kind": "reference",
            "one_core": {"instances_per_s": sample / t_seq, "cores": 1,
                         "sample": f"instances 0-{sample - 1} one after another",
                         "p50_ms": 1e3 * float(np.percentile(d, 50)),
                         "p99_ms": 1e3 * float(np.percentile(d, 99))},
            "processes": {"instances_per_s": n_inst / t_par, "cores": cores,
                          "sample": f"all {n_inst} instances, one process per core",
                          "max_relres": float(max(x[2] for x in allr))}}


class _QuietStdout:
    """Sends file descriptor 1 to /dev/null while the reference's own C code
    runs (fluxos prints its divergence bounds), so stdout keeps one JSON
    line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def coupled_case():
    """The reference's own coupled run (roda.sh: 210 x 42 x 20 cells on
    210 x 210 x 100 m, homogeneous K = 1e-13, conduit file data_1_2.dat,
    well column (105, 21, z >= 10) at 10 MPa, main.c constants)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import karst_cases as KC

    from hmfem_b200.karst import Karst
    prob = KC.reservoir(210, 42, 20, 1.0, 5.0, 5.0)
    WI, pw = KC.well(prob, 105, 21, 10)
    k = Karst.read(os.path.join(ROOT, "tests", "golden", "karst_data_1_2.dat"), 1)
    return prob, k, WI, pw, KC.RHO


def run_coupled(args, world, rank, reps=3):
    """The Picard loop of main.c:383-489 through hmfem_picard (host K, WI,
    pw in; reservoir and conduit pressures out), the chosen solver (FP32
    V-cycle with the exact level-0 reduction in FP64 flexible CG) to
    ||r||/||b|| <= 1e-10 per reservoir solve, Picard tolerance 1e-8; wall
    clock per run (1 warm-up, median of `reps`), max over ranks."""
    import torch

    from hmfem_b200 import gpu, karst
    prob, k, WI, pw, rho = coupled_case()
    s = gpu.Solver(precision=1, schur0=1, bf16_from=1, tol=1e-10, stop_rule=0)
    karst.picard(s, k, prob, WI, pw, rho=rho, fluxes=False)  # warm-up
    torch.cuda.synchronize()
    barrier(world)
    walls, r = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        r = karst.picard(s, k, prob, WI, pw, rho=rho, fluxes=False)
        walls.append(time.perf_counter() - t0)
    s.close()
    wall = max_over_ranks(float(np.median(walls)), world)
    st = r["stats"]
    out = {"workload": "reference run script case: 210x42x20 reservoir + 1 conduit "
                       "(data_1_2.dat: 123 elements, nonlinear Robin ends, 2 fractures) "
                       "+ well column",
           "cells": prob.n, "picard_iterations": st["iterations"],
           "picard_error": st["error"], "cg_iterations": st["cg_iterations"],
           "amg_setups": st["setups"], "wall_ms": 1e3 * wall,
           "device_setup_ms": st["t_setup_ms"], "device_loop_ms": st["t_loop_ms"],
           "timing": "host wall clock around hmfem_picard, host arrays in and out"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_reference"] = coupled_cpu_sample(prob, k, WI, pw, rho)
        per = out["cpu_reference"].get("s_per_iteration")
        if per:
            est = out["cpu_reference"]["first_solve_s"] + per * st["iterations"]
            out["cpu_reference"]["full_run_estimate_s"] = est
            out["speedup_vs_reference_estimate"] = est / wall
    return out


def run_output(args, prob, solver, p, world):
    """The reference's result files of this solve (save_pressure,
    save_flux, vts_StructuredGrid_file) from the GPU writers
    (include/hmfem_textio.h), host pressure and fluxes in.  Timed writing to
    /dev/null (formatting + copies + the write call: what the writers
    themselves cost) and, once, to a scratch directory (adds the disk); the
    reference's own writers (oracle/_ref) on a 64^3 sample, also into
    /dev/null, scaled per byte."""
    import ctypes as C
    import shutil
    import tempfile

    from hmfem_b200 import gpu
    L = gpu.lib()
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.hmfem_save_pressure.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, i]
    L.hmfem_save_flux.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, i]
    L.hmfem_save_vts.argtypes = [C.c_char_p, i, i, i, d, d, d, vp, vp, i]
    v, _, _ = solver.fluxes(p, np.zeros((prob.n, 7)))
    g = (prob.nx, prob.ny, prob.nz, prob.hx, prob.hy, prob.hz)
    pp, pv = C.c_void_p(p.ctypes.data), C.c_void_p(v.ctypes.data)
    calls = {"pressure_reservoir.dat": lambda f: L.hmfem_save_pressure(f, *g, pp, 0),
             "flux_reservoir.dat": lambda f: L.hmfem_save_flux(f, *g, pv, 0),
             "campos.vts": lambda f: L.hmfem_save_vts(f, *g, pv, pp, 0)}
    d_out = tempfile.mkdtemp(prefix="hmfem_out_")
    res = {}
    try:
        calls["pressure_reservoir.dat"](os.devnull.encode())  # warm-up
        for name, fn in calls.items():
            t0 = time.perf_counter()
            rc = fn(os.devnull.encode())
            dt = time.perf_counter() - t0
            path = os.path.join(d_out, name)
            t1 = time.perf_counter()
            fn(path.encode())
            dd = time.perf_counter() - t1
            size = os.path.getsize(path)
            os.remove(path)
            res[name] = {"rc": rc, "s": dt, "bytes": size, "MB_per_s": size / dt / 1e6,
                         "to_disk_s": dd}
    finally:
        shutil.rmtree(d_out, ignore_errors=True)
    out = {"workload": f"result files of the {prob.nx}^3 solve (host arrays in)", "files": res,
           "timing": "host wall clock per file written to /dev/null; to_disk_s: the same "
                     "into a scratch directory (bound by the box's disk)"}
    if not args.no_cpu_baseline:
        out["cpu_reference"] = output_cpu_sample()
        tot_gpu = sum(r["s"] for r in res.values())
        tot_bytes = sum(r["bytes"] for r in res.values())
        per = out["cpu_reference"].get("s_per_byte")
        if per:
            out["cpu_reference"]["estimate_s"] = per * tot_bytes
            out["speedup_vs_reference_estimate"] = per * tot_bytes / tot_gpu
    return out


def output_cpu_sample(size=64):
    """The reference's save_pressure + save_flux + vts_StructuredGrid_file
    (oracle/_ref) on a size^3 field, one core, into files that are links to
    /dev/null (bytes counted from one run into real files)."""
    import ctypes as C
    import tempfile
    try:
        from oracle.oracle import REF_SO
        L = C.CDLL(REF_SO)
        L.ref_save_grid.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    except Exception as e:  # reference build missing
        return {"unavailable": str(e)}
    n = size ** 3
    rng = np.random.default_rng(0)
    p = 6e7 * (1 + 0.01 * rng.standard_normal(n))
    v = rng.standard_normal((n, 7)) * 1e-7
    names = ("pressure_reservoir.dat", "flux_reservoir.dat", "campos.vts")
    args = (size, size, size, 1.0 / size, 1.0 / size, 1.0 / size, p.ctypes.data, v.ctypes.data)
    with tempfile.TemporaryDirectory() as d:
        L.ref_save_grid(d.encode(), *args)
        nbytes = sum(os.path.getsize(os.path.join(d, f)) for f in names)
    with tempfile.TemporaryDirectory() as d:
        for f in names:
            os.symlink(os.devnull, os.path.join(d, f))
        t0 = time.perf_counter()
        L.ref_save_grid(d.encode(), *args)
        dt = time.perf_counter() - t0
    return {"kind": "reference", "cores": 1, "s": dt, "bytes": nbytes, "s_per_byte": dt / nbytes,
            "sample": f"save_pressure + save_flux + vts_StructuredGrid_file at {size}^3 "
                      f"into /dev/null"}


def coupled_cpu_sample(prob, k, WI, pw, rho, iters=2):
    """The reference's own coupled loop (oracle/_ref: its reservoir(),
    conduit(), compute()) for the first `iters` Picard iterations, 1 core."""
    try:
        from oracle.oracle import Ref
        R = Ref()
        with _QuietStdout():
            r0 = R.picard(k, prob, WI, pw, rho=rho, iter_max=0)
            r2 = R.picard(k, prob, WI, pw, rho=rho, iter_max=iters)
    except Exception as e:  # reference build missing
        return {"unavailable": str(e)}
    per = (r2["seconds"] - r0["seconds"]) / iters
    return {"kind": "reference", "cores": 1, "first_solve_s": r0["seconds"],
            "s_per_iteration": per,
            "sample": f"first reservoir solve + {iters} Picard iterations of the "
                      f"reference's loop ({r2['seconds']:.1f} s)"}


def cpu_baseline_sample(size, cores=1, tol=1e-10):
    """The reference's CPU path (oracle/_ref) on one sample of the workload."""
    try:
        n, dt, it, rel, times = _ref_worker((size, 0, tol))
    except Exception as e:  # reference build missing
        return {"value": None, "unavailable": str(e)}
    return {"value": n / dt, "unit": "cells/s", "cores": cores,
            "kind": "reference",
            "sample": f"config2 generator at {size}^3 (same distribution), "
                      f"full reference path: assembly + CSR + AMG setup + "
                      f"PCG to true relres {tol} + flux; {it} iterations, "
                      f"{dt:.1f} s",
            "split_s": dict(zip(["assemble", "setup", "solve", "flux", "total"],
                                [round(t, 3) for t in times]))}


FACES = [0, 1, 2, 3, 5, 6]   # u, d, l, r, t, b of an ELE row (c unused)


def _mem_available_gb():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


ORACLE_TOL = 1e-12   # the FP64 oracle's true relative residual


def _ref_full_worker(size, tol, outdir):
    """The reference's own path (oracle/_ref, the ref_job_* steps of
    ref_solve_all) on the config-2 problem of this size, timed to the bench
    tolerance; then the same CG continued (untimed) to ORACLE_TOL, and the
    fluxes of that solution.  Writes pressure, six face fluxes, timings."""
    from hmfem_b200.problem import config_problem
    from oracle.oracle import Ref
    p = config_problem(2, size=size)
    with _QuietStdout():
        job = Ref().job(p, eps=tol)
        job.assemble()
        job.setup()
        job.iterate(-1)
        _, it, rel, times = job.result(want_p=False)
        job.set_eps(ORACLE_TOL)
        job.iterate(-1)
        v = np.zeros((p.n, 7))
        job.flux(v)
    x, it_o, rel_o, _ = job.result()
    job.close()
    np.save(os.path.join(outdir, "p.npy"), x)
    np.save(os.path.join(outdir, "v.npy"), np.ascontiguousarray(v[:, FACES]))
    json.dump({"n": p.n, "iterations": it, "relres": rel, "times": list(times),
               "oracle_iterations": it_o, "oracle_relres": rel_o},
              open(os.path.join(outdir, "meta.json"), "w"))


def start_reference_full(size, tol, need_gb=24.0):
    """Starts _ref_full_worker in a spawned process (one host core).  None
    when the host has too little free memory for it (~13 GB at 256^3)."""
    import multiprocessing as mp
    import tempfile
    if _mem_available_gb() < need_gb * (size / 256.0) ** 3:
        return {"unavailable": f"host memory: {_mem_available_gb():.0f} GB available"}
    d = tempfile.mkdtemp(prefix="hmfem_ref_")
    proc = mp.get_context("spawn").Process(target=_ref_full_worker, args=(size, tol, d),
                                           daemon=True)
    t0 = time.perf_counter()
    proc.start()
    return {"proc": proc, "dir": d, "t0": t0, "size": size, "tol": tol}


def finish_reference_full(ref, timeout=1500):
    """Waits for start_reference_full's process; returns (cpu_baseline dict,
    pressure, face fluxes) or (dict with the reason, None, None)."""
    import shutil
    if "proc" not in ref:
        return {"value": None, "unavailable": ref.get("unavailable")}, None, None
    proc, d = ref["proc"], ref["dir"]
    proc.join(timeout)
    try:
        if proc.is_alive() or proc.exitcode != 0:
            if proc.is_alive():
                proc.terminate()
            return {"value": None, "unavailable": f"reference process exit {proc.exitcode}"}, \
                None, None
        meta = json.load(open(os.path.join(d, "meta.json")))
        p = np.load(os.path.join(d, "p.npy"))
        v = np.load(os.path.join(d, "v.npy"))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    t = meta["times"]
    size = ref["size"]
    cpu = {"value": meta["n"] / (t[0] + t[1] + t[2]), "unit": "cells/s", "cores": 1,
           "kind": "reference",
           "sample": f"the bench's own config2 {size}^3 problem, one full solve: assembly + "
                     f"CSR + AMG setup + PCG to true relres {ref['tol']} "
                     f"({meta['iterations']} iterations), the reference's sources "
                     f"(oracle/_ref), on one host core beside the GPU arms",
           "split_s": dict(zip(["assemble", "setup", "solve"], [round(x, 2) for x in t[:3]])),
           "iterations": meta["iterations"], "relres": meta["relres"],
           "oracle": f"the same CG continued to true relres {meta['oracle_relres']:.2e} "
                     f"({meta['oracle_iterations']} iterations), untimed: the FP64 "
                     f"solution oracle_error compares with"}
    return cpu, p, v


def pressure_flux_error(solver, x, prob, ref_p, ref_v, dev):
    """Pressure and six face fluxes of a GPU solution against the
    reference's: relative 2-norm errors, and the divvel_pontual maximum
    |div u| relative to the largest face flux over h."""
    import torch
    p = x.to(torch.float64)
    v = torch.zeros((prob.n, 7), dtype=torch.float64, device=dev)
    _, dmin, dmax = solver.fluxes(p, v)
    ph = p.cpu().numpy()
    vh = v[:, FACES].cpu().numpy()
    scale = float(np.abs(ref_v).max()) / min(prob.hx, prob.hy, prob.hz)
    out = {"p_rel": float(np.linalg.norm(ph - ref_p) / np.linalg.norm(ref_p)),
           "flux_rel": float(np.linalg.norm(vh - ref_v) / np.linalg.norm(ref_v)),
           "divmax": dmax, "divmax_rel": dmax / scale if scale > 0 else None}
    del vh
    return out


def _time_steps(s, prob, K, stream, steps, warmup, x):
    import torch
    for _ in range(warmup):
        s.assemble(prob, KX=K, KY=K, KZ=K)
        s.setup()
        with torch.cuda.stream(stream):
            x.zero_()
        s.solve(x=x)
    times, st = [], None
    for _ in range(steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.assemble(prob, KX=K, KY=K, KZ=K)
        s.setup()
        with torch.cuda.stream(stream):
            x.zero_()
        _, st = s.solve(x=x)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.mean(times)), st


def run_config1(args, dev, steps=5, warmup=3):
    """Config 1: 128^3, K = 1e-14 + 4 conduits at 1e-10; the plain FP64
    drop-in against the chosen FP32 V-cycle (level-0 reduction, BF16 levels
    >= 1) in FP64 flexible CG, both to ||r||/||b|| <= tol; K resident, CUDA
    events per step (assembly + setup + solve)."""
    import torch

    from hmfem_b200 import gpu
    from hmfem_b200.problem import config_problem
    prob = config_problem(1)
    K = torch.tensor(prob.KX, device=dev)
    out = {"workload": "config1 128^3, 4 conduits at 1e-10", "cells": prob.n}
    for name, prec in (("plain_fp64", 0), ("fp32_chosen", 1)):
        s = gpu.Solver(precision=prec, tol=args.tol, check_every=2,
                       bf16_from=1 if prec == 1 else -1, schur0=prec)
        stream = torch.cuda.ExternalStream(s.stream)
        x = torch.zeros(prob.n, dtype=torch.float64, device=dev)
        ms, st = _time_steps(s, prob, K, stream, steps, warmup, x)
        out[name] = {"ms_per_step": ms, "cells_per_s": prob.n / (ms / 1e3),
                     "iterations": st["iterations"], "relres": st["relres"],
                     "setup_ms": st["t_setup_ms"], "solve_ms": st["t_solve_ms"]}
        s.close()
    out["speedup_chosen_vs_plain"] = out["plain_fp64"]["ms_per_step"] / out["fp32_chosen"]["ms_per_step"]
    return out


def run_config4(args, dev, model, seeds=range(2048, 2056)):
    """Config 4 on held-out seeds: 128^3 lognormal (std 1.5, correlation 8)
    with 0-6 conduits; the chosen solver from the zero guess and from the
    learned guess (inference inside the timed step), both to tol; CUDA
    events per solve, K resident."""
    import torch

    from hmfem_b200 import gpu, guess
    from hmfem_b200.problem import config_problem
    s = gpu.Solver(precision=1, tol=args.tol, check_every=2, bf16_from=1, schur0=1)
    stream = torch.cuda.ExternalStream(s.stream)
    rows = []
    for sd in seeds:
        prob = config_problem(4, realisation=sd)
        K = torch.tensor(prob.KX, device=dev)
        mask = torch.as_tensor(prob.conduit_mask, device=dev)
        dims = (prob.nx, prob.ny, prob.nz)
        x = torch.zeros(prob.n, dtype=torch.float64, device=dev)
        r = {"zero": [], "net": []}
        # one untimed pass of each, then three timed passes alternating
        for rep, mode in enumerate(("zero", "net") * 4):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.assemble(prob, KX=K, KY=K, KZ=K)
            s.setup()
            with torch.cuda.stream(stream):   # the solver's stream: ordered
                if mode == "net":
                    x.copy_(guess.predict(model, K, mask, dims))
                else:
                    x.zero_()
            _, st = s.solve(x=x)
            e1.record(stream)
            e1.synchronize()
            if rep >= 2:
                r[mode].append((e0.elapsed_time(e1), st["iterations"], st["relres"]))
        rows.append(r)
    s.close()

    def agg(mode):
        ms = [min(t[0] for t in r[mode]) for r in rows]   # per seed: best of three
        return {"iterations_mean": float(np.mean([r[mode][0][1] for r in rows])),
                "ms_median": float(np.median(ms)), "ms_mean": float(np.mean(ms))}
    return {"workload": f"config4 128^3, held-out seeds {seeds[0]}-{seeds[-1]}",
            "zero_guess": agg("zero"), "learned_guess": agg("net"),
            "max_relres": float(max(t[2] for r in rows for m in r for t in r[m])),
            "timing": "CUDA events per solve (assembly + setup + [inference] + solve), "
                      "per seed the best of three passes (alternating), after one "
                      "untimed pass of each"}


def ref_plan(steps, est_iters=56):
    """The reference's path for one problem -- what the GPU step times:
    assembly + CSR, AMG setup + CG start, CG to the tolerance -- split into
    `steps` parts run in order: the CG in chunks of iterations, the last
    part finishing it."""
    if steps <= 1:
        return [["assemble", "setup", ("iterate", -1)]]
    if steps == 2:
        return [["assemble", "setup"], [("iterate", -1)]]
    if steps == 3:
        return [["assemble"], ["setup"], [("iterate", -1)]]
    chunks = steps - 3
    c = -(-est_iters // (chunks + 1))
    return [["assemble"], ["setup"]] + [[("iterate", c)] for _ in range(chunks)] + \
        [[("iterate", -1)]]


def _ref_replica(conn, size, tol, plan):
    """One replica of the reference arm: builds the problem and a reference
    job, then runs the plan's parts on command ("warm", step index,
    "result", "quit")."""
    from hmfem_b200.problem import config_problem
    from oracle.oracle import Ref
    R = Ref()
    p = config_problem(2, size=size)
    job = R.job(p, eps=tol)
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg == "quit":
            break
        if msg == "warm":      # pages the library and its code in
            with _QuietStdout():
                R.solve_all(config_problem(2, size=24), eps=tol)
            conn.send("ok")
        elif msg == "result":
            _, it, rel, times = job.result(want_p=False)
            conn.send((it, rel, list(times)))
        else:
            with _QuietStdout():
                for op in plan[msg]:
                    if op == "assemble":
                        job.assemble()
                    elif op == "setup":
                        job.setup()
                    elif op == "flux":
                        job.flux()
                    else:
                        job.iterate(op[1])
            conn.send("ok")
    job.close()


def run_reference(args):
    """The reference's own CPU path (oracle/_ref) on the bench's own
    configuration: the config-2 problem of --size (256^3), assembly + CSR +
    AMG setup + PCG to the true relative residual --tol + fluxes.  The host
    cores run independent replicas of that solve (the reference is single
    threaded; as many replicas as cores and free memory allow, ~13 GB
    each at 256^3), stepped in lockstep: step i runs part i of ref_plan on
    every replica, so the K timed steps are exactly one full solve per
    replica.  W warm-up steps run a 24^3 solve per replica.  value = replicas
    x cells / time of the K steps."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    import multiprocessing as mp
    size = args.size
    per_gb = 14.0 * (size / 256.0) ** 3 + 0.5
    cores = os.cpu_count() or 1
    reps = max(1, min(cores, 16, int(0.7 * _mem_available_gb() / per_gb)))
    plan = ref_plan(args.steps)
    ctx = mp.get_context("spawn")
    procs, conns = [], []
    for _ in range(reps):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_replica, args=(b, size, args.tol, plan), daemon=True)
        pr.start()
        procs.append(pr)
        conns.append(a)
    for c in conns:
        c.recv()
    for _ in range(args.warmup):
        for c in conns:
            c.send("warm")
        for c in conns:
            c.recv()
    step_s = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        ts = time.perf_counter()
        for c in conns:
            c.send(i)
        for c in conns:
            c.recv()
        step_s.append(time.perf_counter() - ts)
    dt = time.perf_counter() - t0
    for c in conns:
        c.send("result")
    res = [c.recv() for c in conns]
    for c in conns:
        c.send("quit")
    for pr in procs:
        pr.join(60)
    n = size ** 3
    value = reps * n / dt
    its = sorted({r[0] for r in res})
    line = {"impl": "reference", "metric": METRIC, "value": value,
            "unit": "cells/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded lognormal field + random-walk conduits)",
            "config": {"workload": f"config2 {size}^3 lognormal+8 conduits",
                       "cells": n, "tol": args.tol,
                       "l2": "inputs (K 3x8 B/cell, matrix, hierarchy) larger than L2",
                       "parallelism": f"replicas x{reps} (host cores)"},
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": reps,
                             "kind": "reference",
                             "sample": f"{reps} independent replicas of the full {size}^3 "
                                       f"solve, one per host core, in lockstep: the "
                                       f"{args.steps} steps are one complete solve per "
                                       f"replica (assembly + CSR + AMG setup + PCG to true "
                                       f"relres {args.tol}; {its} iterations), "
                                       f"the reference's sources (oracle/_ref); warm-up: "
                                       f"a 24^3 solve per replica per warm-up step",
                             "split_s_replica0": dict(zip(
                                 ["assemble", "setup", "solve", "flux", "total"],
                                 [round(x, 2) for x in res[0][2]])),
                             "step_s": [round(x, 2) for x in step_s],
                             "max_relres": max(r[1] for r in res)},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_step(args):
    import torch

    from hmfem_b200 import gpu
    from hmfem_b200.problem import config_problem
    prob = config_problem(2, size=args.size)
    K = torch.tensor(prob.KX, device="cuda")
    # the options of the bench's variants: plain FP64, or the FP32 V-cycle
    # with levels >= 1 stored in BF16 (from the zero or the learned guess)
    fp32 = args.profile_step >= 1
    s = gpu.Solver(precision=1 if fp32 else 0, tol=args.tol,
                   bf16_from=1 if fp32 else -1, check_every=2, schur0=1 if fp32 else 0)
    x = torch.zeros(prob.n, dtype=torch.float64, device="cuda")
    if args.profile_step == 2:
        from hmfem_b200 import guess
        model = guess.load(os.path.join(ROOT, "hmfem_b200", "models", "unet_config4.npz"))
        mask = torch.as_tensor(prob.conduit_mask, device="cuda")
        _, st = guess.solve_from_guess(s, prob, model, K, mask=mask, x=x)
    else:
        s.assemble(prob, KX=K, KY=K, KZ=K)
        s.setup()
        _, st = s.solve(x=x)
    torch.cuda.synchronize()
    print(json.dumps({"profile_step": args.profile_step, "size": args.size,
                      "iterations": st["iterations"], "relres": st["relres"],
                      "launches": gpu.launch_count()}))


def main():
    args = parse()
    if args.profile_step >= 0:
        profile_step(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
