"""Many independent pressure solves of uneven grids on one GPU.

Each worker thread owns one solver (its own CUDA stream, allocation cache
and captured CG graph) and takes instances from a shared queue: assembly
from the host K arrays, AMG setup, solve to the tolerance, pressure back
to the host.  Instances of 24^3..96^3 cells leave most of a B200 idle when
run one after another (their kernels are small and the setup is
launch-bound), so several streams in flight fill it; the number of workers
is measured once per GPU model and precision by `tune_workers` and kept in
a small JSON file.  Every instance converges on its own (its own control
block), so no instance waits for the slowest one.
"""
import json
import os
import queue
import threading
import time

import numpy as np

from . import gpu

_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "hmfem_b200",
                      "batch_workers.json")


def _gpu_key(precision):
    try:
        import torch
        name = torch.cuda.get_device_name(0)
    except Exception:  # pragma: no cover - torch without CUDA
        name = "gpu"
    return f"{name}|precision={precision}"


def solve_batch(problems, precision=1, tol=1e-10, workers=4, options=None):
    """Solves every problem; returns [(x, stats, seconds)] in input order.

    seconds is the instance's wall time in its worker (assembly + setup +
    solve + copies).  options: extra hmfem_options fields."""
    opts = dict(precision=precision, tol=tol)
    opts.update(options or {})
    jobs = queue.Queue()
    for i, p in enumerate(problems):
        jobs.put((i, p))
    out = [None] * len(problems)
    errors = []

    def work():
        s = gpu.Solver(**opts)
        try:
            while True:
                try:
                    i, p = jobs.get_nowait()
                except queue.Empty:
                    return
                t0 = time.perf_counter()
                s.assemble(p)
                s.setup()
                x = np.zeros(p.n)
                _, st = s.solve(x=x)
                out[i] = (x, st, time.perf_counter() - t0)
        except Exception as e:  # reported to the caller below
            errors.append(e)
        finally:
            s.close()

    threads = [threading.Thread(target=work) for _ in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out


def tune_workers(sample, precision=1, tol=1e-10, candidates=(1, 2, 4, 8, 12),
                 cache=_CACHE, refresh=False, options=None):
    """Worker count with the highest instance throughput on `sample`
    (warmed up once), remembered per GPU model, precision and options in
    `cache`."""
    key = _gpu_key(precision) + "".join(f"|{k}={v}" for k, v in sorted((options or {}).items()))
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if not refresh and key in table:
        return int(table[key]["workers"]), table[key]
    solve_batch(sample[:2], precision, tol, workers=2, options=options)  # warm-up
    rates = {}
    for w in candidates:
        t0 = time.perf_counter()
        solve_batch(sample, precision, tol, workers=w, options=options)
        rates[w] = len(sample) / (time.perf_counter() - t0)
    best = max(rates, key=rates.get)
    entry = {"workers": best, "instances_per_s": rates, "sample": len(sample)}
    table[key] = entry
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        except OSError:
            pass
    return best, entry
