"""Many independent pressure solves of uneven grids on one GPU.

Two drivers:

* `solve_batch_graph` (the default of the bench): every instance is
  assembled and set up by one of `workers` threads (a solver per instance,
  its own stream and allocation cache), then all instances are solved
  together by `hmfem_batch_solve`: one CUDA graph holds one CG iteration of
  every instance -- its V-cycle included -- each on a branch of its own, and
  is replayed until every instance has converged.  A converged instance's
  kernels return at once (its own control block): a per-instance
  convergence mask, each instance stopping at its own tolerance with the
  result it gives solved alone.
* `solve_batch`: each worker thread solves whole instances one after
  another on its own solver (the batch solve of round one, kept for
  comparison).

Instances of 24^3..96^3 cells leave most of a B200 idle when run one after
another (their kernels are small and the setup is launch-bound); the
worker count and the driver are measured once per GPU model, precision and
options by `tune` and kept in a small JSON file.
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


# Solvers of the graph driver, kept between batches (per options): a
# solver's stream, pinned control block and allocation cache are made once
# and its buffers reused by the next instance set up on it.
_POOLS = {}
_POOL_LOCK = threading.Lock()


def _pool(opts, m):
    key = json.dumps(opts, sort_keys=True)
    with _POOL_LOCK:
        pool = _POOLS.setdefault(key, [])
        while len(pool) < m:
            pool.append(gpu.Solver(**opts))
        return pool[:m]


def release_pools():
    """Closes the solvers the graph driver keeps between batches."""
    with _POOL_LOCK:
        for pool in _POOLS.values():
            for s in pool:
                s.close()
        _POOLS.clear()


def solve_batch_graph(problems, precision=1, tol=1e-10, workers=8, options=None):
    """Sets every problem up on `workers` threads (each on a solver of the
    pool kept for these options), then solves them all with one batched
    graph (hmfem_batch_solve); returns [(x, stats, seconds)] in input order,
    seconds = the instance's assembly + setup in its worker + the batched
    solve (which every instance waits for)."""
    opts = dict(precision=precision, tol=tol)
    opts.update(options or {})
    solvers = _pool(opts, len(problems))
    jobs = queue.Queue()
    for i, p in enumerate(problems):
        jobs.put((i, p))
    t_setup = [0.0] * len(problems)
    errors = []

    def work():
        try:
            while True:
                try:
                    i, p = jobs.get_nowait()
                except queue.Empty:
                    return
                t0 = time.perf_counter()
                solvers[i].assemble(p)
                solvers[i].setup()
                t_setup[i] = time.perf_counter() - t0
        except Exception as e:  # reported to the caller below
            errors.append(e)

    threads = [threading.Thread(target=work) for _ in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    xs = [np.zeros(p.n) for p in problems]
    t0 = time.perf_counter()
    stats = gpu.batch_solve(solvers, xs)
    t_solve = time.perf_counter() - t0
    return [(xs[i], stats[i], t_setup[i] + t_solve) for i in range(len(problems))]


DRIVERS = {"graph": solve_batch_graph, "threads": solve_batch}


def tune(sample, precision=1, tol=1e-10, candidates=(2, 4, 8, 12), drivers=("graph", "threads"),
         cache=_CACHE, refresh=False, options=None):
    """The driver and worker count with the highest instance throughput on
    `sample` (each combination: one untimed pass, then the better of two
    timed ones), remembered per GPU model, precision and options in `cache`.
    Returns (driver, workers, entry)."""
    key = "tune|" + _gpu_key(precision) + "".join(
        f"|{k}={v}" for k, v in sorted((options or {}).items()))
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if not refresh and key in table:
        e = table[key]
        return e["driver"], int(e["workers"]), e
    rates = {}
    for d in drivers:
        for w in candidates:
            # an untimed pass builds this candidate's solvers and grows their
            # memory pools; then the better of two timed passes
            DRIVERS[d](sample, precision, tol, workers=w, options=options)
            best = 0.0
            for _ in range(2):
                t0 = time.perf_counter()
                DRIVERS[d](sample, precision, tol, workers=w, options=options)
                best = max(best, len(sample) / (time.perf_counter() - t0))
            rates[f"{d}/{w}"] = best
    best = max(rates, key=rates.get)
    d, w = best.split("/")
    entry = {"driver": d, "workers": int(w), "instances_per_s": rates, "sample": len(sample)}
    table[key] = entry
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        except OSError:
            pass
    return d, int(w), entry


def tune_workers(sample, precision=1, tol=1e-10, candidates=(1, 2, 4, 8, 12),
                 cache=_CACHE, refresh=False, options=None):
    """Worker count of the `solve_batch` driver with the highest instance
    throughput on `sample` (warmed up once), remembered per GPU model,
    precision and options in `cache`."""
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
