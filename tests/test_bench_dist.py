"""The multi-process plumbing of bench.py on the host (gloo, two ranks):
the barrier, the max over ranks that every time goes through, and the
reference arm, which only rank 0 runs."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    r, w, _ = bench.dist_init(None)
    bench.barrier(w)
    # every rank reports its own time; all must agree on the slowest
    m = bench.max_over_ranks(0.5 + r, w)
    bench.barrier(w)
    q.put((r, w, m, dist.get_backend()))
    dist.destroy_process_group()


def test_two_ranks_take_the_max_over_ranks():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("host test (gloo)")
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 1.5, "gloo"), (1, 2, 1.5, "gloo")]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(None)   # returns before reading its arguments
    assert buf.getvalue() == ""
