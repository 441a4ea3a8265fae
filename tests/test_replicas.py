"""The multi-process path of the benchmark on CPU (athenak_b200/replicas.py, gloo, world
size 2, rendezvous on 127.0.0.1): the barrier, the largest time over the ranks on every rank,
the whole-job throughput (all ranks' units over the slowest rank's time); a rank that leaves
before the barrier makes the other rank's barrier end with an error after the group's short
timeout (no wait for ever); the reference arm prints on rank 0 only."""
import contextlib
import io
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from athenak_b200.replicas import Replicas
    try:
        rep = Replicas(world, rank, backend="gloo", timeout_s=5)
        if mode == "leave" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()                  # (the message leaves before the process does)
            os._exit(0)                      # gone before the barrier, nothing in flight
        rep.barrier()
        t = rep.max_over_ranks(10.0 + 5.0 * rank)
        rate = rep.throughput(1000, t)
        rep.barrier()
        rep.close()
        q.put((rank, (t, rate)))
    except Exception as e:                   # the failure the other ranks learn of
        q.put((rank, "error: " + type(e).__name__))


def run_ranks(mode, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, v = q.get(timeout=timeout)
        out[r] = v
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return out


def test_barrier_max_and_throughput_over_two_ranks():
    out = run_ranks("normal")
    for r in (0, 1):
        t, rate = out[r]
        assert t == 15.0                     # the slower rank's time, on both ranks
        assert rate == pytest.approx(2 * 1000 / 0.015)


def test_a_rank_that_leaves_ends_the_others_barrier_with_an_error():
    out = run_ranks("leave")
    assert out[1] == "left"
    assert isinstance(out[0], str) and out[0].startswith("error")


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    from athenak_b200.replicas import Replicas
    rep = Replicas(1, 0)
    rep.barrier()
    assert rep.max_over_ranks(3.5) == 3.5
    assert rep.throughput(100, 50.0) == pytest.approx(2000.0)
    rep.close()


def test_reference_arm_prints_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup, gpus = 1, 1, 2
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(A(), 1, 2)
    assert buf.getvalue() == ""
