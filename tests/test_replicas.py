"""Multi-replica serving on CPU ranks (gloo, world size 2) with fake workers: the request
assignment, the gathered records, and host-side fault injection (a replica that raises has its
requests re-run on the others; a rank that leaves makes the others' next collective fail within
the process-group timeout)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dmff_b200.serving import assign_requests, serve_replicated


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _stream(n=24, seed=0):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(300, 3000, size=n)
    return [{"n_atoms": int(a)} for a in sizes], np.cumsum(rng.exponential(0.001, size=n))


def fake_run(fail_rank=None):
    def run_local(systems, arrivals):
        if dist.get_rank() == fail_rank:
            raise RuntimeError("injected replica failure")
        return [{"n_atoms": s["n_atoms"], "latency": 1e-6 * s["n_atoms"], "rank": dist.get_rank()} for s in systems]
    return run_local


def _worker(rank, world, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    systems, arrivals = _stream()
    try:
        if mode == "ok":
            recs, summ = serve_replicated(systems, arrivals, fake_run())
        elif mode == "raise":
            recs, summ = serve_replicated(systems, arrivals, fake_run(fail_rank=1))
        else:  # rank 1 leaves between steps: the survivor's collective must fail, not hang
            if rank == 1:
                dist.destroy_process_group()
                out.put((rank, "left", None))
                return
            try:
                serve_replicated(systems, arrivals, fake_run())
                out.put((rank, "no-error", None))
            except Exception as e:
                out.put((rank, "error", type(e).__name__))
            return
        out.put((rank, "done", (recs, summ)))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    return sorted(res, key=lambda x: x[0])


def test_assignment_balances_atoms_and_is_deterministic():
    systems, _ = _stream(200, seed=3)
    a = assign_requests([s["n_atoms"] for s in systems], 4)
    assert a == assign_requests([s["n_atoms"] for s in systems], 4)
    load = np.bincount(a, weights=[s["n_atoms"] for s in systems], minlength=4)
    assert load.max() - load.min() <= max(s["n_atoms"] for s in systems)


def test_two_replicas_serve_every_request_once():
    res = _run("ok")
    for rank, kind, payload in res:
        recs, summ = payload
        assert kind == "done" and summ["completed"] == 24 and summ["failed_ranks"] == []
        assert [r["index"] for r in recs] == list(range(24))
        assert {r["rank"] for r in recs} == {0, 1}


def test_failed_replica_requests_are_rerun_on_the_survivor():
    res = _run("raise")
    recs, summ = res[0][2]
    assert summ["failed_ranks"] == [1] and summ["redistributed"] > 0 and summ["completed"] == 24
    assert {r["rank"] for r in recs} == {0}
    assert "injected replica failure" in summ["errors"][0]


def test_rank_leaving_fails_the_survivors_collective():
    res = dict((r, (k, p)) for r, k, p in _run("leave"))
    assert res[1][0] == "left"
    assert res[0][0] == "error"
