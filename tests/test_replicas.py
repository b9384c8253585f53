"""The replica plumbing (cudec_b200/replicas.py) across two processes on CPU
with gloo: the timing reduction is the maximum over ranks, the aggregate is
every rank's work over that time, and a rank that never reaches the collective
turns into an error on the other rank within the group's timeout instead of a
hang."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from cudec_b200 import replicas
    try:
        replicas.init("gloo", timeout_s=5 if mode == "drop" else 60)
        if mode == "drop" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()  # the message is out before the process goes
            os._exit(0)  # leaves between steps, before the collective
        t = replicas.max_over_ranks(1.0 + rank)
        q.put((rank, ("ok", t, replicas.aggregate_rate(100.0, t, world))))
        replicas.finish()
    except Exception as e:  # the surviving rank reports the failure
        q.put((rank, ("error", type(e).__name__)))


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_max_over_ranks_and_aggregate_with_gloo():
    out = _run("ok")
    for r in (0, 1):
        status, t, rate = out[r]
        assert status == "ok" and t == 2.0 and rate == pytest.approx(100.0)


def test_a_rank_that_leaves_is_an_error_not_a_hang():
    out = _run("drop")
    assert out[1] == "left"
    assert out[0][0] == "error"
