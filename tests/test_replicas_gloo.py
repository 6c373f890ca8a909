"""The multi-GPU path of bench.py (independent replicas, the timings reduced
with a MAX over ranks) with world_size 2 on the CPU (gloo), and failure
detection on the host: a rank that never joins the collective makes the other
one's call end with an error after the process group's short timeout (no GPU
is involved; nothing faults or hangs a device)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, mode, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from quantizer_b200 import replicas
    try:
        replicas.init("gloo", timeout_s=10.0)
        w, r, _ = replicas.env()
        ms = 100.0 + 50.0 * r  # rank 1 is the slow one
        if mode == "absent" and r == 1:
            out[r] = "left"
            return  # leaves between steps, before the collective, without finishing
        m = replicas.max_over_ranks(ms)
        rate = replicas.whole_job_rate(1000.0, 10, m, w)
        out[r] = (m, rate, replicas.seed_for(r))
    except Exception as e:  # the survivor of a missing rank lands here
        out[rank] = "error: " + type(e).__name__
    finally:
        if mode != "absent":
            replicas.finish()


def _run(mode):
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, mode, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
                pytest.fail("a rank did not end")
        return dict(out)


def test_replicas_reduce_the_slowest_rank():
    out = _run("ok")
    assert out[0][0] == out[1][0] == 150.0
    assert out[0][1] == pytest.approx(2 * 1000.0 * 10 / 0.150)
    assert (out[0][2], out[1][2]) == (1, 2)


def test_missing_rank_is_an_error_not_a_hang():
    out = _run("absent")
    assert out[1] == "left"
    assert str(out[0]).startswith("error")
