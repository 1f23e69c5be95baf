"""Multi-rank replica plumbing (one shot per GPU) on CPU: two gloo ranks on
127.0.0.1, as torchrun would start them.  Covers the max-over-ranks device
time, the whole-job aggregate, the reference-arm rank rule, and failure
detection on the host: a rank that dies before a collective makes the
other's collective fail within the process-group timeout."""
import multiprocessing as mp
import os
import socket
import time

import pytest

from konglong_b200 import replicas as R


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    return {"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
            "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)}


def _rank_main(rank, world, port, mode, q):
    os.environ.update(_env(rank, world, port))
    ranks = R.Ranks.from_env()
    try:
        R.init(ranks, "gloo", timeout_s=5.0)
        if mode == "ok":
            ms = 10.0 + 5.0 * rank  # rank 1 is slower
            R.barrier(ranks)
            mx = R.max_over_ranks(ranks, ms)
            value = R.aggregate_gpts(ranks.world, 1_000_000, 20, mx)
            q.put((rank, "ok", mx, value, R.runs_reference_arm(ranks)))
            R.finish(ranks)
        else:  # "die": rank 1 fails between steps, before the collective
            if rank == 1:
                q.put((rank, "died", None, None, None))
                q.close()
                q.join_thread()  # flush before the hard exit
                os._exit(3)
            t0 = time.time()
            try:
                R.max_over_ranks(ranks, 1.0)
                q.put((rank, "no-error", None, None, None))
            except Exception as e:  # the process group reports the lost rank
                q.put((rank, "error", time.time() - t0, type(e).__name__, None))
    except Exception as e:
        q.put((rank, "exception", None, repr(e), None))


def _run(mode, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = []
    t0 = time.time()
    while len(out) < world and time.time() - t0 < timeout:
        try:
            out.append(q.get(timeout=1.0))
        except Exception:
            pass
    for p in ps:
        p.join(timeout=10)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda r: r[0])


def test_ranks_from_env():
    r = R.Ranks.from_env(_env(1, 4, 0))
    assert (r.rank, r.world, r.local_rank) == (1, 4, 1) and r.distributed
    assert not R.Ranks.from_env({}).distributed
    assert R.runs_reference_arm(R.Ranks(0, 2, 0)) and not R.runs_reference_arm(R.Ranks(1, 2, 1))


def test_aggregate_is_whole_job():
    # 2 ranks x 1e6 cells x 20 steps in 10 ms -> 4 Gpts/s
    assert R.aggregate_gpts(2, 1_000_000, 20, 10.0) == pytest.approx(4.0)
    assert R.max_over_ranks(R.Ranks(), 7.5) == 7.5


def test_two_gloo_ranks_max_over_ranks():
    out = _run("ok")
    assert [o[1] for o in out] == ["ok", "ok"], out
    for rank, _, mx, value, ref in out:
        assert mx == 15.0  # the slower rank's time, on every rank
        assert value == pytest.approx(R.aggregate_gpts(2, 1_000_000, 20, 15.0))
        assert ref == (rank == 0)


def test_lost_rank_fails_the_collective():
    out = _run("die")
    status = {o[0]: o[1] for o in out}
    assert status.get(1) == "died", out
    assert status.get(0) == "error", out
    # detected within the process-group timeout (5 s) plus start-up slack
    assert out[0][2] < 30.0
