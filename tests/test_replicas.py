"""Replica coordination of the multi-GPU bench (one process per GPU, no
collective on the data path), exercised with two gloo ranks on the CPU: the
slowest rank's time sets the whole job's rate, every rank sees the same
maximum and sum, and a rank that leaves early is reported, not waited on
forever."""
import multiprocessing as mp
import os
import socket

import pytest

from mlmq_tpds_withl3_b200.replicas import whole_job_rate


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from mlmq_tpds_withl3_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    slowest = rep.max(1.5 + rank)        # rank 1 is the slow one
    total = rep.sum(10.0 * (rank + 1))
    rate = whole_job_rate(100, rep.world, slowest)
    cfg = rep.broadcast({"delta": 50000, "warps_per_block": 8} if rank == 0 else {"delta": -1})
    rep.close()
    out.put((rank, rep.world, slowest, total, rate, cfg))


def _run(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res)


def test_two_ranks_agree_on_max_and_sum():
    res = _run(2)
    assert [r[0] for r in res] == [0, 1]
    for _, world, slowest, total, rate, cfg in res:
        assert world == 2
        assert slowest == 2.5
        assert total == 30.0
        assert rate == pytest.approx(2 * 100 / 2.5)
        assert cfg == {"delta": 50000, "warps_per_block": 8}  # rank 0's tuned configuration


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from mlmq_tpds_withl3_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert (rep.world, rep.rank) == (1, 0)
    assert rep.max(3.0) == 3.0 and rep.sum(3.0) == 3.0
    rep.barrier()
    rep.close()


def _lonely_rank(port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK="0",
                      LOCAL_RANK="0")
    from mlmq_tpds_withl3_b200.replicas import Replicas
    try:
        Replicas("gloo", timeout_s=3)
        out.put("joined")
    except Exception as e:  # the missing rank never joins: rendezvous times out
        out.put(type(e).__name__)


def test_missing_rank_times_out_instead_of_hanging():
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    p = ctx.Process(target=_lonely_rank, args=(port, out))
    p.start()
    msg = out.get(timeout=120)
    p.join(timeout=60)
    assert msg != "joined"
