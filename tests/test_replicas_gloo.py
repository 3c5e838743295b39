"""CPU: the multi-rank plumbing of bench.py (one replica per GPU) over gloo,
world size 2: rendezvous on 127.0.0.1, the start barrier, and the timing
reduction (max over ranks) that makes the job's ms/step the slowest rank's."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    got_ws, got_rank, _, pg = bench.dist_setup(timeout_s=60)
    assert pg is not None and pg.get_backend() == "gloo"
    bench.barrier(pg)
    # rank r "took" 10 + 5 r ms per step: the job's time is the slowest replica's
    t = bench.max_over_ranks(pg, 10.0 + 5.0 * rank)
    q.put((got_rank, got_ws, t))
    pg.barrier()
    pg.destroy_process_group()


def test_two_replicas_reduce_to_the_slowest():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(ws))
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == ws and r[2] == pytest.approx(15.0) for r in res)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    ws, rank, local, pg = bench.dist_setup()
    assert (ws, rank, local, pg) == (1, 0, 0, None)
    assert bench.max_over_ranks(pg, 3.5) == 3.5
