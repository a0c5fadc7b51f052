"""The N-GPU bench path (one process per GPU, one replica each) on the CPU: two `gloo` ranks
run the bench's own rank plumbing (`bench.Ranks`).  Checks the reductions the bench reports
(time = max over ranks, updates = sum), and that a retry wanted by one rank is taken by every
rank, so all ranks keep calling their collectives in the same order."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    ranks = bench.Ranks(world, "gloo", "cpu")
    ranks.barrier()
    res = {"max": ranks.max(10.0 * (rank + 1)), "sum": ranks.sum(rank + 1.0),
           "any_one": ranks.any(rank == world - 1), "any_none": ranks.any(False)}
    # the bench's timing loop: the last rank "solves inside the timed region" on its first
    # attempt only; every rank must repeat that attempt
    attempts = 0
    for attempt in range(4):
        attempts += 1
        ranks.barrier()
        steps_done = 3 if (rank == world - 1 and attempt == 0) else 5
        ranks.barrier()
        if not ranks.any(steps_done != 5):
            break
    res["attempts"] = attempts
    # value as the bench forms it: total updates of all ranks / slowest rank's time
    t_max = ranks.max(1.0 + rank)
    res["value"] = ranks.sum(800.0 * 5) / t_max
    ranks.close()
    out.put((rank, res))


@pytest.mark.parametrize("world", [2])
def test_ranks_collectives_and_lockstep_retry(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        res = got[r]
        assert res["max"] == 10.0 * world
        assert res["sum"] == sum(range(1, world + 1))
        assert res["any_one"] is True and res["any_none"] is False
        assert res["attempts"] == 2
        assert res["value"] == pytest.approx(800.0 * 5 * world / world)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    r = bench.Ranks(1, "gloo", "cpu")
    r.barrier()
    assert r.max(3.0) == 3.0 and r.sum(2.0) == 2.0 and r.any(True) and not r.any(False)
    r.close()
