"""Job partition of the batched form across ranks (host logic, gloo on CPU)."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fw2v import synth
from fw2v.shard import assign_jobs


def _tokens():
    return [s["nodes"] * s["walks_per_node"] * (s["walk_len"] + 1) for s in synth.c5_job_specs()]


def test_partition_covers_every_job_once_and_balances():
    tok = _tokens()
    for n in (1, 2, 3, 8):
        parts = assign_jobs(tok, n)
        flat = sorted(j for p in parts for j in p)
        assert flat == list(range(len(tok)))
        loads = [sum(tok[j] for j in p) for p in parts]
        assert max(loads) - min(loads) <= max(tok)  # greedy bound


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = assign_jobs(_tokens(), world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.destroy_process_group()
    q.put((rank, got))


@pytest.mark.parametrize("world", [2])
def test_ranks_agree_on_the_partition_without_exchanging_it(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    expect = assign_jobs(_tokens(), world)
    for r in range(world):
        assert res[r] == expect
    assert not set(expect[0]) & set(expect[1])
