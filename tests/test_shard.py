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


def _fake_rank_run(specs, share, rank):
    """Stand-in for a rank's GPU work in bench.run_c5: every job's words are its
    tokens; the rank trains at a rate of its own (so the ranks finish at
    different times); alone, each job at half that rate."""
    from fw2v.shard import job_tokens
    tok = job_tokens([specs[j] for j in share])
    rate = 1e8 * (1 + rank)
    return float(sum(tok)), sum(tok) / rate, float(sum(tok)), 2 * sum(tok) / rate


def _c5_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from fw2v.shard import combine_ranks, rank_share
    specs = synth.c5_job_specs()
    share = rank_share(specs, world, rank)
    words, secs, alone_words, alone_secs = _fake_rank_run(specs, share, rank)
    tot = combine_ranks(words, secs, alone_words, alone_secs, device="cpu")
    dist.destroy_process_group()
    q.put((rank, share, secs, tot))


def test_c5_rank_flow_sums_words_and_takes_the_slowest_rank():
    """The per-rank bookkeeping of the batched configuration on 2 gloo ranks
    with the GPU work stubbed: each rank takes its share of the 256 jobs, and
    every rank reports the same totals: words of all jobs over the slowest
    rank's time, for the batch and for the jobs alone."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_c5_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        rank, share, secs, tot = q.get(timeout=120)
        res[rank] = (share, secs, tot)
    for p in procs:
        p.join(timeout=60)
    assert sorted(res[0][0] + res[1][0]) == list(range(256))
    total = float(sum(_tokens()))
    slowest = max(res[0][1], res[1][1])
    for r in range(world):
        tot = res[r][2]
        assert tot == res[0][2]
        assert tot["words"] == total and tot["alone_words"] == total
        assert abs(tot["seconds"] - slowest) <= 1e-12 * slowest
        assert abs(tot["value"] - total / slowest) <= 1e-9 * tot["value"]
        assert abs(tot["alone_value"] - tot["value"] / 2) <= 1e-9 * tot["value"]


def test_combine_ranks_without_a_process_group():
    from fw2v.shard import combine_ranks
    tot = combine_ranks(1000, 2.0, 1000, 4.0)
    assert tot["value"] == 500 and tot["alone_value"] == 250
