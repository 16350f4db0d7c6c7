"""Partition of independent jobs across ranks (one process per GPU) for the
batched form: the jobs share nothing, so each rank trains its own batch and no
collective touches the data path."""
from __future__ import annotations


def assign_jobs(tokens: list[int], n_ranks: int) -> list[list[int]]:
    """Longest-first greedy bin-pack by token count: jobs in descending size
    (ties by index) each go to the least-loaded rank (ties to the lowest).
    Deterministic, so every rank computes the same assignment on its own.
    Returns the job indices of each rank, in increasing order."""
    if n_ranks < 1:
        raise ValueError("n_ranks >= 1")
    load = [0] * n_ranks
    out: list[list[int]] = [[] for _ in range(n_ranks)]
    for j in sorted(range(len(tokens)), key=lambda i: (-tokens[i], i)):
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        out[r].append(j)
        load[r] += tokens[j]
    return [sorted(x) for x in out]


def job_tokens(specs: list[dict]) -> list[int]:
    """Tokens of each graph job (walks per node x nodes x (walk length + 1))."""
    return [s["nodes"] * s["walks_per_node"] * (s["walk_len"] + 1) for s in specs]


def rank_share(specs: list[dict], world: int, rank: int) -> list[int]:
    """This rank's jobs (indices into specs) under assign_jobs."""
    return assign_jobs(job_tokens(specs), world)[rank]


def combine_ranks(words: float, seconds: float, alone_words: float = 0.0, alone_seconds: float = 0.0,
                  device=None) -> dict:
    """Whole-job figures of a partitioned batch: words summed over ranks, time
    the slowest rank's (max), for the batch and for the jobs trained alone.
    Uses torch.distributed when a process group is initialised (any backend;
    `device` is where the reduction tensors live: "cuda" under NCCL, "cpu"
    under gloo), else this process alone.  Every rank calls it at the same
    point (two all-reduces, the same on every rank)."""
    import torch
    import torch.distributed as dist

    w = torch.tensor([float(words), float(alone_words)], dtype=torch.float64, device=device)
    t = torch.tensor([float(seconds), float(alone_seconds)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w, t = w.cpu().tolist(), t.cpu().tolist()
    out = {"words": w[0], "seconds": t[0], "value": w[0] / t[0] if t[0] > 0 else 0.0}
    if t[1] > 0:
        out.update(alone_words=w[1], alone_seconds=t[1], alone_value=w[1] / t[1])
    return out
