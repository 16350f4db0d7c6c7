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
