"""Embedding quality on the synthetic corpora (the reference measures quality with
public word-similarity sets under analysis/hyperwords/, which are not available
offline).

heldout_loss: the SGNS loss of held-out text, summed in FP64 on the GPU by the
library (fw2v_heldout_loss), per (context, centre) pair: -log s(<v_c, o_w>) -
sum_k log s(-<v_c, o_nk>).  The negatives come from the library's own sampler
with subsampling off and fixed LCG streams, so two models are scored on
identical pairs.

precision_at_10: for query words, the share of their 10 nearest neighbours by
cosine similarity (syn0) that share their planted topic or block; the
neighbour search is this library's kernel (fw2v_neighbours).
"""
from __future__ import annotations

import numpy as np

from . import Trainer, default_config


def sentence_chunks(stream: np.ndarray, msl: int) -> np.ndarray:
    """Chunk starts of a token stream: every sentence (ended by a 0, or by the
    end of the stream) cut into pieces of at most msl tokens."""
    n = len(stream)
    ends = np.nonzero(stream == 0)[0] + 1
    if len(ends) == 0 or ends[-1] < n:
        ends = np.concatenate([ends, [n]])
    begins = np.concatenate([[0], ends[:-1]])
    out = [np.arange(b, e, msl, dtype=np.int64) for b, e in zip(begins, ends) if e > b]
    return np.concatenate(out) if out else np.zeros(1, np.int64)


def heldout_pairs(counts, train_words, held_stream, *, window, negative, msl=1000, threads=16):
    """(lens, ids, negs) of held-out sentences with K negatives per word.  A 0
    in held_stream ends a sentence (walk corpora); otherwise sentences are
    pieces of msl tokens."""
    held = np.asarray(held_stream, np.int32)
    chunk_off = sentence_chunks(held, msl)
    cfg = default_config(layer_size=8, window=window, negative=negative, epochs=1,
                         threads=min(threads, len(chunk_off)), msl=msl, sample=0.0)
    stream = np.concatenate([held, [0]]).astype(np.int32)
    with Trainer(cfg) as t:
        t.set_vocab(counts, train_words)
        t.load_corpus(stream, chunk_off)
        t.sample_epoch()
        per = t.epoch_samples()
    lens = np.concatenate([p[0] for p in per])
    ids = np.concatenate([p[2] for p in per])
    negs = np.concatenate([p[3] for p in per])
    return lens, ids, negs


def heldout_loss(trainer: Trainer, pairs) -> float:
    """Mean held-out SGNS loss per (context, centre) pair."""
    lens, ids, negs = pairs
    total, n = trainer.heldout_loss(lens, ids, negs)
    return total / max(n, 1)


def neighbours(table, cand: np.ndarray, queries: np.ndarray, k: int = 10, *, precision: int = 0,
               layer_size: int | None = None, device="cuda"):
    """The k nearest other candidates of each query by cosine similarity
    (fw2v_neighbours, this library's kernel): (indices into cand [n_q, k],
    cosines [n_q, k]).  `table`: rows of FP32 (or bfloat16 bits, precision
    BF16) as a numpy array or a device tensor."""
    import torch

    from . import lib
    t = table if isinstance(table, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(table))
    t = t.to(device)
    d = layer_size or t.shape[1]
    c = torch.from_numpy(np.ascontiguousarray(cand, np.int32)).to(device)
    q = torch.from_numpy(np.ascontiguousarray(queries, np.int32)).to(device)
    out_i = torch.empty((len(queries), k), dtype=torch.int32, device=device)
    out_s = torch.empty((len(queries), k), dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(t.device)
    st = lib().fw2v_neighbours(t.data_ptr(), precision, t.stride(0), d, c.data_ptr(), len(cand), q.data_ptr(),
                               len(queries), k, out_i.data_ptr(), out_s.data_ptr(), stream.cuda_stream)
    if st != 0:
        raise RuntimeError(f"fw2v_neighbours failed: status {st}")
    stream.synchronize()
    return out_i.cpu().numpy(), out_s.cpu().numpy()


def precision_at_10(syn0: np.ndarray, label: np.ndarray, counts: np.ndarray, *, purity=None,
                    min_purity: float = 0.5, queries: int = 2000, min_count: int = 5, seed: int = 0,
                    device="cuda") -> tuple[float, int]:
    """Same-label precision@10 by cosine similarity over the words that carry
    their planted label (purity above min_purity, count at least min_count):
    queries are drawn from them (all of them with queries=0) and neighbours
    searched among all of them by this library's kernel (fw2v_neighbours).
    Returns (precision, number of such words)."""
    ok = (label >= 0) & (counts >= min_count)
    if purity is not None:
        ok &= purity > min_purity
    cand = np.nonzero(ok)[0]
    if len(cand) < 11:
        return float("nan"), len(cand)
    if queries and queries < len(cand):
        q = np.random.default_rng(seed).choice(len(cand), size=queries, replace=False)
    else:
        q = np.arange(len(cand))
    top, _ = neighbours(syn0, cand, q, 10, device=device)
    lab = label[cand]
    return float((lab[top] == lab[q][:, None]).mean()), len(cand)
