"""Embedding quality on the synthetic corpora (the reference measures quality with
public word-similarity sets under analysis/hyperwords/, which are not available
offline).

heldout_loss: the SGNS loss of held-out text, summed in FP64 on the GPU by the
library (fw2v_heldout_loss), per (context, centre) pair: -log s(<v_c, o_w>) -
sum_k log s(-<v_c, o_nk>).  The negatives come from the library's own sampler
with subsampling off and fixed LCG streams, so two models are scored on
identical pairs.

precision_at_10: for query words, the share of their 10 nearest neighbours by
cosine similarity (syn0) that share their planted topic or block.
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


def precision_at_10(syn0: np.ndarray, label: np.ndarray, counts: np.ndarray, *, purity=None,
                    min_purity: float = 0.5, queries: int = 2000, min_count: int = 5, seed: int = 0,
                    device="cuda") -> tuple[float, int]:
    """Same-label precision@10 by cosine similarity over the words that carry
    their planted label (purity above min_purity, count at least min_count):
    queries are drawn from them and neighbours searched among them.  Returns
    (precision, number of such words)."""
    import torch

    ok = (label >= 0) & (counts >= min_count)
    if purity is not None:
        ok &= purity > min_purity
    cand = np.nonzero(ok)[0]
    if len(cand) < 11:
        return float("nan"), len(cand)
    rng = np.random.default_rng(seed)
    q = rng.choice(len(cand), size=min(queries, len(cand)), replace=False)
    E = torch.from_numpy(np.ascontiguousarray(syn0[cand], np.float32)).to(device)
    E = E / E.norm(dim=1, keepdim=True).clamp_min(1e-12)
    qi = torch.from_numpy(q).to(device)
    sims = E[qi] @ E.T
    sims[torch.arange(len(q), device=device), qi] = -2.0
    top = torch.topk(sims, 10, dim=1).indices.cpu().numpy()
    lab = label[cand]
    return float((lab[top] == lab[q][:, None]).mean()), len(cand)
