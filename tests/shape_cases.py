"""Parity cases at the shapes of the benchmark configurations.

Each case is a seeded synthetic corpus (the benchmark's own generator,
fw2v.synth.topic_tokens, written one 1000-token sentence per line) and the
reference program's flags.  tests/golden/make_golden.py runs the reference's
host code (oracle/_ref/fw2v_ref_host) on the text of each case and stores, in
tests/golden/shape_<name>.json, digests of what it produced: the vocabulary
file, the exported initial vectors and, per sampling thread, the batches its
host loop shipped to the GPU (sentence lengths, kept ids and negatives, and
learning rates).  The corpora are too large to commit; the digests pin them
and everything derived from them.

  c1_t1, c1_t16   the C1 corpus itself: 1M tokens, V=10k, 20 topics,
                  Zipf(1.0); d=100, window 5, negative 5, sample 1e-4,
                  msl 1000, 1 and 16 sampling streams.
  c2cut_t64       2M tokens of the C2 generator (71k-word law, 100 topics,
                  Zipf(1.0)), min-count 5, window 8, 2 epochs, 64 streams.
  c3cut_t3125     12.5M tokens over the C3 vocabulary size and law (555k
                  words, Zipf(1.05)) with 20 topics so that the generator's
                  per-topic tables stay small and frequent words are
                  subsampled; the benchmark's 3125 streams and msl 1000.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = {
    "c1_t1": dict(gen=dict(n_tokens=1_000_000, vocab=10_000, topics=20, zipf_s=1.0, seed=1235),
                  flags="-size 100 -window 5 -negative 5 -sample 1e-4 -iter 1 -threads 1 -min-count 1 "
                        "-msl 1000 -alpha 0.025"),
    "c1_t16": dict(gen=dict(n_tokens=1_000_000, vocab=10_000, topics=20, zipf_s=1.0, seed=1235),
                   flags="-size 100 -window 5 -negative 5 -sample 1e-4 -iter 1 -threads 16 -min-count 1 "
                         "-msl 1000 -alpha 0.025"),
    "c2cut_t64": dict(gen=dict(n_tokens=2_000_000, vocab=71_000, topics=100, zipf_s=1.0, seed=1236),
                      flags="-size 128 -window 8 -negative 5 -sample 1e-4 -iter 2 -threads 64 -min-count 5 "
                            "-msl 1000 -alpha 0.025"),
    "c3cut_t3125": dict(gen=dict(n_tokens=12_500_000, vocab=555_000, topics=20, zipf_s=1.05, seed=1237),
                        flags="-size 300 -window 5 -negative 5 -sample 1e-4 -iter 1 -threads 3125 "
                              "-min-count 1 -msl 1000 -alpha 0.025", no_export=True),
}


def flags_of(name: str) -> dict:
    toks = CASES[name]["flags"].split()
    f = {toks[i].lstrip("-").replace("-", "_"): toks[i + 1] for i in range(0, len(toks), 2)}
    return {"size": int(f["size"]), "window": int(f["window"]), "negative": int(f["negative"]),
            "sample": float(f["sample"]), "iter": int(f["iter"]), "threads": int(f["threads"]),
            "min_count": int(f["min_count"]), "msl": int(f["msl"]), "alpha": float(f["alpha"])}


def raw_tokens(name: str):
    """(raw token ids, sentence ends, planted topic per raw id) of a case."""
    from fw2v import synth
    g = CASES[name]["gen"]
    raw, planted, _ = synth.topic_tokens(g["n_tokens"], g["vocab"], g["topics"], g["zipf_s"], seed=g["seed"])
    ends = np.arange(1000, len(raw) + 1000, 1000)
    ends[-1] = len(raw)
    return raw, ends, planted


def corpus(name: str):
    """The case's corpus as the reference's text front end builds it from the
    text (fw2v.synth.build_stream), and the text's sha256."""
    from fw2v import synth
    raw, ends, planted = raw_tokens(name)
    c = synth.build_stream(raw, ends, planted, min_count=flags_of(name)["min_count"], msl=flags_of(name)["msl"])
    return c, hashlib.sha256(synth.text_of(raw, ends)).hexdigest()


def vocab_file(c) -> bytes:
    """The reference's -save-vocab file of a corpus (`word count` per line)."""
    words = ["</s>"] + [f"w{r}" for r in c.raw_of_vocab[1:]]
    return "".join(f"{w} {int(n)}\n" for w, n in zip(words, c.counts)).encode()


def _h(*arrays) -> str:
    m = hashlib.sha256()
    for a, dt in arrays:
        m.update(np.ascontiguousarray(a, dtype=dt).tobytes())
        m.update(b"|")
    return m.hexdigest()[:16]


def stream_digest(lens, ids, negs) -> str:
    """Digest of one sampling stream's batches over all epochs, in order."""
    return _h((lens, "<i4"), (ids, "<i4"), (negs, "<i4"))


def alpha_digest(alphas) -> str:
    return _h((alphas, "<f4"))


def digests(per_stream):
    """per_stream: [(lens, alphas, ids, negs)] -> sorted [(stream digest,
    alpha digest, entries, kept)]: a multiset, because the reference's dump
    files are numbered in the order its threads first launched."""
    out = [(stream_digest(l, i, n), alpha_digest(a), int(len(l)), int(len(i))) for l, a, i, n in per_stream]
    return sorted(out)


def load(name: str) -> dict:
    with open(os.path.join(GOLDEN, f"shape_{name}.json")) as f:
        return json.load(f)
