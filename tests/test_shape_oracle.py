"""The oracle against the reference's host code at the benchmark shapes.

tests/shape_cases.py defines corpora of 1M to 12.5M tokens built by the
benchmark's own generator; tests/golden/shape_*.json hold digests of what the
reference program (oracle/_ref/fw2v_ref_host, FULL-W2V-driver.cu:166-302 with
improved_driver_functions.cpp) made of their text.  Checked here, on the CPU:

  * the generator still writes the same text (sha256);
  * fw2v.synth.build_stream builds the reference's vocabulary from it
    (the -save-vocab file, byte for byte);
  * the oracle's batch builder gives every sampling thread's batches bit for
    bit — sentence lengths, kept ids, the K negatives of every kept id — and
    the "Overall Words" count; learning rates too with one thread (with T
    threads the reference reads a racy shared word count);
  * syn0 initialisation (improved_driver_functions.cpp:1-35) at V=10k/70k.

The same digests pin the device sampler in tests/test_shape_gpu.py.
"""
import hashlib

import numpy as np
import pytest

import shape_cases as S
from oracle import oracle as O


def oracle_streams(c, f):
    oc = O.Corpus(c.stream, c.chunk_off, c.counts, [], c.train_words)
    out = O.sample_streams(oc, threads=f["threads"], msl=f["msl"], negative=f["negative"], epochs=f["iter"],
                           alpha0=f["alpha"], sample=f["sample"])
    per = [(np.concatenate([e.lens for e in s]), np.concatenate([e.alphas for e in s]),
            np.concatenate([e.ids for e in s]), np.concatenate([e.negs for e in s])) for s in out]
    words = sum(e.words_read for s in out for e in s)
    return per, words


@pytest.mark.parametrize("name", list(S.CASES))
def test_oracle_sampler_matches_reference_at_shape(name):
    g = S.load(name)
    f = S.flags_of(name)
    c, text_sha = S.corpus(name)
    assert text_sha == g["text_sha256"], "the generator no longer writes the golden corpus"
    assert hashlib.sha256(S.vocab_file(c)).hexdigest() == g["vocab_sha256"]
    assert len(c.counts) == g["vocab_size"]
    per, words = oracle_streams(c, f)
    assert words == g["overall_words"]
    got = S.digests(per)
    ref = [tuple(x) for x in g["streams"]]
    assert len(got) == f["threads"] == len(ref)
    # lengths, ids and negatives of every thread, as a multiset of threads
    assert [(a, n, k) for a, _, n, k in got] == [(a, n, k) for a, _, n, k in ref]
    if f["threads"] == 1:
        assert got[0][1] == ref[0][1], "learning rates differ"


@pytest.mark.parametrize("name", [n for n in S.CASES if not S.CASES[n].get("no_export")])
def test_oracle_syn0_init_matches_reference_at_shape(name):
    g = S.load(name)
    f = S.flags_of(name)
    V, d = g["vocab_size"], f["size"]
    s0 = O.init_syn0(V, d, d)
    assert hashlib.sha256(np.ascontiguousarray(s0[:, :d]).tobytes()).hexdigest() == g["syn0_init_sha256"]
