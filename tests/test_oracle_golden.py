"""The oracle against the reference's own host code (golden fixtures).

These pin the CPU restatement before anything is checked against it: vocab
order and counts, the token stream, subsampling decisions, negative-sample ids
(which pin the unigram table at every drawn index), per-sentence learning
rates, the word count behind words/sec, and syn0 initialisation.
"""
import hashlib

import numpy as np
import pytest

from golden_cases import CASES, load
from oracle import oracle as O


def _sample(g):
    c = g["cfg"]
    corpus = O.corpus_from_text(g["text"], min_count=c["min_count"], msl=c["msl"],
                                cache_eos=c["cache_eos"])
    out = O.sample_streams(corpus, threads=c["threads"], msl=c["msl"], negative=c["negative"],
                           epochs=c["iter"], alpha0=c["alpha"], sample=c["sample"])
    return corpus, out


def _concat(per_epoch, key):
    return np.concatenate([getattr(e, key) for e in per_epoch])


@pytest.mark.parametrize("name", CASES)
def test_vocab_matches_reference(name):
    g = load(name)
    c = g["cfg"]
    words, counts, _ = O.learn_vocab(g["text"], c["min_count"])
    assert [w.decode("latin-1") for w in words] == list(g["vocab_words"])
    np.testing.assert_array_equal(counts, g["vocab_counts"])


@pytest.mark.parametrize("name", CASES)
def test_sampler_matches_reference(name):
    g = load(name)
    corpus, out = _sample(g)
    c = g["cfg"]
    ref = g["threads_out"]
    assert len(out) == len(ref) == c["threads"]
    # Reference threads dump in launch order; match each to its stream by content.
    unmatched = list(range(len(ref)))
    for s, per_epoch in enumerate(out):
        lens = _concat(per_epoch, "lens")
        ids = _concat(per_epoch, "ids")
        hit = [t for t in unmatched if np.array_equal(ref[t]["lens"], lens)
               and np.array_equal(ref[t]["ids"], ids)]
        assert hit, f"stream {s}: no reference thread with the same sentences"
        t = hit[0]
        unmatched.remove(t)
        np.testing.assert_array_equal(_concat(per_epoch, "negs"), ref[t]["negs"])
        if c["threads"] == 1:
            # With T > 1 the reference's shared learning rate depends on thread timing.
            np.testing.assert_array_equal(_concat(per_epoch, "alphas"), ref[t]["alphas"])
    total = sum(e.words_read for per_epoch in out for e in per_epoch)
    assert total == int(g["overall_words"])


@pytest.mark.parametrize("name", CASES)
def test_syn0_init_matches_reference(name):
    g = load(name)
    d = g["cfg"]["size"]
    V = len(g["vocab_counts"])
    init = O.init_syn0(V, d, d)
    np.testing.assert_array_equal(init[:8], g["syn0_init_head"])
    assert hashlib.sha256(init.tobytes()).hexdigest() == str(g["syn0_init_sha256"])


def test_exp_table_known_values():
    t = O.exp_table()
    assert t[0] == 0.0 and t[999] == 1.0
    # sigma(0) sits at i = 500: x = (500/1000*2-1)*6 = 0
    assert t[500] == np.float32(0.5)
    assert np.all(np.diff(t) >= 0)
    # reference header value at index 1 (expTable.h line 1)
    assert t[1] == np.float32(0.00250239903107285499572753906250)


def test_unigram_quirk_word1_takes_eos_share():
    # </s> count 0 => word 1 gets a zero share: only the two entries the
    # one-step-per-entry fill cannot skip (indices 0 and 1)
    counts = np.array([0, 50, 30, 20], np.uint32)
    starts, words = O.unigram_runs(counts, table_size=1000)
    assert words[0] == 1 and starts[1] - starts[0] == 2
    # with a non-zero </s> count word 1 receives exactly that share
    counts = np.array([10, 50, 30, 20], np.uint32)
    starts, words, table = O.unigram_runs(counts, table_size=100000, full=True)
    share = 10 ** 0.75 / sum(c ** 0.75 for c in counts)
    assert abs(np.mean(table == 1) - share) < 1e-4
    # runs reproduce the literal table
    for j, w in enumerate(words):
        assert np.all(table[starts[j]:starts[j + 1]] == w)


def _match_streams(out, ref, check_alpha):
    unmatched = list(range(len(ref)))
    for per_epoch in out:
        lens, ids = _concat(per_epoch, "lens"), _concat(per_epoch, "ids")
        hit = [t for t in unmatched if np.array_equal(ref[t]["lens"], lens)
               and np.array_equal(ref[t]["ids"], ids)]
        assert hit, "a stream differs from every reference thread"
        unmatched.remove(hit[0])
        np.testing.assert_array_equal(_concat(per_epoch, "negs"), ref[hit[0]]["negs"])
        if check_alpha:
            np.testing.assert_array_equal(_concat(per_epoch, "alphas"), ref[hit[0]]["alphas"])


@pytest.mark.parametrize("name", CASES)
def test_cache_fed_sampler_matches_reference(name):
    """The reference run from its own vocabulary file and corpus cache."""
    g = load(name)
    c = g["cfg"]
    words, counts, _ = O.read_vocab(g["vocab_text"], c["min_count"])
    stream, offs, tw = O.read_corpus_cache(g["cache_text"], c["msl"], c["cache_eos"])
    corpus = O.Corpus(stream, offs, counts, words, tw)
    out = O.sample_streams(corpus, threads=c["threads"], msl=c["msl"], negative=c["negative"],
                           epochs=c["iter"], alpha0=c["alpha"], sample=c["sample"])
    _match_streams(out, g["cache_threads_out"], c["threads"] == 1)
    assert sum(e.words_read for p in out for e in p) == int(g["cache_overall_words"])
