"""The CPU baseline's bounded sample (CPU only): its sentences are the first
batch entries of each stream's epoch, bit for bit those of the full epoch,
and its word count is the tokens those sentences consumed."""
import numpy as np
import pytest

from golden_cases import load
from oracle import oracle as O

K = 5


def _corpus(eos):
    g = load("eos_t1" if eos else "zipf_t1")
    c = g["cfg"]
    return O.corpus_from_text(g["text"], min_count=c["min_count"], msl=40, cache_eos=c["cache_eos"])


@pytest.mark.parametrize("eos", [False, True])
@pytest.mark.parametrize("sample", [0.0, 1e-3])
@pytest.mark.parametrize("n", [1, 3, 10**6])
def test_prefix_is_the_start_of_the_full_epoch(eos, sample, n):
    corpus = _corpus(eos)
    kw = dict(threads=2, msl=40, negative=K, alpha0=0.025, sample=sample)
    full = O.sample_streams(corpus, epochs=1, **kw)
    for s in range(2):
        f = full[s][0]
        p = O.sample_stream_prefix(corpus, s, n, **kw)
        m = min(n, len(f.lens))
        assert np.array_equal(p.lens, f.lens[:m]) and np.array_equal(p.alphas, f.alphas[:m])
        k = int(p.lens.sum())
        assert np.array_equal(p.ids, f.ids[:k]) and np.array_equal(p.negs, f.negs[:k * K])
        if m == len(f.lens):
            assert p.words_read == f.words_read
        else:
            assert k <= p.words_read < f.words_read
        if sample == 0.0 and not eos and m < len(f.lens):
            assert p.words_read == k  # every token read is kept (no epoch-end drop yet)


def test_cpu_sgns_counts_the_words_of_its_sample():
    corpus = _corpus(False)
    kw = dict(threads=2, msl=40, negative=K, alpha0=0.025, sample=1e-3)
    V, d = len(corpus.counts), 16
    syn0 = O.init_syn0(V, d, d)
    syn1 = np.zeros_like(syn0)
    wr, wk = O.cpu_sgns(corpus, syn0, syn1, epochs=1, d=d, window=3, n_threads=2, max_entries_per_stream=3, **kw)
    parts = [O.sample_stream_prefix(corpus, s, 3, **kw) for s in range(2)]
    assert wr == sum(p.words_read for p in parts)
    assert wk == sum(int(p.lens.sum()) for p in parts)
    assert np.isfinite(syn0).all() and np.abs(syn1).max() > 0
