"""Batched training of many jobs (fw2v_batch_*) against the oracle.

In the deterministic mode one warp trains every round's sentences in order, so
each job of a batch must equal the oracle run of that job alone, bit for bit:
its sampling (the LCG streams from its seed, subsampling, negatives found by
binary search over the unigram run boundaries instead of the 1e8 table), its
FP32 updates with the lane layout the job's shape uses, and for bfloat16
tables its stochastic rounding with the single-job seeds and sentence numbers.
"""
import numpy as np
import pytest

import fw2v
from fw2v import synth
from golden_cases import load
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MASK = (1 << 64) - 1
K = 5


def _golden_corpus(name, msl):
    g = load(name)
    c = g["cfg"]
    return O.corpus_from_text(g["text"], min_count=c["min_count"], msl=msl, cache_eos=c["cache_eos"])


def _topic_corpus():
    raw, planted, _ = synth.topic_tokens(60_000, 3_000, 8, 1.0, sentence_len=200, seed=21)
    ends = np.arange(200, len(raw) + 1, 200)
    return synth.build_stream(raw, ends, planted, min_count=2, msl=100)


def _walk_corpus():
    walks, block = synth.sbm_walks(1500, 6, 8.0, 20.0, 4, 24, seed=5)
    raw = walks.ravel()
    ends = np.arange(walks.shape[1], len(raw) + 1, walks.shape[1])
    return synth.build_stream(raw, ends, block, min_count=1, msl=1000, cache_eos=True)


def _jobs():
    """(corpus, config overrides) of a mixed batch."""
    return [
        (_golden_corpus("zipf_t1", 50), dict(layer_size=8, window=3, threads=1, msl=50, epochs=2, sample=1e-3, seed=0)),
        (_golden_corpus("messy_t1", 45), dict(layer_size=40, window=5, threads=2, msl=45, epochs=1, sample=1e-3,
                                               seed=7)),
        (_topic_corpus(), dict(layer_size=64, window=10, threads=4, msl=100, epochs=2, sample=1e-3, seed=3)),
        (_walk_corpus(), dict(layer_size=100, window=5, threads=3, msl=1000, epochs=1, sample=1e-3, seed=11)),
        (_golden_corpus("zipf_t3", 40), dict(layer_size=128, window=2, threads=3, msl=40, epochs=3, sample=1e-3,
                                              seed=5)),
        (_golden_corpus("eos_t1", 60), dict(layer_size=200, window=2, threads=1, msl=60, epochs=2, sample=1e-4,
                                             seed=17)),
        (_walk_corpus(), dict(layer_size=300, window=4, threads=2, msl=1000, epochs=1, sample=1e-3, seed=23)),
    ]


def _config(over):
    return fw2v.default_config(negative=K, alpha=0.025, **over)


def _oracle_job(corpus, over, shape, bf16=False):
    """The job alone on the oracle: (syn0, syn1neg) as float32 arrays [V, d]."""
    d, W, E, seed = over["layer_size"], over["window"], over["epochs"], over["seed"]
    lane_vec, lane_nv = shape[0], shape[1]
    V = len(corpus.counts)
    out = O.sample_streams(corpus, threads=over["threads"], msl=over["msl"], negative=K, epochs=E, alpha0=0.025,
                           sample=over["sample"], seed=seed)
    syn0 = O.init_syn0(V, d, d, seed=seed)
    syn1 = np.zeros_like(syn0)
    if bf16:
        syn0, syn1 = O.bf16_bits(syn0), O.bf16_bits(syn1)
    for e in range(E):
        lens = np.concatenate([o[e].lens for o in out])
        alphas = np.concatenate([o[e].alphas for o in out])
        ids = np.concatenate([o[e].ids for o in out])
        negs = np.concatenate([o[e].negs for o in out])
        if bf16:
            sr = O.mix64((0x5EEDF00D + e + O.seed_offset(seed)) & MASK)
            O.train_bf16(syn0, syn1, lens, alphas, ids, negs, d=d, window=W, negative=K, seed=sr, sigmoid="table",
                         vec=lane_vec, nv=lane_nv)
        else:
            O.train(syn0, syn1, lens, alphas, ids, negs, d=d, window=W, negative=K, sigmoid="table", precision=32,
                    vec=lane_vec, nv=lane_nv)
    if bf16:
        return O.bf16_float(syn0), O.bf16_float(syn1)
    return syn0, syn1


def _words(corpus, over):
    out = O.sample_streams(corpus, threads=over["threads"], msl=over["msl"], negative=K, epochs=over["epochs"],
                           alpha0=0.025, sample=over["sample"], seed=over["seed"])
    return sum(o[e].words_read for o in out for e in range(over["epochs"]))


def _batch(jobs, precision=fw2v.FP32, **kw):
    b = fw2v.Batch(precision=precision, **kw)
    for corpus, over in jobs:
        b.add_job(_config(over), corpus.counts, corpus.train_words, corpus.stream, corpus.chunk_off)
    return b


@pytest.fixture(scope="module")
def jobs():
    return _jobs()


# group_bytes 1: every job a group of its own; -1: all jobs interleaved
@pytest.mark.parametrize("use_graph,group_bytes", [(True, 0), (False, 0), (True, 1), (True, -1)])
def test_deterministic_batch_equals_each_job_alone_fp32(jobs, use_graph, group_bytes):
    with _batch(jobs, deterministic=True, use_graph=use_graph, round_tokens=3000, group_bytes=group_bytes) as b:
        st = b.train()
        assert st.rounds > 3 and st.epochs == 3
        for j, (corpus, over) in enumerate(jobs):
            r0, r1 = _oracle_job(corpus, over, b.shape(j))
            np.testing.assert_array_equal(b.syn0(j), r0[:, :over["layer_size"]])
            np.testing.assert_array_equal(b.syn1neg(j), r1[:, :over["layer_size"]])
            assert b.job_words(j)[0] == _words(corpus, over)


@pytest.mark.parametrize("group_bytes", [0, 1])
def test_deterministic_batch_equals_each_job_alone_bf16(jobs, group_bytes):
    with _batch(jobs, precision=fw2v.BF16, deterministic=True, round_tokens=5000, group_bytes=group_bytes) as b:
        b.train()
        for j, (corpus, over) in enumerate(jobs):
            r0, r1 = _oracle_job(corpus, over, b.shape(j), bf16=True)
            np.testing.assert_array_equal(b.syn0(j), r0[:, :over["layer_size"]])
            np.testing.assert_array_equal(b.syn1neg(j), r1[:, :over["layer_size"]])


SHAPES = ([(2, (2, 1, s, 0)) for s in (2, 3, 4, 6)] + [(2, (4, 1, s, 0)) for s in (2, 3, 4, 6)] +
          [(5, (4, 2, s, 0)) for s in (2, 3, 4, 6)] + [(6, (4, 3, s, 0)) for s in (2, 3, 4)] +
          [(2, (2, 1, 6, 1)), (2, (4, 1, 6, 1)), (5, (4, 2, 6, 1)), (3, (4, 1, 6, 1)),
           (2, (2, 1, 2, 1)), (2, (4, 1, 3, 1)), (5, (4, 2, 3, 1)), (6, (4, 3, 2, 1)), (6, (4, 3, 4, 1))] +
          # bit 1: context rows staged by bulk copies (short sentences of job 5, walks of jobs 3 and 6)
          [(5, (4, 2, 3, 2)), (5, (4, 2, 6, 3)), (6, (4, 3, 2, 3)), (2, (2, 1, 6, 2)), (3, (4, 1, 6, 3)),
           (1, (2, 1, 4, 3))])


@pytest.mark.parametrize("job,shape", SHAPES)
def test_every_shape_trains_bit_exact(jobs, job, shape):
    corpus, over = jobs[job]  # d = 64 (one-vector layouts), 200 and 300 (wide rows)
    with _batch([(corpus, over)], deterministic=True) as b:
        b.set_shape(0, *shape)
        b.train()
        r0, r1 = _oracle_job(corpus, over, shape)
        np.testing.assert_array_equal(b.syn0(0), r0)
        np.testing.assert_array_equal(b.syn1neg(0), r1)


def test_batch_job_equals_single_job_handle(jobs):
    corpus, over = jobs[3]
    with _batch([(corpus, over)], deterministic=True) as b:
        b.set_shape(0, 4, 1, 6, 0)  # the single-job kernel's layout for d = 100 and negative 5
        b.train()
        got0, got1 = b.syn0(0), b.syn1neg(0)
    with fw2v.Trainer(_config(dict(over, deterministic=1))) as t:
        t.set_vocab(corpus.counts, corpus.train_words)
        t.load_corpus(corpus.stream, corpus.chunk_off)
        t.train()
        np.testing.assert_array_equal(t.syn0(), got0)
        np.testing.assert_array_equal(t.syn1neg(), got1)


def test_epochs_one_call_at_a_time_continue_like_a_single_job(jobs):
    """Epoch by epoch: the LCG streams, learning rates and rounding seeds
    continue across calls, and a call after the last epoch trains nothing."""
    corpus, over = jobs[4]  # three epochs
    with _batch([(corpus, over)], precision=fw2v.BF16, deterministic=True) as b:
        assert b.train_epochs(1).epochs == 1
        assert b.train_epochs(1).epochs == 1
        assert b.train().epochs == 1
        assert b.train().words_read == 0
        got = b.syn0(0)
    with fw2v.Trainer(_config(dict(over, deterministic=1, precision=fw2v.BF16))) as t:
        t.set_vocab(corpus.counts, corpus.train_words)
        t.load_corpus(corpus.stream, corpus.chunk_off)
        t.train()
        t.train()
        np.testing.assert_array_equal(t.syn0(), got)


@pytest.mark.parametrize("precision", [fw2v.FP32, fw2v.BF16])
def test_concurrent_batch_learns_every_job(jobs, precision):
    with _batch(jobs, precision=precision, round_tokens=20000) as b:
        st = b.train()
        assert st.words_read == sum(_words(c, o) for c, o in jobs)
        for j, (corpus, over) in enumerate(jobs):
            s0 = b.syn0(j)
            assert np.isfinite(s0).all()
            init = O.init_syn0(len(corpus.counts), over["layer_size"], over["layer_size"], seed=over["seed"])
            assert np.abs(s0 - init).max() > 1e-3  # every job trained
            assert np.abs(b.syn1neg(j)).max() > 0


def test_tuner_picks_valid_shapes_and_restores_state(jobs):
    with _batch(jobs, precision=fw2v.BF16) as b:
        before = [b.syn0(j) for j in range(len(jobs))]
        rep = b.tune(sample_tokens=4000)
        assert rep["classes"] and all(c["tuned_wps"] >= c["default_wps"] > 0 for c in rep["classes"])
        for j, (corpus, over) in enumerate(jobs):
            np.testing.assert_array_equal(b.syn0(j), before[j])
            vec, nv, st, _ = b.shape(j)
            assert st in (2, 3, 4, 6) and vec * nv * 32 >= over["layer_size"]
        st = b.train()  # sampler state was restored: the same words as never tuned
        assert st.words_read == sum(_words(c, o) for c, o in jobs)


def test_tuner_cache_round_trip(jobs, tmp_path):
    path = str(tmp_path / "tune.json")
    with _batch(jobs[:3]) as b:
        first = b.tune(sample_tokens=3000, cache=path)
        shapes = [b.shape(j) for j in range(3)]
    with _batch(jobs[:3]) as b:
        again = b.tune(cache=path)
        assert not first["cached"] and again["cached"]
        assert [b.shape(j) for j in range(3)] == shapes


def test_batch_rejects_bad_jobs(jobs):
    corpus, over = jobs[0]
    with fw2v.Batch() as b:
        with pytest.raises(fw2v.Fw2vError):
            b.add_job(_config(dict(over, layer_size=400)), corpus.counts, corpus.train_words, corpus.stream,
                      corpus.chunk_off)
        b.add_job(_config(over), corpus.counts, corpus.train_words, corpus.stream, corpus.chunk_off)
        with pytest.raises(fw2v.Fw2vError):
            b.add_job(fw2v.default_config(negative=3, **{k: v for k, v in over.items()}), corpus.counts,
                      corpus.train_words, corpus.stream, corpus.chunk_off)
        for bad_shape in ((2, 1, 5, 0), (4, 2, 6, 0), (2, 2, 4, 0)):  # stages; d = 8 needs one vector; 2-float wide
            with pytest.raises(fw2v.Fw2vError):
                b.set_shape(0, *bad_shape)
        bad = corpus.stream.copy()
        bad[3] = len(corpus.counts) + 7
        with pytest.raises(fw2v.Fw2vError):
            b.add_job(_config(over), corpus.counts, corpus.train_words, bad, corpus.chunk_off)


def test_tuning_between_epochs_undoes_the_sampling_ahead(jobs):
    """After a call the next epoch's first round is sampled ahead; tuning (or a
    new plan) undoes it, so the streams continue exactly."""
    sel = [jobs[0], jobs[2]]  # two and three epochs
    with _batch(sel, round_tokens=20000) as b:
        first = b.train_epochs(1)
        b.tune(sample_tokens=3000)
        rest = b.train()
        assert first.words_read + rest.words_read == sum(_words(c, o) for c, o in sel)
        for j, (c, o) in enumerate(sel):
            assert b.job_words(j)[0] == _words(c, o)
