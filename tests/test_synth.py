"""The synthetic workloads against the benchmark configurations they stand in
for: sizes and laws of the topic-mixture corpora (C1-C3), the stochastic block
model and its walks (C4), the 256 job specifications (C5), and the text front
end's vocabulary and stream rules that build_stream restates
(improved_driver_functions.cpp:136-164, 244-281).  CPU only."""
import numpy as np
import pytest

from fw2v import synth


def test_topic_configs_match_the_benchmark_configurations():
    c1, c2, c3 = (synth.CONFIGS[k] for k in ("c1", "c2", "c3"))
    assert (c1["n_tokens"], c1["vocab"], c1["topics"], c1["zipf_s"]) == (1_000_000, 10_000, 20, 1.0)
    assert (c1["d"], c1["window"], c1["negative"], c1["sample"], c1["epochs"]) == (100, 5, 5, 1e-4, 1)
    assert (c2["n_tokens"], c2["vocab"], c2["topics"], c2["zipf_s"], c2["min_count"]) == (17_000_000, 71_000, 100,
                                                                                        1.0, 5)
    assert (c2["d"], c2["window"], c2["negative"], c2["sample"], c2["epochs"]) == (128, 8, 5, 1e-4, 5)
    assert (c3["n_tokens"], c3["vocab"], c3["topics"], c3["zipf_s"]) == (800_000_000, 555_000, 1000, 1.05)
    assert (c3["d"], c3["window"], c3["negative"], c3["sample"], c3["epochs"]) == (300, 5, 5, 1e-4, 1)
    c4 = synth.GRAPH_CONFIGS["c4"]
    assert (c4["nodes"], c4["blocks"], c4["degree"], c4["p_ratio"]) == (1_000_000, 64, 20.0, 20.0)
    assert (c4["walks_per_node"], c4["walk_len"], c4["d"], c4["window"], c4["negative"], c4["sample"]) == (
        10, 80, 128, 10, 5, 1e-3)
    assert c4["nodes"] * c4["walks_per_node"] * c4["walk_len"] == 800_000_000


def test_topic_tokens_laws():
    V, topics, s = 2000, 8, 1.0
    raw, planted, purity = synth.topic_tokens(200_000, V, topics, s, seed=3)
    assert raw.shape == (200_000,) and raw.dtype == np.int32
    assert raw.min() >= 0 and raw.max() < V
    assert planted.shape == (V,) and planted.min() >= 0 and planted.max() < topics
    assert np.all((purity > 0) & (purity <= 1))
    # Dirichlet(0.1) weights: a sentence is dominated by few topics, so its
    # words' planted topics concentrate (a uniform mixture would give ~1/8)
    sent = raw.reshape(-1, 1000)
    top_share = [np.bincount(planted[r], minlength=topics).max() / 1000 for r in sent]
    assert np.mean(top_share) > 0.5
    # Zipf(1) per topic: over the whole corpus the most frequent word is far
    # more frequent than the median word
    cnt = np.sort(np.bincount(raw, minlength=V))[::-1]
    assert cnt[0] > 20 * max(cnt[V // 2], 1)
    # seeded
    raw2, _, _ = synth.topic_tokens(200_000, V, topics, s, seed=3)
    assert np.array_equal(raw, raw2)


def test_build_stream_follows_the_text_front_end():
    # three lines; raw words 7, 5, 9, 3 (3 below min_count 2)
    raw = np.array([7, 5, 7, 9, 5, 7, 9, 3], np.int32)
    ends = np.array([3, 6, 8])
    label = np.arange(10, dtype=np.int32) * 10
    c = synth.build_stream(raw, ends, label, min_count=2, msl=2)
    # "</s>" first with one count per line but the last; then by count, ties in
    # first-occurrence order (5 before 9)
    assert list(c.raw_of_vocab) == [-1, 7, 5, 9]
    assert list(c.counts) == [2, 3, 2, 2]
    assert c.train_words == int(c.counts.sum()) + 1
    # in-vocabulary ids only, a trailing 0, chunks of msl
    assert list(c.stream) == [1, 2, 1, 3, 2, 1, 3, 0]
    assert list(c.chunk_off) == [0, 2, 4, 6]
    assert list(c.label) == [-1, 70, 50, 90]
    # with -cache-eos: "</s>" after every line, chunks end at it or at msl
    e = synth.build_stream(raw, ends, label, min_count=2, msl=3, cache_eos=True)
    assert list(e.stream) == [1, 2, 1, 0, 3, 2, 1, 0, 3, 0, 0]
    assert list(e.chunk_off) == [0, 3, 4, 7, 8]


def test_text_of_writes_one_sentence_per_line():
    raw = np.array([4, 0, 12, 4], np.int32)
    assert synth.text_of(raw, np.array([2, 4])) == b"w4 w0\nw12 w4\n"


@pytest.mark.parametrize("builder", ["numpy", "torch"])
@pytest.mark.parametrize("nodes,blocks", [(100_000, 64), (1000, 64), (3000, 4)])
def test_sbm_graph_has_the_configured_degree_and_ratio(builder, nodes, blocks):
    degree, ratio = 20.0, 20.0
    rng = np.random.default_rng(7)
    if builder == "numpy":
        offs, dst, block = synth.sbm_graph(nodes, blocks, degree, ratio, rng)
    else:
        import torch
        gen = torch.Generator(device="cpu")
        gen.manual_seed(7)
        offs, dst, block = (t.numpy() for t in synth.sbm_graph_torch(nodes, blocks, degree, ratio, rng, gen,
                                                                     torch.device("cpu")))
    src = np.repeat(np.arange(nodes), np.diff(offs))
    dst = dst.astype(np.int64)
    assert len(offs) == nodes + 1 and dst.min() >= 0 and dst.max() < nodes
    assert not np.any(src == dst)
    # undirected: every edge appears in both directions
    fwd = np.sort(src * nodes + dst)
    assert np.array_equal(fwd, np.sort(dst * nodes + src))
    # mean degree and the share of in-block edges of the configured law
    bsize = nodes / blocks
    p_out = degree / (ratio * (bsize - 1) + (nodes - bsize))
    expect_in = ratio * p_out * (bsize - 1) / degree
    tol = 4 / np.sqrt(len(src))
    assert abs(len(src) / nodes / degree - 1) < tol
    assert abs(np.mean(block[src] == block[dst]) - expect_in) < tol


def test_sbm_walks_degree_and_block_structure():
    nodes, blocks, degree, ratio = 4000, 8, 20.0, 20.0
    walks, block = synth.sbm_walks(nodes, blocks, degree, ratio, 2, 30, seed=11)
    assert walks.shape == (2 * nodes, 30)
    assert np.array_equal(walks[:, 0], np.repeat(np.arange(nodes), 2))
    assert np.array_equal(np.bincount(block), np.full(blocks, nodes // blocks))
    # a step stays in its block with probability p_in (bsize-1) / degree
    bsize = nodes / blocks
    p_out = degree / (ratio * (bsize - 1) + (nodes - bsize))
    expect_in = ratio * p_out * (bsize - 1) / degree
    same = block[walks[:, 1:]] == block[walks[:, :-1]]
    assert abs(same.mean() - expect_in) < 0.01
    # at degree 20 almost no node is isolated, so almost every walk moves
    w2, _ = synth.sbm_walks(nodes, blocks, degree, ratio, 1, 2, seed=12)
    moved = w2[:, 1] != w2[:, 0]
    assert moved.mean() > 0.99


def test_c5_job_specs_cover_the_configured_ranges():
    specs = synth.c5_job_specs()
    assert len(specs) == 256
    nodes = np.array([s["nodes"] for s in specs])
    assert nodes.min() >= 1000 and nodes.max() <= 200_000
    # log-uniform: about half the jobs below the geometric mean (14.1k)
    assert 0.35 < np.mean(nodes < np.sqrt(1000 * 200_000)) < 0.65
    assert all(4 <= s["blocks"] <= 64 and 10 <= s["degree"] <= 30 for s in specs)
    assert all(40 <= s["walk_len"] <= 80 and s["walks_per_node"] == 10 for s in specs)
    assert {s["d"] for s in specs} == {64, 128} and {s["window"] for s in specs} == {5, 10}
    assert all(s["negative"] == 5 for s in specs)
    assert len({s["seed"] for s in specs}) == 256
    assert synth.c5_job_specs() == specs  # seeded


@pytest.mark.parametrize("name", ["c1"])
def test_make_topic_corpus_at_config_size(name):
    corpus, cfg = synth.make_topic_corpus(name)
    assert cfg == synth.CONFIGS[name]
    assert len(corpus.stream) == cfg["n_tokens"] + 1 and corpus.stream[-1] == 0
    assert len(corpus.counts) <= cfg["vocab"] + 1
    assert corpus.counts[1:].sum() == cfg["n_tokens"]
    assert np.all(np.diff(corpus.counts[1:].astype(np.int64)) <= 0)
    assert np.all(np.diff(corpus.chunk_off) == 1000)


def test_topic_corpus_on_the_device_generator_laws():
    """The device generator (torch; run here on the CPU) at a small size."""
    V, topics, n = 3000, 8, 300_000
    corpus, held = synth.topic_corpus_gpu(n, V, topics, 1.0, min_count=1, seed=5, device="cpu",
                                          heldout_tokens=20_000)
    stream = corpus.stream.numpy()
    assert stream[-1] == 0 and len(stream) == n + 1  # min_count 1 keeps every token
    assert stream[:-1].min() >= 1 and stream[:-1].max() < len(corpus.counts)
    assert np.array_equal(corpus.chunk_off.numpy(), np.arange(0, n, 1000))
    counts = corpus.counts.astype(np.int64)
    assert counts[0] == n // 1000 - 1 and np.all(np.diff(counts[1:]) <= 0)
    assert np.array_equal(np.bincount(stream[:-1], minlength=len(counts))[1:], counts[1:])
    # planted topics concentrate within a sentence (Dirichlet(0.1) weights)
    lab = corpus.label[stream[:-1]].reshape(-1, 1000)
    assert np.mean([np.bincount(r, minlength=topics).max() / 1000 for r in lab]) > 0.5
    # Zipf(1) over affine permutations: the top word of each topic is its
    # planted topic's word of rank 0, far above the median
    assert counts[1] > 20 * counts[len(counts) // 2]
    assert held is not None and len(held) <= 20_000 and held.min() >= 1


def test_c3_corpus_keeps_every_word_at_sample_1e4():
    """Subsampling never drops a word at the C3 shape: every word's expected
    share of the corpus stays below the always-keep bound of the word2vec
    rule, (sqrt(x) + 1) / x >= 1 for x = count / (sample * train_words) <=
    ((1 + sqrt 5) / 2)^2 (improved_driver_functions.cpp:60-78)."""
    c = synth.CONFIGS["c3"]
    V, topics, s = c["vocab"], c["topics"], c["zipf_s"]
    a, b = synth._affine_perms(V, topics, np.random.default_rng(1234 + 3))
    p = np.arange(1, V + 1, dtype=np.float64) ** -s
    p /= p.sum()
    share = np.zeros(V)
    words = np.arange(V, dtype=np.int64)
    for z in range(topics):
        rank = (pow(int(a[z]), -1, V) * ((words - b[z]) % V)) % V
        share += p[rank]
    share /= topics
    bound = ((1 + 5 ** 0.5) / 2) ** 2 * c["sample"]
    assert share.max() < 0.8 * bound
