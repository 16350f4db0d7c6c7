"""Chunk shuffles: the reference's libc rand() shuffle and the library's seeded
device Fisher-Yates.

  * CPU: the oracle's restatement of shuffleSentences
    (improved_driver_functions.cpp:283-291, libc rand(), unseeded), applied
    once before training (-pre-shuffle) and between epochs (-epoch-shuffle,
    FULL-W2V-driver.cu:249-266), gives the reference program's batches
    (tests/golden/shuffle_t2.npz, made by oracle/_ref/fw2v_ref_host) bit for
    bit.
  * GPU: the full-w2v program with the same flags trains to the oracle's
    vectors on those batches (deterministic mode), so its libc path shuffles
    as the reference does.
  * GPU: fw2v_shuffle_chunks permutes the chunks exactly as the oracle's
    restatement of the seeded Fisher-Yates, in shared memory and in global
    memory; with -seed the program uses it and trains to the oracle's vectors.
"""
import os
import subprocess

import numpy as np
import pytest

import fw2v
from golden_cases import GOLDEN, parse_flags
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "full-w2v_b200", "full-w2v")


def _golden():
    z = np.load(os.path.join(GOLDEN, "shuffle_t2.npz"))
    g = {k: z[k] for k in z.files}
    flags = str(g["flags"]).split()
    g["bool_flags"] = [f for f in flags if f in ("-pre-shuffle", "-epoch-shuffle")]
    g["value_flags"] = [f for f in flags if f not in g["bool_flags"]]
    g["cfg"] = parse_flags(" ".join(g["value_flags"]))
    g["text"] = g["corpus"].tobytes()
    return g


def _shuffled_samples(corpus, c, order_of_epoch, seed=0):
    return O.sample_streams(corpus, threads=c["threads"], msl=c["msl"], negative=c["negative"], epochs=c["iter"],
                            alpha0=c["alpha"], sample=c["sample"], orders=order_of_epoch, seed=seed)


def _libc_orders(chunk_off, epochs):
    """The chunk order of each epoch under -pre-shuffle -epoch-shuffle in a
    fresh process: one shuffle before training, one after every epoch but the
    last."""
    O.libc_srand(1)
    orders = [O.libc_shuffle(chunk_off)]
    for _ in range(epochs - 1):
        orders.append(O.libc_shuffle(orders[-1]))
    return orders


def test_libc_shuffles_match_reference_batches():
    g = _golden()
    c = g["cfg"]
    corpus = O.corpus_from_text(g["text"], min_count=c["min_count"], msl=c["msl"], cache_eos=False)
    out = _shuffled_samples(corpus, c, _libc_orders(corpus.chunk_off, c["iter"]))
    assert sum(e.words_read for s in out for e in s) == int(g["overall_words"])
    unmatched = list(range(int(g["n_threads"])))
    for s in out:
        lens = np.concatenate([e.lens for e in s])
        ids = np.concatenate([e.ids for e in s])
        negs = np.concatenate([e.negs for e in s])
        hit = [t for t in unmatched if np.array_equal(g[f"t{t}_lens"], lens)
               and np.array_equal(g[f"t{t}_ids"].astype(np.int32), ids)
               and np.array_equal(g[f"t{t}_negs"].astype(np.int32), negs)]
        assert hit, "a stream's shuffled batches differ from every reference thread"
        unmatched.remove(hit[0])


def _train_oracle(corpus, c, out, d, seed):
    V = len(corpus.counts)
    vec, nv, _ = fw2v.lane_layout(d)
    syn0, syn1 = O.init_syn0(V, d, d, seed=seed), np.zeros((V, d), np.float32)
    for e in range(c["iter"]):
        lens = np.concatenate([s[e].lens for s in out])
        alphas = np.concatenate([s[e].alphas for s in out])
        ids = np.concatenate([s[e].ids for s in out])
        negs = np.concatenate([s[e].negs for s in out])
        O.train(syn0, syn1, lens, alphas, ids, negs, d=d, window=c["window"], negative=c["negative"],
                sigmoid="table", precision=32, vec=vec, nv=nv)
    return syn0


def _read_vec(path):
    raw = open(path, "rb").read()
    hdr, rest = raw.split(b"\n", 1)
    V, d = (int(x) for x in hdr.split())
    rows, p = [], 0
    for _ in range(V):
        p = rest.index(b" ", p) + 1
        rows.append(np.frombuffer(rest[p:p + 4 * d], np.float32))
        p += 4 * d + 1
    return np.stack(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 7])
def test_program_shuffles_train_like_the_oracle(tmp_path, seed):
    g = _golden()
    c = g["cfg"]
    (tmp_path / "corpus.txt").write_bytes(g["text"])
    args = ["-train", "corpus.txt", "-output", "s.vec", "-binary", "1", "-debug", "0", "-deterministic", "1",
            "-seed", str(seed)] + g["value_flags"] + g["bool_flags"]
    r = subprocess.run([CLI] + args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _read_vec(tmp_path / "s.vec")
    corpus = O.corpus_from_text(g["text"], min_count=c["min_count"], msl=c["msl"], cache_eos=False)
    if seed == 0:
        orders = _libc_orders(corpus.chunk_off, c["iter"])
    else:
        key = [(seed + 0x9E3779B97F4A7C15 * (n + 1)) & (2**64 - 1) for n in range(c["iter"])]
        orders = [O.device_shuffle(corpus.chunk_off, key[0])]
        for n in range(1, c["iter"]):
            orders.append(O.device_shuffle(orders[-1], key[n]))
    want = _train_oracle(corpus, c, _shuffled_samples(corpus, c, orders, seed=seed), c["size"], seed)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("n_chunks", [1000, 28000, 60000])
def test_device_fisher_yates_matches_oracle(n_chunks):
    """Shared-memory path (up to 28k chunks of 8 bytes) and global-memory path;
    three shuffles in a row, each from the previous order."""
    msl = 2
    V = 50
    rng = np.random.default_rng(n_chunks)
    stream = np.concatenate([rng.integers(1, V, n_chunks * msl), [0]]).astype(np.int32)
    chunk_off = np.arange(0, n_chunks * msl, msl, dtype=np.int64)
    counts = np.bincount(stream, minlength=V).astype(np.uint32)
    cfg = fw2v.default_config(layer_size=8, window=1, negative=1, threads=4, msl=msl)
    with fw2v.Trainer(cfg) as t:
        t.set_vocab(counts, int(counts.sum()))
        t.load_corpus(stream, chunk_off)
        want = chunk_off
        for key in (1, 0xDEADBEEF12345678, 2**64 - 1):
            t.shuffle_chunks(key)
            want = O.device_shuffle(want, key)
            np.testing.assert_array_equal(t.chunks(n_chunks), want)
        assert sorted(want) == list(chunk_off)
