"""TEST INFRASTRUCTURE ONLY — the checker, never the product.

ctypes binding for ``oracle/build/liboracle.so`` (the C restatement of the
FULL-W2V hot path in ``fw2v_oracle.c``) plus a pure-Python restatement of the
reference's text front end (word reader, vocabulary, global token stream).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.

Reference citations are relative to the tlranda/FULL-W2V repository root.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
UNIGRAM_TABLE_SIZE = 100_000_000
MAX_STRING = 800
_lib = None


def lib():
    """Load liboracle.so, building it with make if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "build/liboracle.so"], check=True)
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


class SamplerCfg(C.Structure):
    _fields_ = [
        ("stream", C.c_void_p), ("stream_len", C.c_int64),
        ("chunk_off", C.c_void_p), ("n_chunks", C.c_int64),
        ("p_keep", C.c_void_p), ("sample", C.c_float),
        ("run_start", C.c_void_p), ("run_word", C.c_void_p), ("n_runs", C.c_int64),
        ("table_size", C.c_int64),
        ("threads", C.c_int), ("msl", C.c_int), ("negative", C.c_int), ("epochs", C.c_int),
        ("alpha0", C.c_float), ("train_words", C.c_uint64),
    ]


class StreamState(C.Structure):
    _fields_ = [("lcg", C.c_uint64), ("wca_own", C.c_uint64), ("alpha", C.c_float)]


class TrainCfg(C.Structure):
    _fields_ = [
        ("d", C.c_int), ("pitch", C.c_int64), ("window", C.c_int), ("negative", C.c_int),
        ("sigmoid", C.c_int), ("vec", C.c_int), ("nv", C.c_int), ("exp_table", C.c_void_p),
    ]


def _declare(L):
    P = C.c_void_p
    L.orc_lcg_next.restype = C.c_uint64
    L.orc_lcg_next.argtypes = [C.c_uint64]
    L.orc_exp_table.argtypes = [P]
    L.orc_init_syn0.argtypes = [P, C.c_int64, C.c_int, C.c_int64]
    L.orc_init_syn0_from.argtypes = [P, C.c_int64, C.c_int, C.c_int64, C.c_uint64]
    L.orc_subsample_table.argtypes = [P, C.c_int64, C.c_float, C.c_uint64, P]
    L.orc_unigram_runs.restype = C.c_int64
    L.orc_unigram_runs.argtypes = [P, C.c_int64, C.c_int64, P, P, P]
    L.orc_stream_init.argtypes = [C.POINTER(SamplerCfg), C.c_int, C.POINTER(StreamState)]
    L.orc_stream_range.argtypes = [C.POINTER(SamplerCfg), C.c_int, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64)]
    L.orc_sample_epoch.restype = C.c_int
    L.orc_sample_epoch.argtypes = [C.POINTER(SamplerCfg), C.c_int, C.POINTER(StreamState),
                                   C.c_int64, P, P, C.c_int64, P, P,
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_uint64)]
    L.orc_sample_epoch_prefix.restype = C.c_int
    L.orc_sample_epoch_prefix.argtypes = [C.POINTER(SamplerCfg), C.c_int, C.POINTER(StreamState), C.c_int64,
                                          C.c_int64, P, P, C.c_int64, P, P,
                                          C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                          C.POINTER(C.c_uint64)]
    for name in ("orc_train_f32", "orc_train_f64"):
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = [C.POINTER(TrainCfg), P, P, C.c_int64, C.c_int64, P, P, P, P, P]
    L.orc_train_bf16.restype = C.c_int
    L.orc_train_bf16.argtypes = [C.POINTER(TrainCfg), P, P, C.c_int64, C.c_int64, P, P, P, P, P,
                                 C.c_uint64]
    L.orc_bf16_nearest.restype = C.c_uint16
    L.orc_bf16_nearest.argtypes = [C.c_float]
    L.orc_bf16_writeback1.restype = C.c_uint16
    L.orc_bf16_writeback1.argtypes = [C.c_uint16, C.c_float, C.c_float, C.c_uint32]
    L.orc_cpu_sgns.restype = C.c_int
    L.orc_cpu_sgns.argtypes = [C.POINTER(SamplerCfg), C.POINTER(TrainCfg), P, P, C.c_int,
                               C.c_int64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.orc_heldout_loss.restype = C.c_double
    L.orc_heldout_loss.argtypes = [P, P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int64,
                                   P, P, P, P, C.POINTER(C.c_int64)]


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def lcg_next(r: int) -> int:
    return int(lib().orc_lcg_next(C.c_uint64(r)))


def exp_table() -> np.ndarray:
    t = np.zeros(1000, np.float32)
    lib().orc_exp_table(_p(t))
    return t


def seed_offset(seed: int) -> int:
    """Offset of every LCG start state and stochastic-rounding seed for a
    configuration's seed (the library's seed_offset; 0 keeps the reference's)."""
    return mix64(seed) if seed else 0


def init_syn0(V: int, d: int, pitch: int, seed: int = 0) -> np.ndarray:
    out = np.zeros((V, pitch), np.float32)
    lib().orc_init_syn0_from(_p(out), V, d, pitch, (1 + seed_offset(seed)) & (2**64 - 1))
    return out


def subsample_table(counts: np.ndarray, sample: float, train_words: int) -> np.ndarray:
    counts = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(len(counts), np.float32)
    lib().orc_subsample_table(_p(counts), len(counts), C.c_float(sample), train_words, _p(out))
    return out


def unigram_runs(counts: np.ndarray, table_size: int = UNIGRAM_TABLE_SIZE, full: bool = False):
    """Runs (start, word) of the reference unigram table; optionally the full table."""
    counts = np.ascontiguousarray(counts, np.uint32)
    V = len(counts)
    starts = np.zeros(V + 1, np.int64)
    words = np.zeros(V + 1, np.int32)
    table = np.zeros(table_size, np.int32) if full else None
    n = lib().orc_unigram_runs(_p(counts), V, table_size, _p(starts), _p(words),
                               _p(table) if full else None)
    starts = starts[: n + 1].copy()
    words = words[:n].copy()
    return (starts, words, table) if full else (starts, words)


@dataclass
class Corpus:
    """Token stream and chunk table as createGlobalStream builds them."""
    stream: np.ndarray      # int32, trailing 0 included
    chunk_off: np.ndarray   # int64
    counts: np.ndarray      # uint32 vocab counts, vocab order
    words: list = field(default_factory=list)
    train_words: int = 0


@dataclass
class StreamEpoch:
    lens: np.ndarray
    alphas: np.ndarray
    ids: np.ndarray
    negs: np.ndarray
    words_read: int


def sample_streams(corpus: Corpus, *, threads: int, msl: int, negative: int, epochs: int,
                   alpha0: float, sample: float, table_size: int = UNIGRAM_TABLE_SIZE,
                   runs=None, seed: int = 0, orders=None):
    """Run the reference batch builder for every stream and epoch.

    orders: optional chunk order of each epoch (the stored sentences permuted
    between epochs, as -pre-shuffle / -epoch-shuffle do); the streams' LCG and
    learning-rate state carry across epochs either way.
    Returns out[stream][epoch] -> StreamEpoch.
    """
    L = lib()
    stream = np.ascontiguousarray(corpus.stream, np.int32)
    counts = np.ascontiguousarray(corpus.counts, np.uint32)
    p_keep = subsample_table(counts, sample, corpus.train_words) if sample > 0 else \
        np.zeros(len(counts), np.float32)
    if runs is None:
        runs = unigram_runs(counts, table_size)
    rs, rw = runs
    if orders is None:
        orders = [corpus.chunk_off] * epochs
    orders = [np.ascontiguousarray(o, np.int64) for o in orders]
    cfgs = [SamplerCfg(_p(stream).value, len(stream), _p(o).value, len(o), _p(p_keep).value, sample,
                       _p(rs).value, _p(rw).value, len(rw), table_size, threads, msl, negative, epochs,
                       alpha0, corpus.train_words) for o in orders]
    out = []
    for s in range(threads):
        st = StreamState()
        L.orc_stream_init(C.byref(cfgs[0]), s, C.byref(st))
        st.lcg = (st.lcg + seed_offset(seed)) & (2**64 - 1)
        per_epoch = []
        for e in range(epochs):
            cfg, chunk_off = cfgs[e], orders[e]
            a, b = C.c_int64(), C.c_int64()
            L.orc_stream_range(C.byref(cfg), s, C.byref(a), C.byref(b))
            # a chunk holds at most msl + 1 tokens (msl, or up to and including a 0)
            cap = min(len(stream), (b.value - a.value) * (msl + 1)) + 2
            lens = np.zeros(cap + 2, np.int32)
            alphas = np.zeros(cap + 2, np.float32)
            ids = np.zeros(cap + 2, np.int32)
            negs = np.zeros((cap + 2) * max(negative, 1), np.int32)
            ne, nk, wr = C.c_int64(), C.c_int64(), C.c_uint64()
            rc = L.orc_sample_epoch(C.byref(cfg), s, C.byref(st), len(lens), _p(lens),
                                    _p(alphas), len(ids), _p(ids), _p(negs), C.byref(ne),
                                    C.byref(nk), C.byref(wr))
            if rc != 0:
                raise RuntimeError(f"orc_sample_epoch failed: {rc}")
            n, k = ne.value, nk.value
            per_epoch.append(StreamEpoch(lens[:n].copy(), alphas[:n].copy(), ids[:k].copy(),
                                         negs[: k * negative].copy(), int(wr.value)))
        out.append(per_epoch)
    return out


def sample_stream_prefix(corpus: Corpus, stream_id: int, max_entries: int, *, threads: int, msl: int,
                         negative: int, alpha0: float, sample: float, table_size: int = UNIGRAM_TABLE_SIZE,
                         epochs: int = 1) -> StreamEpoch:
    """The first max_entries batch entries of stream stream_id's first epoch
    (orc_sample_epoch_prefix, the CPU baseline's bounded sample), with the
    tokens they consumed."""
    L = lib()
    stream = np.ascontiguousarray(corpus.stream, np.int32)
    chunk_off = np.ascontiguousarray(corpus.chunk_off, np.int64)
    counts = np.ascontiguousarray(corpus.counts, np.uint32)
    p_keep = subsample_table(counts, sample, corpus.train_words) if sample > 0 else \
        np.zeros(len(counts), np.float32)
    rs, rw = unigram_runs(counts, table_size)
    cfg = SamplerCfg(_p(stream).value, len(stream), _p(chunk_off).value, len(chunk_off), _p(p_keep).value, sample,
                     _p(rs).value, _p(rw).value, len(rw), table_size, threads, msl, negative, epochs, alpha0,
                     corpus.train_words)
    st = StreamState()
    L.orc_stream_init(C.byref(cfg), stream_id, C.byref(st))
    cap = len(stream) + 2
    lens = np.zeros(cap, np.int32)
    alphas = np.zeros(cap, np.float32)
    ids = np.zeros(cap, np.int32)
    negs = np.zeros(cap * max(negative, 1), np.int32)
    ne, nk, wr = C.c_int64(), C.c_int64(), C.c_uint64()
    rc = L.orc_sample_epoch_prefix(C.byref(cfg), stream_id, C.byref(st), max_entries, cap, _p(lens), _p(alphas),
                                   cap, _p(ids), _p(negs), C.byref(ne), C.byref(nk), C.byref(wr))
    if rc != 0:
        raise RuntimeError(f"orc_sample_epoch_prefix failed: {rc}")
    n, k = ne.value, nk.value
    return StreamEpoch(lens[:n].copy(), alphas[:n].copy(), ids[:k].copy(), negs[: k * negative].copy(),
                       int(wr.value))


def libc_shuffle(chunk_off: np.ndarray) -> np.ndarray:
    """shuffleSentences (improved_driver_functions.cpp:283-291): Fisher-Yates
    over the stored sentence pointers with the C library's rand(), from i =
    n-1 down to 1, j = (int)((rand() / (double)RAND_MAX) * (i + 1)) (j = i + 1,
    when rand() returns RAND_MAX, is taken as i: the reference would index one
    past the array).  Continues this process's rand() sequence, as the
    reference's successive shuffles continue its own; call libc_srand(1) first
    for the sequence of a fresh process."""
    libc = C.CDLL(None)
    libc.rand.restype = C.c_int
    out = np.array(chunk_off, np.int64, copy=True)
    n = len(out)
    RAND_MAX = 2147483647
    for i in range(n - 1, 0, -1):
        j = int((libc.rand() / float(RAND_MAX)) * (i + 1))
        j = min(j, i)
        out[i], out[j] = out[j], out[i]
    return out


def libc_srand(seed: int) -> None:
    C.CDLL(None).srand(C.c_uint(seed))


def device_shuffle(chunk_off: np.ndarray, key: int) -> np.ndarray:
    """The library's seeded Fisher-Yates (fw2v_shuffle_chunks): from i = n-1 down
    to 1, j = the high 64 bits of mix64(key ^ mix64(i)) * (i + 1), swap."""
    out = np.array(chunk_off, np.int64, copy=True)
    for i in range(len(out) - 1, 0, -1):
        j = (mix64(key ^ mix64(i)) * (i + 1)) >> 64
        out[i], out[j] = out[j], out[i]
    return out


def cpu_sgns(corpus: Corpus, syn0, syn1neg, *, threads: int, msl: int, negative: int,
             epochs: int, alpha0: float, sample: float, d: int, window: int, n_threads: int,
             max_entries_per_stream: int = 0, sigmoid: str = "table"):
    """Timed CPU baseline: sample + train every stream on n_threads host threads.

    Returns (words_read, words_kept); tables are updated in place (Hogwild)."""
    L = lib()
    stream = np.ascontiguousarray(corpus.stream, np.int32)
    chunk_off = np.ascontiguousarray(corpus.chunk_off, np.int64)
    counts = np.ascontiguousarray(corpus.counts, np.uint32)
    p_keep = subsample_table(counts, sample, corpus.train_words) if sample > 0 else \
        np.zeros(len(counts), np.float32)
    rs, rw = unigram_runs(counts)
    scfg = SamplerCfg(_p(stream).value, len(stream), _p(chunk_off).value, len(chunk_off),
                      _p(p_keep).value, sample, _p(rs).value, _p(rw).value, len(rw),
                      UNIGRAM_TABLE_SIZE, threads, msl, negative, epochs, alpha0,
                      corpus.train_words)
    table = exp_table()
    tcfg = _train_cfg(d, syn0.shape[1], window, negative, 0 if sigmoid == "table" else 1, 4, 1,
                      table)
    wr, wk = C.c_uint64(), C.c_uint64()
    rc = L.orc_cpu_sgns(C.byref(scfg), C.byref(tcfg), _p(syn0), _p(syn1neg), n_threads,
                        max_entries_per_stream, C.byref(wr), C.byref(wk))
    if rc != 0:
        raise RuntimeError(f"orc_cpu_sgns failed: {rc}")
    return int(wr.value), int(wk.value)


def _train_cfg(d, pitch, window, negative, sigmoid, vec, nv, table):
    return TrainCfg(d, pitch, window, negative, sigmoid, vec, nv, _p(table).value)


def train(syn0, syn1neg, lens, alphas, ids, negs, *, d, window, negative, sigmoid="table",
          precision=32, vec=4, nv=1):
    """Serial SGNS over the sentences in order; updates syn0/syn1neg in place.

    precision 32: float32 tables, kernel-order arithmetic; 64: float64 tables.
    """
    table = exp_table()
    pitch = syn0.shape[1]
    cfg = _train_cfg(d, pitch, window, negative, 0 if sigmoid == "table" else 1, vec, nv, table)
    lens = np.ascontiguousarray(lens, np.int32)
    starts = np.zeros(len(lens), np.int64)
    if len(lens) > 1:
        starts[1:] = np.cumsum(lens[:-1].astype(np.int64))
    alphas = np.ascontiguousarray(alphas, np.float32)
    ids = np.ascontiguousarray(ids, np.int32)
    negs = np.ascontiguousarray(negs, np.int32)
    if negs.size == 0:
        negs = np.zeros(1, np.int32)
    fn = lib().orc_train_f32 if precision == 32 else lib().orc_train_f64
    want = np.float32 if precision == 32 else np.float64
    assert syn0.dtype == want and syn1neg.dtype == want
    assert syn0.flags.c_contiguous and syn1neg.flags.c_contiguous
    rc = fn(C.byref(cfg), _p(syn0), _p(syn1neg), syn0.shape[0], len(lens), _p(starts),
            _p(lens), _p(alphas), _p(ids), _p(negs))
    if rc != 0:
        raise RuntimeError(f"oracle train failed: {rc}")


def mix64(z: int) -> int:
    M = (1 << 64) - 1
    z = (z + 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns, round to nearest even."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_float(h: np.ndarray) -> np.ndarray:
    return (h.astype(np.uint32) << 16).view(np.float32)


def bf16_writeback1(stored: int, a: float, b: float, r16: int) -> int:
    """One element of the bfloat16 write-back: the stored bits after the row
    moved from b to a, with 16 random bits."""
    return int(lib().orc_bf16_writeback1(stored, a, b, r16))


def train_bf16(syn0, syn1neg, lens, alphas, ids, negs, *, d, window, negative, seed, sigmoid="table",
               vec=4, nv=1):
    """Serial SGNS on bfloat16 tables (uint16 arrays, updated in place) with the
    library's stochastic rounding (seed = the training launch's seed)."""
    table = exp_table()
    cfg = _train_cfg(d, syn0.shape[1], window, negative, 0 if sigmoid == "table" else 1, vec, nv, table)
    lens = np.ascontiguousarray(lens, np.int32)
    starts = np.zeros(len(lens), np.int64)
    if len(lens) > 1:
        starts[1:] = np.cumsum(lens[:-1].astype(np.int64))
    alphas = np.ascontiguousarray(alphas, np.float32)
    ids = np.ascontiguousarray(ids, np.int32)
    negs = np.ascontiguousarray(negs, np.int32) if negs.size else np.zeros(1, np.int32)
    assert syn0.dtype == np.uint16 and syn1neg.dtype == np.uint16
    rc = lib().orc_train_bf16(C.byref(cfg), _p(syn0), _p(syn1neg), syn0.shape[0], len(lens),
                              _p(starts), _p(lens), _p(alphas), _p(ids), _p(negs), seed)
    if rc != 0:
        raise RuntimeError(f"oracle bf16 train failed: {rc}")


def heldout_loss(syn0, syn1neg, lens, ids, negs, *, d, window, negative):
    lens = np.ascontiguousarray(lens, np.int32)
    starts = np.zeros(len(lens), np.int64)
    if len(lens) > 1:
        starts[1:] = np.cumsum(lens[:-1].astype(np.int64))
    ids = np.ascontiguousarray(ids, np.int32)
    negs = np.ascontiguousarray(negs, np.int32) if negs.size else np.zeros(1, np.int32)
    pairs = C.c_int64()
    tot = lib().orc_heldout_loss(_p(syn0), _p(syn1neg), syn0.shape[1], d, window, negative,
                                 len(lens), _p(starts), _p(lens), _p(ids), _p(negs),
                                 C.byref(pairs))
    return float(tot), int(pairs.value)


# ---------------------------------------------------------------------------
# Text front end (improved_driver_functions.cpp:86-164, 244-281;
# legacy_driver_functions.cpp:26-95)
# ---------------------------------------------------------------------------

def read_word(buf: bytes, pos: int):
    """improved_driver_functions.cpp:86-124 (mmap ReadWord). Returns (word, new_pos)."""
    n = len(buf)
    word = bytearray()
    read = 0
    while pos < n:
        read = buf[pos]
        pos += 1
        if read == 13:
            continue
        if read == 10:
            if len(word) > 0:
                pos -= 1
                break
            return b"</s>", pos
        if read == 32 or read == 9:
            if len(word) > 0:
                break
            continue
        word.append(read)
        if len(word) >= MAX_STRING - 1:
            break
    if pos == n or read in (32, 9, 10):
        return bytes(word), pos
    while pos < n and read not in (32, 9, 10):
        read = buf[pos]
        pos += 1
    return bytes(word), pos - 1


def learn_vocab(buf: bytes, min_count: int):
    """LearnVocabFromTrainFile + SortVocab (improved:136-164, legacy:74-95).

    Returns (words, counts, train_words).  The sort is stable (glibc's qsort
    is a stable merge sort), count descending, </s> pinned at index 0.
    """
    index = {b"</s>": 0}
    words = [b"</s>"]
    counts = [0]
    pos, n = 0, len(buf)
    while pos < n:
        w, pos = read_word(buf, pos)
        if pos == n:
            break
        i = index.get(w)
        if i is None:
            index[w] = len(words)
            words.append(w)
            counts.append(1)
        else:
            counts[i] += 1
    order = sorted(range(1, len(words)), key=lambda k: -counts[k])
    order = [0] + [k for k in order if counts[k] >= min_count]
    words = [words[k] for k in order]
    counts = [counts[k] for k in order]
    train_words = sum(counts) + 1
    return words, np.array(counts, np.uint32), train_words


def create_stream(buf: bytes, words, msl: int, cache_eos: bool):
    """createGlobalStream (improved:244-281). OOV words are skipped
    (ReadWordIndex, improved:127-134)."""
    index = {w: i for i, w in enumerate(words)}
    stream, chunk_off = [], []
    sent_length = 0
    pos, n = 0, len(buf)
    while pos < n:
        w = -1
        while pos < n and w == -1:
            tok, pos = read_word(buf, pos)
            w = index.get(tok, -1)
        if w == -1:
            break  # OOV run reached EOF; the reference would store -1 here
        if cache_eos or w != 0:
            if sent_length == 0:
                chunk_off.append(len(stream))
            stream.append(w)
            sent_length += 1
            if w == 0 or sent_length >= msl:
                sent_length = 0
    stream.append(0)
    return np.array(stream, np.int32), np.array(chunk_off, np.int64)


def _sort_cut(words, counts, min_count):
    order = sorted(range(1, len(words)), key=lambda k: -counts[k])
    order = [0] + [k for k in order if counts[k] >= min_count]
    return [words[k] for k in order], [counts[k] for k in order]


def read_vocab(buf: bytes, min_count: int):
    """ReadVocab (improved_driver_functions.cpp:167-196): "word count" pairs,
    then SortVocab.  train_words is the sum of the kept counts."""
    words, counts = [], []
    pos, n = 0, len(buf)
    while pos < n:
        w, pos = read_word(buf, pos)
        c, pos = read_word(buf, pos)
        words.append(w)
        counts.append(int(c) & 0xFFFFFFFF if c.lstrip(b"-").isdigit() else 0)
        pos += 1
    words, counts = _sort_cut(words, counts, min_count)
    return words, np.array(counts, np.uint32), int(sum(counts))


def read_corpus_cache(buf: bytes, msl: int, cache_eos: bool):
    """readCorpusCache (improved_driver_functions.cpp:320-401).

    Header "S N": N is train_words.  A "</s>" ends a chunk when cache_eos; an
    id arriving after msl ids of a chunk starts a new one (a 0 is stored between).
    The last chunk pointer, which points past the last chunk started, is not a
    sentence (sentence_count = pointers - 1), so that chunk is never read.
    Returns (stream with a trailing 0, chunk offsets, train_words)."""
    pos = 0
    _, pos = read_word(buf, pos)
    tw, pos = read_word(buf, pos)
    pos += 1
    stream, offs = [], [0]
    trigger = 0
    n = len(buf)
    while pos < n:
        w, pos = read_word(buf, pos)
        if w == b"</s>":
            if cache_eos:
                stream.append(0)
                offs.append(len(stream))
                trigger = 0
        else:
            if trigger == msl:
                stream.append(0)
                offs.append(len(stream))
                trigger = 0
            else:
                trigger += 1
            stream.append(int(w))
    offs.pop()
    stream.append(0)
    return np.array(stream, np.int32), np.array(offs, np.int64), int(tw)


def corpus_from_text(buf: bytes, *, min_count: int, msl: int, cache_eos: bool) -> Corpus:
    words, counts, tw = learn_vocab(buf, min_count)
    stream, chunk_off = create_stream(buf, words, msl, cache_eos)
    return Corpus(stream, chunk_off, counts, words, tw)
