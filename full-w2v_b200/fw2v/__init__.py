"""Python binding of libfw2v.so, the B200 SGNS trainer (C ABI: include/fw2v.h).

This mirrors the reference's training path (tlranda/FULL-W2V
``src/FULL-W2V/FULL-W2V-driver.cu``): a vocabulary with counts, a token stream
cut into stored sentence chunks, and the epoch loop of ``Train_SGNS`` — here
an on-device batch builder and training kernel behind a handle.  Errors raise
``Fw2vError`` with the library's status and message; the library never exits
the process.  There is no CPU fallback: without the built library or a B200
the calls fail.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libfw2v.so")

FP32, BF16 = 0, 1
SIGMOID_TABLE, SIGMOID_EXACT = 0, 1
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
          4: "call out of order", 5: "id out of range", 6: "no usable CUDA device",
          7: "request exceeds a fixed-size library buffer"}
NOALLOC_SCRATCH_BYTES = 16 << 20


class Fw2vError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"fw2v status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [
        ("layer_size", C.c_int32), ("window", C.c_int32), ("negative", C.c_int32),
        ("epochs", C.c_int32), ("threads", C.c_int32), ("msl", C.c_int32),
        ("alpha", C.c_float), ("sample", C.c_float), ("sigmoid", C.c_int32),
        ("precision", C.c_int32), ("deterministic", C.c_int32), ("device", C.c_int32),
        ("seed", C.c_uint64),
    ]


class EpochStats(C.Structure):
    _fields_ = [("words_read", C.c_uint64), ("words_kept", C.c_uint64),
                ("sentences", C.c_uint64), ("sampler_ms", C.c_float), ("train_ms", C.c_float)]


class BatchConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("use_graph", C.c_int32),
                ("deterministic", C.c_int32), ("round_tokens", C.c_int64),
                ("group_bytes", C.c_int64)]


class BatchStats(C.Structure):
    _fields_ = [("words_read", C.c_uint64), ("words_kept", C.c_uint64), ("ms", C.c_float),
                ("epochs", C.c_int32), ("rounds", C.c_int32), ("train_ms", C.c_float),
                ("train_launches", C.c_int32)]


class TuneReport(C.Structure):
    _fields_ = [("n_classes", C.c_int32), ("class_d", C.c_int32 * 16), ("class_window", C.c_int32 * 16),
                ("class_lane_vec", C.c_int32 * 16), ("class_lane_nv", C.c_int32 * 16),
                ("class_stages", C.c_int32 * 16), ("class_prefetch", C.c_int32 * 16),
                ("tuned_wps", C.c_double * 16),
                ("default_wps", C.c_double * 16), ("warps_per_block", C.c_int32 * 3),
                ("blocks_per_sm", C.c_int32 * 3)]


# Every entry point declared in include/fw2v.h (tests check the library exports them all).
EXPORTS = [
    "fw2v_config_default", "fw2v_create", "fw2v_destroy", "fw2v_set_vocab", "fw2v_load_corpus",
    "fw2v_load_corpus_device", "fw2v_sample_epoch", "fw2v_epoch_sample_sizes", "fw2v_epoch_samples", "fw2v_train_sampled",
    "fw2v_train_epoch", "fw2v_train", "fw2v_words_trained", "fw2v_get_syn0", "fw2v_get_syn1neg",
    "fw2v_set_tables", "fw2v_train_sentences", "fw2v_heldout_loss", "fw2v_kernel_batch",
    "fw2v_kernel_batch_error", "fw2v_lane_layout", "fw2v_exp_table", "fw2v_unigram_firsts",
    "fw2v_get_unigram", "fw2v_status_string", "fw2v_last_error", "fw2v_version", "fw2v_stream",
    "fw2v_kernel_batch_noalloc", "fw2v_reorder_chunks", "fw2v_shuffle_chunks", "fw2v_get_chunks",
    "fw2v_batch_config_default", "fw2v_batch_create", "fw2v_batch_destroy", "fw2v_batch_last_error",
    "fw2v_batch_add_job", "fw2v_batch_add_job_device", "fw2v_batch_set_shape", "fw2v_batch_get_shape", "fw2v_batch_set_launch",
    "fw2v_batch_get_launch", "fw2v_batch_tune", "fw2v_batch_train", "fw2v_batch_train_epochs",
    "fw2v_batch_job_words",
    "fw2v_batch_get_syn0", "fw2v_batch_get_syn1neg", "fw2v_neighbours", "fw2v_random_walks",
    "fw2v_relabel_stream",
]

_lib = None


def lib() -> C.CDLL:
    """Load libfw2v.so from the package directory (built by `make -C full-w2v_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run make -C full-w2v_b200")
        L = C.CDLL(LIB_PATH)
        P, I32, I64, U64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
        H = C.c_void_p
        sig = {
            "fw2v_config_default": (None, [C.POINTER(Config)]),
            "fw2v_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
            "fw2v_destroy": (None, [H]),
            "fw2v_set_vocab": (C.c_int, [H, P, I64, U64]),
            "fw2v_load_corpus": (C.c_int, [H, P, I64, P, I64]),
            "fw2v_load_corpus_device": (C.c_int, [H, P, I64, P, I64]),
            "fw2v_reorder_chunks": (C.c_int, [H, P, I64]),
            "fw2v_shuffle_chunks": (C.c_int, [H, U64]),
            "fw2v_get_chunks": (C.c_int, [H, P]),
            "fw2v_sample_epoch": (C.c_int, [H]),
            "fw2v_epoch_sample_sizes": (C.c_int, [H, C.POINTER(I64), C.POINTER(I64)]),
            "fw2v_epoch_samples": (C.c_int, [H, P, P, P, P, P, P, P]),
            "fw2v_train_sampled": (C.c_int, [H, C.POINTER(EpochStats)]),
            "fw2v_train_epoch": (C.c_int, [H, C.POINTER(EpochStats)]),
            "fw2v_train": (C.c_int, [H, C.POINTER(U64)]),
            "fw2v_words_trained": (C.c_int, [H, C.POINTER(U64)]),
            "fw2v_get_syn0": (C.c_int, [H, P, I64]),
            "fw2v_get_syn1neg": (C.c_int, [H, P, I64]),
            "fw2v_set_tables": (C.c_int, [H, P, P, I64]),
            "fw2v_train_sentences": (C.c_int, [H, P, P, P, P, P, I64]),
            "fw2v_heldout_loss": (C.c_int, [H, P, P, P, P, I64, C.POINTER(C.c_double),
                                            C.POINTER(I64)]),
            "fw2v_kernel_batch": (C.c_int, [P, P, P, P, P, P, I32, I32, I32, I32, I32,
                                            C.c_uint32, I64, P]),
            "fw2v_kernel_batch_error": (C.c_int, [P]),
            "fw2v_kernel_batch_noalloc": (C.c_int, [P, P, P, P, P, P, I32, I32, I32, I32, I32,
                                                    C.c_uint32, I64, P]),
            "fw2v_lane_layout": (None, [I32, I32, C.POINTER(I32), C.POINTER(I32),
                                        C.POINTER(I64)]),
            "fw2v_exp_table": (None, [P]),
            "fw2v_unigram_firsts": (C.c_int, [P, I64, I64, P]),
            "fw2v_get_unigram": (C.c_int, [H, I64, I64, P]),
            "fw2v_status_string": (C.c_char_p, [C.c_int]),
            "fw2v_last_error": (C.c_char_p, [H]),
            "fw2v_version": (C.c_char_p, []),
            "fw2v_stream": (C.c_void_p, [H]),
            "fw2v_batch_config_default": (None, [C.POINTER(BatchConfig)]),
            "fw2v_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.POINTER(C.c_void_p)]),
            "fw2v_batch_destroy": (None, [H]),
            "fw2v_batch_last_error": (C.c_char_p, [H]),
            "fw2v_batch_add_job": (C.c_int, [H, C.POINTER(Config), P, I64, U64, P, I64, P, I64,
                                             C.POINTER(I32)]),
            "fw2v_batch_add_job_device": (C.c_int, [H, C.POINTER(Config), P, I64, U64, P, I64, P, I64,
                                                    C.POINTER(I32)]),
            "fw2v_batch_set_shape": (C.c_int, [H, I32, I32, I32, I32, I32]),
            "fw2v_batch_get_shape": (C.c_int, [H, I32, C.POINTER(I32), C.POINTER(I32), C.POINTER(I32),
                                               C.POINTER(I32)]),
            "fw2v_batch_set_launch": (C.c_int, [H, I32, I32, I32]),
            "fw2v_batch_get_launch": (C.c_int, [H, I32, C.POINTER(I32), C.POINTER(I32)]),
            "fw2v_batch_tune": (C.c_int, [H, I64, C.POINTER(TuneReport)]),
            "fw2v_batch_train": (C.c_int, [H, C.POINTER(BatchStats)]),
            "fw2v_batch_train_epochs": (C.c_int, [H, I32, C.POINTER(BatchStats)]),
            "fw2v_batch_job_words": (C.c_int, [H, I32, C.POINTER(U64), C.POINTER(U64)]),
            "fw2v_batch_get_syn0": (C.c_int, [H, I32, P, I64]),
            "fw2v_batch_get_syn1neg": (C.c_int, [H, I32, P, I64]),
            "fw2v_neighbours": (C.c_int, [P, I32, I64, I32, P, I64, P, I64, I32, P, P, P]),
            "fw2v_random_walks": (C.c_int, [P, P, I64, P, I64, I32, U64, P, P]),
            "fw2v_relabel_stream": (C.c_int, [P, I64, P, I64, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _on_device(a) -> bool:
    return type(a).__module__.startswith("torch") and a.is_cuda


def _device_pair(stream, chunk_off):
    """A device stream (int32) and its chunk offsets (int64) as contiguous CUDA
    tensors on the stream's device (offsets given on the host are copied)."""
    import torch
    st = stream.to(torch.int32).contiguous()
    co = chunk_off if _on_device(chunk_off) else torch.from_numpy(np.ascontiguousarray(chunk_off, np.int64))
    co = co.to(device=st.device, dtype=torch.int64).contiguous()
    torch.cuda.current_stream(st.device).synchronize()  # the tensors are written before the library reads them
    return st, co


def default_config(**overrides) -> Config:
    c = Config()
    lib().fw2v_config_default(C.byref(c))
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def lane_layout(layer_size: int, precision: int = FP32):
    vec, nv, pitch = C.c_int32(), C.c_int32(), C.c_int64()
    lib().fw2v_lane_layout(layer_size, precision, C.byref(vec), C.byref(nv), C.byref(pitch))
    return vec.value, nv.value, pitch.value


def exp_table() -> np.ndarray:
    t = np.zeros(1000, np.float32)
    lib().fw2v_exp_table(_p(t))
    return t


def unigram_firsts(counts: np.ndarray, table_size: int = 100_000_000) -> np.ndarray:
    counts = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(len(counts) - 1, np.int64)
    if lib().fw2v_unigram_firsts(_p(counts), len(counts), table_size, _p(out)) != 0:
        raise ValueError("vocabulary needs at least two words")
    return out


class Trainer:
    """One SGNS job on one GPU (a libfw2v handle)."""

    def __init__(self, config: Config | None = None, **overrides):
        cfg = config if config is not None else default_config()
        for k, v in overrides.items():
            setattr(cfg, k, v)
        self.config = cfg
        h = C.c_void_p()
        st = lib().fw2v_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise Fw2vError(st, "fw2v_create")
        self._h = h
        self.vocab_size = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().fw2v_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, what: str):
        if st != 0:
            msg = lib().fw2v_last_error(self._h)
            raise Fw2vError(st, f"{what}: {msg.decode() if msg else ''}")

    # -- setup ---------------------------------------------------------------
    def set_vocab(self, counts: np.ndarray, train_words: int):
        counts = np.ascontiguousarray(counts, np.uint32)
        self._check(lib().fw2v_set_vocab(self._h, _p(counts), len(counts), int(train_words)),
                    "set_vocab")
        self.vocab_size = len(counts)

    def load_corpus(self, stream, chunk_off):
        """Token stream and chunk offsets: numpy arrays (host memory), or CUDA
        tensors (int32 / int64), which are loaded on the device without a host
        round trip (fw2v_load_corpus_device)."""
        if _on_device(stream):
            st, co = _device_pair(stream, chunk_off)
            self._check(lib().fw2v_load_corpus_device(self._h, st.data_ptr(), st.numel(), co.data_ptr(),
                                                      co.numel()), "load_corpus_device")
            return
        stream = np.ascontiguousarray(stream, np.int32)
        chunk_off = np.ascontiguousarray(chunk_off, np.int64)
        self._check(lib().fw2v_load_corpus(self._h, _p(stream), len(stream), _p(chunk_off),
                                           len(chunk_off)), "load_corpus")

    def reorder_chunks(self, chunk_off: np.ndarray):
        chunk_off = np.ascontiguousarray(chunk_off, np.int64)
        self._check(lib().fw2v_reorder_chunks(self._h, _p(chunk_off), len(chunk_off)),
                    "reorder_chunks")

    def shuffle_chunks(self, key: int):
        """Seeded Fisher-Yates of the stored chunks on the device."""
        self._check(lib().fw2v_shuffle_chunks(self._h, key & (2**64 - 1)), "shuffle_chunks")

    def chunks(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.int64)
        self._check(lib().fw2v_get_chunks(self._h, _p(out)), "get_chunks")
        return out

    # -- epoch loop ----------------------------------------------------------
    def sample_epoch(self):
        self._check(lib().fw2v_sample_epoch(self._h), "sample_epoch")

    def epoch_samples(self):
        """Last sampled epoch: per-stream lists of (lens, alphas, ids, negs, words_read)."""
        ne, nk = C.c_int64(), C.c_int64()
        self._check(lib().fw2v_epoch_sample_sizes(self._h, C.byref(ne), C.byref(nk)), "sizes")
        T, K = self.config.threads, self.config.negative
        lens = np.zeros(max(ne.value, 1), np.int32)
        alphas = np.zeros(max(ne.value, 1), np.float32)
        ids = np.zeros(max(nk.value, 1), np.int32)
        negs = np.zeros(max(nk.value * K, 1), np.int32)
        eps = np.zeros(T, np.int64)
        kps = np.zeros(T, np.int64)
        wps = np.zeros(T, np.uint64)
        self._check(lib().fw2v_epoch_samples(self._h, _p(lens), _p(alphas), _p(ids), _p(negs),
                                             _p(eps), _p(kps), _p(wps)), "epoch_samples")
        out, eo, ko = [], 0, 0
        for s in range(T):
            e, k = int(eps[s]), int(kps[s])
            out.append((lens[eo:eo + e].copy(), alphas[eo:eo + e].copy(), ids[ko:ko + k].copy(),
                        negs[ko * K:(ko + k) * K].copy(), int(wps[s])))
            eo += e
            ko += k
        return out

    def train_sampled(self) -> EpochStats:
        st = EpochStats()
        self._check(lib().fw2v_train_sampled(self._h, C.byref(st)), "train_sampled")
        return st

    def train_epoch(self) -> EpochStats:
        st = EpochStats()
        self._check(lib().fw2v_train_epoch(self._h, C.byref(st)), "train_epoch")
        return st

    def train(self) -> int:
        w = C.c_uint64()
        self._check(lib().fw2v_train(self._h, C.byref(w)), "train")
        return int(w.value)

    def words_trained(self) -> int:
        w = C.c_uint64()
        self._check(lib().fw2v_words_trained(self._h, C.byref(w)), "words_trained")
        return int(w.value)

    # -- tables --------------------------------------------------------------
    def syn0(self) -> np.ndarray:
        out = np.zeros((self.vocab_size, self.config.layer_size), np.float32)
        self._check(lib().fw2v_get_syn0(self._h, _p(out), self.config.layer_size), "get_syn0")
        return out

    def syn1neg(self) -> np.ndarray:
        out = np.zeros((self.vocab_size, self.config.layer_size), np.float32)
        self._check(lib().fw2v_get_syn1neg(self._h, _p(out), self.config.layer_size),
                    "get_syn1neg")
        return out

    def set_tables(self, syn0: np.ndarray | None, syn1neg: np.ndarray | None):
        d = self.config.layer_size
        a = None if syn0 is None else np.ascontiguousarray(syn0, np.float32)
        b = None if syn1neg is None else np.ascontiguousarray(syn1neg, np.float32)
        self._check(lib().fw2v_set_tables(self._h, _p(a), _p(b), d), "set_tables")

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) every kernel of this trainer runs on."""
        return lib().fw2v_stream(self._h) or 0

    def unigram(self, first: int, n: int) -> np.ndarray:
        out = np.zeros(n, np.int32)
        self._check(lib().fw2v_get_unigram(self._h, first, n, _p(out)), "get_unigram")
        return out

    # -- explicit sentences ----------------------------------------------------
    @staticmethod
    def _pack(lens, ids, negs):
        lens = np.ascontiguousarray(lens, np.int32)
        starts = np.zeros(len(lens), np.int64)
        if len(lens) > 1:
            starts[1:] = np.cumsum(lens[:-1].astype(np.int64))
        ids = np.ascontiguousarray(ids, np.int32)
        negs = np.ascontiguousarray(negs, np.int32)
        return lens, starts, ids, negs

    def train_sentences(self, lens, alphas, ids, negs):
        lens, starts, ids, negs = self._pack(lens, ids, negs)
        alphas = np.ascontiguousarray(alphas, np.float32)
        self._check(lib().fw2v_train_sentences(self._h, _p(ids), _p(negs) if negs.size else None,
                                               _p(starts), _p(lens), _p(alphas), len(lens)),
                    "train_sentences")

    def heldout_loss(self, lens, ids, negs):
        lens, starts, ids, negs = self._pack(lens, ids, negs)
        loss, pairs = C.c_double(), C.c_int64()
        self._check(lib().fw2v_heldout_loss(self._h, _p(ids), _p(negs) if negs.size else None,
                                            _p(starts), _p(lens), len(lens), C.byref(loss),
                                            C.byref(pairs)), "heldout_loss")
        return loss.value, pairs.value


class Batch:
    """Many independent SGNS jobs trained together on one GPU (a libfw2v
    batch): one persistent training kernel per round drains a work queue of
    (job, sentence) items from every job.  Jobs need layer_size <= 384, the
    table sigmoid and the same `negative`."""

    def __init__(self, precision: int = FP32, device: int = 0, use_graph: bool = True,
                 deterministic: bool = False, round_tokens: int = 0, group_bytes: int = 0):
        cfg = BatchConfig()
        lib().fw2v_batch_config_default(C.byref(cfg))
        cfg.precision, cfg.device = precision, device
        cfg.use_graph, cfg.deterministic, cfg.round_tokens = int(use_graph), int(deterministic), round_tokens
        cfg.group_bytes = group_bytes
        h = C.c_void_p()
        st = lib().fw2v_batch_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise Fw2vError(st, "fw2v_batch_create")
        self._h = h
        self.config = cfg
        self.jobs: list[tuple[Config, int]] = []

    def close(self):
        if getattr(self, "_h", None):
            lib().fw2v_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, what: str):
        if st != 0:
            msg = lib().fw2v_batch_last_error(self._h)
            raise Fw2vError(st, f"{what}: {msg.decode() if msg else ''}")

    def add_job(self, config: Config, counts: np.ndarray, train_words: int, stream, chunk_off) -> int:
        """A job; its stream and chunk offsets as numpy arrays or as CUDA
        tensors (loaded on the device, fw2v_batch_add_job_device)."""
        counts = np.ascontiguousarray(counts, np.uint32)
        j = C.c_int32()
        if _on_device(stream):
            st, co = _device_pair(stream, chunk_off)
            self._check(lib().fw2v_batch_add_job_device(self._h, C.byref(config), _p(counts), len(counts),
                                                        int(train_words), st.data_ptr(), st.numel(), co.data_ptr(),
                                                        co.numel(), C.byref(j)), "batch_add_job_device")
        else:
            stream = np.ascontiguousarray(stream, np.int32)
            chunk_off = np.ascontiguousarray(chunk_off, np.int64)
            self._check(lib().fw2v_batch_add_job(self._h, C.byref(config), _p(counts), len(counts),
                                                 int(train_words), _p(stream), len(stream), _p(chunk_off),
                                                 len(chunk_off), C.byref(j)), "batch_add_job")
        self.jobs.append((config, len(counts)))
        return j.value

    def set_shape(self, job: int, lane_vec: int, lane_nv: int, stages: int, prefetch: int = 0):
        self._check(lib().fw2v_batch_set_shape(self._h, job, lane_vec, lane_nv, stages, prefetch),
                    "batch_set_shape")

    def shape(self, job: int) -> tuple[int, int, int, int]:
        """(lane vector width, vectors per lane, stages, prefetch)."""
        v, n, s, p = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self._check(lib().fw2v_batch_get_shape(self._h, job, C.byref(v), C.byref(n), C.byref(s), C.byref(p)),
                    "batch_get_shape")
        return v.value, n.value, s.value, p.value

    def set_launch(self, family: int, warps_per_block: int, blocks_per_sm: int = 0):
        """Warps per block of a kernel family (1..8, 1..6, 1..4 for families
        0, 1, 2; 0: the count that keeps the most warps resident) and a cap on
        blocks per SM (0: as many as fit)."""
        self._check(lib().fw2v_batch_set_launch(self._h, family, warps_per_block, blocks_per_sm),
                    "batch_set_launch")

    def launch(self, family: int) -> tuple[int, int]:
        w, b = C.c_int32(), C.c_int32()
        self._check(lib().fw2v_batch_get_launch(self._h, family, C.byref(w), C.byref(b)), "batch_get_launch")
        return w.value, b.value

    def tune(self, sample_tokens: int = 0, cache: str | None = None) -> dict:
        """Pick every job class's shape and the grid by measurement
        (fw2v_batch_tune).  With `cache`, a JSON file of earlier choices keyed
        by device, precision and (d class, window, negative): classes found
        there are applied without timing; if all are, nothing is timed."""
        import json

        keys = [self._class_key(c) for c, _ in self.jobs]
        launch_keys = [f"launch{f}:{self._device_key()}" for f in (0, 1, 2)]
        store = {}
        if cache and os.path.exists(cache):
            with open(cache) as f:
                store = json.load(f)
        if keys and all(k in store for k in keys + launch_keys):
            for j, k in enumerate(keys):
                self.set_shape(j, *store[k])
            for f, k in enumerate(launch_keys):
                self.set_launch(f, *store[k])
            return {"cached": True}
        rep = TuneReport()
        self._check(lib().fw2v_batch_tune(self._h, int(sample_tokens), C.byref(rep)), "batch_tune")
        out = {"cached": False, "warps_per_block": list(rep.warps_per_block), "classes": []}
        for c in range(rep.n_classes):
            out["classes"].append({"d": rep.class_d[c], "window": rep.class_window[c],
                                   "lane_vec": rep.class_lane_vec[c], "lane_nv": rep.class_lane_nv[c],
                                   "stages": rep.class_stages[c], "prefetch": rep.class_prefetch[c],
                                   "tuned_wps": rep.tuned_wps[c],
                                   "default_wps": rep.default_wps[c]})
        if cache:
            for j, k in enumerate(keys):
                store[k] = list(self.shape(j))
            for f, k in enumerate(launch_keys):
                store[k] = list(self.launch(f))
            with open(cache, "w") as f:
                json.dump(store, f, indent=1, sort_keys=True)
        return out

    def _device_key(self) -> str:
        return f"dev{self.config.device}:p{self.config.precision}"

    def _class_key(self, c: Config) -> str:
        pitch = (c.layer_size + 7) // 8 * 8
        cls = 64 if pitch <= 64 else 128 if pitch <= 128 else 256 if pitch <= 256 else 384
        return f"{self._device_key()}:d{cls}:w{c.window}:k{c.negative}"

    def train(self) -> BatchStats:
        """Every job's remaining epochs."""
        st = BatchStats()
        self._check(lib().fw2v_batch_train(self._h, C.byref(st)), "batch_train")
        return st

    def train_epochs(self, n: int) -> BatchStats:
        """The next n epochs of every job that has epochs left."""
        st = BatchStats()
        self._check(lib().fw2v_batch_train_epochs(self._h, n, C.byref(st)), "batch_train_epochs")
        return st

    def job_words(self, job: int) -> tuple[int, int]:
        r, k = C.c_uint64(), C.c_uint64()
        self._check(lib().fw2v_batch_job_words(self._h, job, C.byref(r), C.byref(k)), "batch_job_words")
        return r.value, k.value

    def syn0(self, job: int) -> np.ndarray:
        cfg, V = self.jobs[job]
        out = np.zeros((V, cfg.layer_size), np.float32)
        self._check(lib().fw2v_batch_get_syn0(self._h, job, _p(out), cfg.layer_size), "batch_get_syn0")
        return out

    def syn1neg(self, job: int) -> np.ndarray:
        cfg, V = self.jobs[job]
        out = np.zeros((V, cfg.layer_size), np.float32)
        self._check(lib().fw2v_batch_get_syn1neg(self._h, job, _p(out), cfg.layer_size), "batch_get_syn1neg")
        return out
