"""Host-side checks of libfw2v.so that need no GPU: the library loads, exports
every entry point include/fw2v.h declares, and its host helpers agree with the
oracle (sigmoid table, unigram table boundaries, row layout)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import fw2v
from golden_cases import CASES, load
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "fw2v.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fw2v_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = fw2v.lib()
    declared = header_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(fw2v.EXPORTS) == declared


def test_version_string():
    assert b"sm_100a" in fw2v.lib().fw2v_version()


def test_create_without_device_fails_cleanly():
    # On a machine without a B200 the handle is refused with a status, not a crash.
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(fw2v.Fw2vError) as e:
        fw2v.Trainer(fw2v.default_config())
    assert e.value.status == 6


def test_batch_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(fw2v.Fw2vError) as e:
        fw2v.Batch()
    assert e.value.status == 6
    cfg = fw2v.BatchConfig()
    fw2v.lib().fw2v_batch_config_default(C.byref(cfg))
    assert (cfg.precision, cfg.use_graph, cfg.deterministic, cfg.round_tokens, cfg.group_bytes) == (fw2v.FP32, 1, 0, 0, 0)
    bad = fw2v.BatchConfig(precision=7)
    assert fw2v.lib().fw2v_batch_create(C.byref(bad), C.byref(C.c_void_p())) == 1


def test_default_config_seed_is_the_references():
    assert fw2v.default_config().seed == 0


def test_invalid_config_rejected_before_device_use():
    c = fw2v.default_config(window=16)
    h = C.c_void_p()
    assert fw2v.lib().fw2v_create(C.byref(c), C.byref(h)) in (1, 6)


def test_exp_table_matches_oracle():
    np.testing.assert_array_equal(fw2v.exp_table(), O.exp_table())


def _firsts_from_runs(starts, words, V, size):
    firsts = np.full(V - 1, size, np.int64)
    for s, w in zip(starts[:-1], words):
        firsts[w - 1] = s
    return firsts


@pytest.mark.parametrize("name", ["zipf_t1", "zipf_t3", "messy_t1"])
def test_unigram_firsts_match_literal_fill_golden_vocab(name):
    counts = load(name)["vocab_counts"]
    size = O.UNIGRAM_TABLE_SIZE
    starts, words = O.unigram_runs(counts, size)
    np.testing.assert_array_equal(fw2v.unigram_firsts(counts, size),
                                  _firsts_from_runs(starts, words, len(counts), size))


@pytest.mark.parametrize("seed", [0, 1])
def test_unigram_firsts_with_lagging_fill(seed):
    # Tiny table: many words have shares below one entry, so the fill lags
    # behind the running share and every word still gets one entry.
    rng = np.random.default_rng(seed)
    counts = np.concatenate([[rng.integers(0, 50)], rng.integers(1, 1000, 3000)]).astype(np.uint32)
    for size in (1000, 5000, 100_003):
        starts, words = O.unigram_runs(counts, size)
        np.testing.assert_array_equal(fw2v.unigram_firsts(counts, size),
                                      _firsts_from_runs(starts, words, len(counts), size))


def test_lane_layout():
    assert fw2v.lane_layout(8) == (2, 1, 8)
    assert fw2v.lane_layout(64) == (2, 1, 64)
    assert fw2v.lane_layout(100) == (4, 1, 104)
    assert fw2v.lane_layout(128) == (4, 1, 128)
    assert fw2v.lane_layout(300) == (4, 3, 304)
    assert fw2v.lane_layout(1000) == (4, 8, 1000)
