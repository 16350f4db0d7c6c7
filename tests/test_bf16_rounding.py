"""The bfloat16 write-back rule on the CPU (oracle): the increment from the
loaded value to the stochastic rounding of the new value, added with
round-to-nearest, gives exactly that stochastic rounding when nobody else wrote
the row; one training step stays within the stated bound of the FP64 step.
The GPU tests check that the kernel applies the same rule bit for bit."""
import numpy as np
import pytest

from golden_cases import load
from oracle import oracle as O


def bf16(x):
    return int(O.bf16_bits(np.array([x], np.float32))[0])


def f(h):
    return float(O.bf16_float(np.array([h], np.uint16))[0])


def all_outcomes(stored, a, b):
    return np.array([O.bf16_writeback1(stored, a, b, r) for r in range(65536)], np.uint16)


def next_up(h):
    """The bfloat16 bits of the next value towards +infinity."""
    return h + 1 if h < 0x8000 else (h - 1 if h != 0x8000 else 1)


@pytest.mark.parametrize("x,frac", [(1.0, 0.25), (-0.0371, 0.5), (3.5e-3, 0.9), (1.0, 0.0), (1.0, 0.1),
                                    (-2.0, 0.999), (-1.0, 0.3), (0.25, 0.49), (-0.125, 0.0)])
def test_small_changes_round_to_a_neighbour_without_bias(x, frac):
    h = bf16(x)
    lo, up = f(h), f(next_up(h))
    a = np.float32(lo + frac * (up - lo))
    assert lo <= a <= up
    vals = O.bf16_float(all_outcomes(h, float(a), lo)).astype(np.float64)
    assert set(np.unique(vals)) <= {lo, up}
    if frac == 0.0:
        assert (vals == lo).all()
    # over all 2^16 random draws the mean is the new value itself
    assert vals.mean() == float(a)


def test_no_stagnation_for_updates_far_below_an_ulp():
    """Round-to-nearest would drop these updates every time."""
    h = bf16(0.5)
    ulp = f(h + 1) - f(h)
    a = np.float32(f(h) + ulp / 1000)
    outs = all_outcomes(h, float(a), f(h))
    assert 0 < (outs != h).sum() < 200


@pytest.mark.parametrize("x,dx", [(1e-3, 0.05), (0.0, 0.02), (-0.01, 0.3)])
def test_large_changes_stay_within_two_ulps(x, dx):
    h = bf16(x)
    a = np.float32(f(h) + dx)
    outs = O.bf16_float(all_outcomes(h, float(a), f(h))).astype(np.float64)
    ulp = 2.0 ** (np.floor(np.log2(abs(float(a)))) - 7)
    assert np.abs(outs - float(a)).max() <= 2 * ulp


def test_other_writers_updates_are_kept():
    """The increment lands on whatever is stored: another writer's change
    between this writer's load and its write-back survives."""
    b = f(bf16(0.75))
    other = f(bf16(0.75 + 0.125))  # stored value after another writer's update
    a = np.float32(b + 0.0625)
    outs = O.bf16_float(all_outcomes(bf16(other), float(a), b)).astype(np.float64)
    assert np.allclose(outs, other + 0.0625, atol=2 * 2.0 ** -8)


def test_oracle_bf16_step_within_stated_bound_of_fp64():
    """One sentence at a time from a common start, bfloat16 tables (the kernel's
    rule) against FP64: per row, at most 2 ulps of the row's largest magnitude
    per write-back of the row."""
    g = load("zipf_t1")
    c = dict(g["cfg"])
    corpus = O.corpus_from_text(g["text"], min_count=c["min_count"], msl=c["msl"], cache_eos=c["cache_eos"])
    out = O.sample_streams(corpus, threads=c["threads"], msl=c["msl"], negative=c["negative"], epochs=1,
                           alpha0=c["alpha"], sample=c["sample"])
    lens = np.concatenate([o[0].lens for o in out])
    alphas = np.concatenate([o[0].alphas for o in out])
    ids = np.concatenate([o[0].ids for o in out])
    negs = np.concatenate([o[0].negs for o in out])
    starts = np.concatenate([[0], np.cumsum(lens[:-1])]).astype(np.int64)
    K, W, d, V = c["negative"], c["window"], 64, len(corpus.counts)
    rng = np.random.default_rng(3)
    s0 = O.bf16_bits(O.init_syn0(V, d, d))
    s1 = O.bf16_bits((rng.standard_normal((V, d)) * 0.05).astype(np.float32))
    worst, typical = 0.0, []
    for s in [i for i in range(len(lens)) if lens[i] > 1][:6]:
        sl = slice(starts[s], starts[s] + lens[s])
        sid, sneg = ids[sl], negs[starts[s] * K:(starts[s] + lens[s]) * K]
        a0, a1 = O.bf16_float(s0), O.bf16_float(s1)
        O.train_bf16(s0, s1, [lens[s]], [alphas[s]], sid, sneg, d=d, window=W, negative=K,
                     seed=O.mix64(0x5EEDF00D + s), sigmoid="exact", vec=2, nv=1)
        r0, r1 = a0.astype(np.float64), a1.astype(np.float64)
        O.train(r0, r1, [lens[s]], [alphas[s]], sid, sneg, d=d, window=W, negative=K, sigmoid="exact", precision=64)
        n0 = np.bincount(sid, minlength=V)
        n1 = np.bincount(np.concatenate([sid[:, None], sneg.reshape(-1, K)], 1).ravel(), minlength=V)
        for got, ref, start, n in ((O.bf16_float(s0), r0, a0, n0), (O.bf16_float(s1), r1, a1, n1)):
            err = np.abs(got.astype(np.float64) - ref).max(1)
            scale = np.maximum(np.abs(start).max(1), np.abs(ref).max(1)) * 2.0 ** -7
            assert (err[n == 0] == 0).all()
            ratio = err[n > 0] / (2.0 * n[n > 0] * scale[n > 0])
            worst = max(worst, float(ratio.max()))
            typical.append(float(np.median(ratio)))
    assert 0 < worst <= 1.0, worst
    assert np.median(typical) < 0.5
