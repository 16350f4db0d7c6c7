"""fw2v_neighbours (the precision@10 evaluator's kernel) against a float64
numpy search on small tables: the same k nearest candidates by cosine (apart
from near-ties, where FP32 rounding may swap neighbours) and cosines within
1e-5; BF16 tables read as the values their bits hold."""
import numpy as np
import pytest

import fw2v
from fw2v import evaluate
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def reference(table, cand, queries, k):
    E = table[cand].astype(np.float64)
    n = np.linalg.norm(E, axis=1)
    n[n == 0] = 1.0
    S = (E[queries] @ E.T) / n[queries][:, None] / n[None, :]
    S[np.arange(len(queries)), queries] = -np.inf
    order = np.lexsort((np.broadcast_to(np.arange(len(cand)), S.shape), -S), axis=1)[:, :k]
    return order, np.take_along_axis(S, order, 1)


@pytest.mark.parametrize("d,n_rows,n_cand,n_q,k", [(64, 3000, 2500, 700, 10), (300, 5000, 4000, 37, 10),
                                                   (128, 1200, 1100, 1100, 32), (500, 900, 800, 9, 5)])
def test_neighbours_match_float64_search(d, n_rows, n_cand, n_q, k):
    rng = np.random.default_rng(d + n_q)
    # clustered rows, so that neighbours are well separated from the rest
    centres = rng.standard_normal((40, d))
    table = (centres[rng.integers(0, 40, n_rows)] + 0.4 * rng.standard_normal((n_rows, d))).astype(np.float32)
    cand = np.sort(rng.choice(n_rows, n_cand, replace=False)).astype(np.int32)
    queries = rng.choice(n_cand, n_q, replace=False).astype(np.int32)
    got_i, got_s = evaluate.neighbours(table, cand, queries, k)
    want_i, want_s = reference(table, cand, queries, k)
    np.testing.assert_allclose(got_s, want_s, atol=1e-5, rtol=0)
    assert (got_i != queries[:, None]).all()
    # the same neighbours wherever the k-th and (k+1)-th cosines are apart
    same = (got_i == want_i).all(1)
    assert same.mean() > 0.98, same.mean()


def test_neighbours_bf16_table():
    rng = np.random.default_rng(5)
    d, n = 96, 1500
    f32 = rng.standard_normal((n, d)).astype(np.float32)
    bits = O.bf16_bits(f32)
    cand = np.arange(n, dtype=np.int32)
    queries = np.arange(0, n, 7, dtype=np.int32)
    got_i, got_s = evaluate.neighbours(bits, cand, queries, 10, precision=fw2v.BF16)
    want_i, want_s = reference(O.bf16_float(bits), cand, queries, 10)
    np.testing.assert_allclose(got_s, want_s, atol=1e-5, rtol=0)
    assert (got_i == want_i).all(1).mean() > 0.98


def test_precision_at_10_uses_all_labelled_words():
    rng = np.random.default_rng(9)
    V, d = 2000, 32
    label = rng.integers(0, 5, V).astype(np.int32)
    label[0] = -1
    centres = rng.standard_normal((5, d)) * 3
    syn0 = (centres[np.maximum(label, 0)] + rng.standard_normal((V, d))).astype(np.float32)
    counts = np.full(V, 10, np.uint32)
    p_all, n = evaluate.precision_at_10(syn0, label, counts, queries=0)
    assert n == V - 1 and p_all > 0.9
    p_some, _ = evaluate.precision_at_10(syn0, label, counts, queries=300)
    assert abs(p_some - p_all) < 0.05
