"""fw2v_kernel_batch_noalloc: the kernel seam for callers that cannot allocate
device memory (programs whose device memory belongs to a framework's pool
allocator, where a direct cudaMalloc bypasses the pool and can fail; plugin
hosts with a fixed memory budget).  It must give the same tables as
fw2v_kernel_batch, call after call, and refuse requests whose per-warp scratch
would not fit its fixed buffer.

This file is named to be collected last: a failure here leaves every other
test already run.
"""
import numpy as np
import pytest

import fw2v

V, D, W, K, MSL, PITCH = 96, 128, 3, 4, 24, 128


def _batch(rng, n):
    lens = rng.integers(1, MSL + 1, n).astype(np.int32)
    sen = rng.integers(1, V, (n, MSL)).astype(np.int32)
    neg = rng.integers(1, V, (n, MSL, K)).astype(np.int32)
    alpha = np.full(n, 0.025, np.float32)
    return lens, sen, neg, alpha


@pytest.mark.gpu
def test_noalloc_matches_seam_on_consecutive_calls():
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(21)
    syn0 = torch.from_numpy((rng.standard_normal((V, PITCH)) * 0.05).astype(np.float32)).to(dev)
    syn1 = torch.from_numpy((rng.standard_normal((V, PITCH)) * 0.05).astype(np.float32)).to(dev)
    # the same starting tables for both entry points
    a0, a1 = syn0.clone(), syn1.clone()
    b0, b1 = syn0.clone(), syn1.clone()
    L = fw2v.lib()
    for call in range(2):
        lens, sen, neg, alpha = (torch.from_numpy(x).to(dev) for x in _batch(rng, 5))
        # one sentence per launch, so that both entry points apply the updates
        # in the same order and the comparison can be exact
        for b in range(5):
            args = (sen[b].data_ptr(), neg[b].data_ptr(), lens[b:].data_ptr(), alpha[b:].data_ptr(),
                    1, D, W, K, MSL, PITCH, V, None)
            assert L.fw2v_kernel_batch(a0.data_ptr(), a1.data_ptr(), *args) == 0
            assert L.fw2v_kernel_batch_noalloc(b0.data_ptr(), b1.data_ptr(), *args) == 0
        assert L.fw2v_kernel_batch_error(None) == 0
        torch.cuda.synchronize()
        assert torch.equal(a0, b0), f"syn0 differs after call {call + 1}"
        assert torch.equal(a1, b1), f"syn1neg differs after call {call + 1}"
        assert not torch.equal(a1, syn1)  # the calls did train


def test_noalloc_rejects_scratch_beyond_its_buffer():
    # A row pitch so large that one block's scratch exceeds the fixed buffer is
    # refused before any device access (the pointers are never dereferenced).
    per_block = 4 * (2 * W + 1) * 4
    pitch = (fw2v.NOALLOC_SCRATCH_BYTES // per_block + 4) // 4 * 4
    dummy = 256
    st = fw2v.lib().fw2v_kernel_batch_noalloc(dummy, dummy, dummy, dummy, dummy, dummy, 1, D, W, K,
                                              MSL, pitch, V, None)
    assert st == 7


@pytest.mark.gpu
def test_noalloc_many_sentences_per_call_capped_grid():
    """Many sentences in one call on wide rows with the longest window
    (d = pitch = 1024, W = 15): the fixed buffer then holds 132 warps' scratch,
    fewer than the SMs, so the launch caps its grid and every warp works at its
    own offset in the buffer.  Each sentence draws its ids and negatives from
    its own range of rows, so the result does not depend on which warp trains
    which sentence or when, and must equal the seam's and the oracle's."""
    import torch

    from oracle import oracle as O

    d = pitch = 1024
    w, k, msl, n, rows = 15, 5, 24, 200, 40
    assert (fw2v.NOALLOC_SCRATCH_BYTES // 4) // ((2 * w + 1) * pitch) < 148
    vocab = 1 + n * rows
    rng = np.random.default_rng(33)
    lens = rng.integers(1, msl + 1, n).astype(np.int32)
    base = (1 + np.arange(n) * rows)[:, None]
    sen = (base + rng.integers(0, rows, (n, msl))).astype(np.int32)
    neg = (base[:, :, None] + rng.integers(0, rows, (n, msl, k))).astype(np.int32)
    alpha = np.full(n, 0.025, np.float32)
    syn0 = (rng.standard_normal((vocab, pitch)) * 0.05).astype(np.float32)
    syn1 = (rng.standard_normal((vocab, pitch)) * 0.05).astype(np.float32)
    dev = torch.device("cuda:0")
    tsen, tneg = torch.from_numpy(sen).to(dev), torch.from_numpy(neg).to(dev)
    tlen, talpha = torch.from_numpy(lens).to(dev), torch.from_numpy(alpha).to(dev)
    a0, a1 = torch.from_numpy(syn0).to(dev), torch.from_numpy(syn1).to(dev)
    b0, b1 = a0.clone(), a1.clone()
    L = fw2v.lib()
    args = (tsen.data_ptr(), tneg.data_ptr(), tlen.data_ptr(), talpha.data_ptr(), n, d, w, k, msl, pitch,
            vocab, None)
    for _ in range(2):  # two calls in a row: the buffer keeps the first call's contents
        assert L.fw2v_kernel_batch(a0.data_ptr(), a1.data_ptr(), *args) == 0
        assert L.fw2v_kernel_batch_noalloc(b0.data_ptr(), b1.data_ptr(), *args) == 0
    assert L.fw2v_kernel_batch_error(None) == 0
    torch.cuda.synchronize()
    assert torch.equal(a0, b0) and torch.equal(a1, b1)
    flat_ids = np.concatenate([sen[b, :lens[b]] for b in range(n)])
    flat_negs = np.concatenate([neg[b, :lens[b]].ravel() for b in range(n)])
    for _ in range(2):
        O.train(syn0, syn1, lens, alpha, flat_ids, flat_negs, d=d, window=w, negative=k, sigmoid="table",
                precision=32, vec=4, nv=8)
    np.testing.assert_array_equal(b0.cpu().numpy(), syn0)
    np.testing.assert_array_equal(b1.cpu().numpy(), syn1)


@pytest.mark.gpu
def test_noalloc_rejects_shared_memory_beyond_a_block():
    """One warp needs its ring and staged rows in shared memory: about
    (2W+12)*pitch*4 bytes.  A pitch far beyond the layer size makes that too
    large for a block, which is refused with FW2V_ERR_ARGUMENT before any
    device access (the pointers are never dereferenced)."""
    dummy = 256
    st = fw2v.lib().fw2v_kernel_batch_noalloc(dummy, dummy, dummy, dummy, dummy, dummy, 1, 16, 1, 0,
                                              MSL, 16384, V, None)
    assert st == 1
