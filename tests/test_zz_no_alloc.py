"""fw2v_kernel_batch_noalloc: the kernel seam for callers that cannot allocate
device memory (code recording a CUDA graph, where cudaMalloc/cudaFree are not
allowed; programs whose device memory belongs to a framework's pool allocator).
It must give the same tables as fw2v_kernel_batch, call after call, and refuse
requests whose per-warp scratch would not fit its fixed buffer.

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
