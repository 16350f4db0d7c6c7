"""Host logic of the quality evaluators (CPU only): how a held-out stream is
cut into sentences before its pairs are sampled."""
import numpy as np

from fw2v import evaluate


def test_sentence_chunks_cut_at_eos_and_msl():
    # two sentences ended by 0, then a tail without one
    s = np.array([5, 6, 7, 0, 8, 0, 9, 10, 11, 12, 13], np.int32)
    assert list(evaluate.sentence_chunks(s, 1000)) == [0, 4, 6]
    # pieces of at most msl tokens inside every sentence
    assert list(evaluate.sentence_chunks(s, 2)) == [0, 2, 4, 6, 8, 10]


def test_sentence_chunks_of_a_stream_without_eos():
    s = np.arange(1, 11, dtype=np.int32)
    assert list(evaluate.sentence_chunks(s, 4)) == [0, 4, 8]


def test_sentence_chunks_of_an_empty_stream():
    assert list(evaluate.sentence_chunks(np.zeros(0, np.int32), 4)) == [0]
