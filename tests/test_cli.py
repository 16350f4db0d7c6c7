"""The full-w2v command line against the reference program's own outputs.

CPU (preprocessing only, no -output, as the reference allows): the vocabulary
file, the corpus cache, the interpreted corpus, and the cache round trip
(-read-vocab + -read-corpus-cache + -save-corpus-cache) are byte-identical to
the reference's.  GPU: the untrained export (-iter 0) is byte-identical to the
reference's .vec, a deterministic epoch equals the FP32 oracle bit for bit, and
the word count line equals the reference's.
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import fw2v
from golden_cases import CASES, load
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "full-w2v_b200", "full-w2v")


def _flags(g, drop=()):
    toks = str(g["flags"]).split()
    out, i = [], 0
    while i < len(toks):
        t = toks[i]
        if t == "-cache-eos":
            out.append(t)
            i += 1
            continue
        if t not in drop:
            out += [t, toks[i + 1]]
        i += 2
    return out


def _run(args, cwd):
    r = subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(CLI):
        pytest.skip("full-w2v is not built")


@pytest.mark.parametrize("read_threads", [1, 3, 16])
@pytest.mark.parametrize("name", CASES)
def test_preprocessing_files_match_reference(name, read_threads, tmp_path):
    """Serial and parallel text readers (the file cut into 3 or 16 segments at
    line starts) give the reference's vocabulary, cache and corpus files."""
    g = load(name)
    (tmp_path / "corpus.txt").write_bytes(g["text"])
    _run(["-train", "corpus.txt", "-debug", "0", "-save-vocab", "v.txt", "-save-corpus-cache", "c.txt",
          "-save-corpus", "s.txt", "-read-threads", str(read_threads)] + _flags(g), tmp_path)
    assert (tmp_path / "v.txt").read_bytes() == g["vocab_text"]
    assert (tmp_path / "c.txt").read_bytes() == g["cache_text"]
    assert _sha(tmp_path / "s.txt") == str(g["corpus_text_sha256"])


@pytest.mark.parametrize("name", CASES)
def test_cache_round_trip_matches_reference(name, tmp_path):
    g = load(name)
    (tmp_path / "v.txt").write_bytes(g["vocab_text"])
    (tmp_path / "c.txt").write_bytes(g["cache_text"])
    _run(["-read-vocab", "v.txt", "-read-corpus-cache", "c.txt", "-debug", "0",
          "-save-corpus-cache", "re.txt"] + _flags(g), tmp_path)
    assert _sha(tmp_path / "re.txt") == str(g["recache_sha256"])


def test_help_and_missing_input(tmp_path):
    assert "-train" in _run([], tmp_path)
    r = subprocess.run([CLI, "-output", "x.vec", "-debug", "0"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "No vocabulary or training file" in r.stdout


def _read_vec(path, binary=True):
    raw = open(path, "rb").read()
    hdr, rest = raw.split(b"\n", 1)
    V, d = (int(x) for x in hdr.split())
    words, rows, p = [], [], 0
    for _ in range(V):
        sp = rest.index(b" ", p)
        words.append(rest[p:sp])
        p = sp + 1
        if binary:
            rows.append(np.frombuffer(rest[p:p + 4 * d], np.float32))
            p += 4 * d + 1
        else:
            nl = rest.index(b"\n", p)
            rows.append(np.array(rest[p:nl].split(), np.float32))
            p = nl + 1
    return words, np.stack(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_untrained_export_matches_reference_bytes(name, tmp_path):
    g = load(name)
    (tmp_path / "corpus.txt").write_bytes(g["text"])
    out = _run(["-train", "corpus.txt", "-output", "o.vec", "-binary", "1", "-debug", "0"]
               + _flags(g, drop=("-iter",)) + ["-iter", "0"], tmp_path)
    assert "Overall Words: 0" in out
    assert _sha(tmp_path / "o.vec") == str(g["vec_file_sha256"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["zipf_t1", "eos_t1", "zipf_t3"])
def test_deterministic_training_export_matches_oracle(name, tmp_path):
    g = load(name)
    c = g["cfg"]
    (tmp_path / "corpus.txt").write_bytes(g["text"])
    out = _run(["-train", "corpus.txt", "-output", "o.vec", "-binary", "1", "-debug", "0",
                "-deterministic", "1"] + _flags(g), tmp_path)
    assert f"Overall Words: {int(g['overall_words'])}" in out
    words, vec = _read_vec(tmp_path / "o.vec")
    corpus = O.corpus_from_text(g["text"], min_count=c["min_count"], msl=c["msl"],
                                cache_eos=c["cache_eos"])
    assert words == corpus.words
    d = c["size"]
    vec_, nv, pitch = fw2v.lane_layout(d)
    syn0 = O.init_syn0(len(corpus.counts), d, d)
    syn1 = np.zeros_like(syn0)
    out = O.sample_streams(corpus, threads=c["threads"], msl=c["msl"], negative=c["negative"],
                           epochs=c["iter"], alpha0=c["alpha"], sample=c["sample"])
    for e in range(c["iter"]):
        lens = np.concatenate([out[s][e].lens for s in range(len(out))])
        alphas = np.concatenate([out[s][e].alphas for s in range(len(out))])
        ids = np.concatenate([out[s][e].ids for s in range(len(out))])
        negs = np.concatenate([out[s][e].negs for s in range(len(out))])
        O.train(syn0, syn1, lens, alphas, ids, negs, d=d, window=c["window"], negative=c["negative"],
                sigmoid="table", precision=32, vec=vec_, nv=nv)
    np.testing.assert_array_equal(vec, syn0)


@pytest.mark.gpu
def test_text_export_and_shuffles(tmp_path):
    g = load("eos_t1")
    (tmp_path / "corpus.txt").write_bytes(g["text"])
    args = ["-train", "corpus.txt", "-debug", "0"] + _flags(g)
    _run(args + ["-output", "b.vec", "-binary", "1", "-deterministic", "1"], tmp_path)
    _run(args + ["-output", "t.vec", "-binary", "0", "-deterministic", "1"], tmp_path)
    wb, vb = _read_vec(tmp_path / "b.vec")
    wt, vt = _read_vec(tmp_path / "t.vec", binary=False)
    assert wb == wt
    # "%f" prints 6 decimals
    np.testing.assert_allclose(vt, vb, atol=5.1e-7, rtol=0)
    for extra in (["-pre-shuffle"], ["-epoch-shuffle"]):
        out = _run(args + ["-output", "s.vec", "-binary", "1"] + extra, tmp_path)
        assert f"Overall Words: {int(g['overall_words'])}" in out
        _, vs = _read_vec(tmp_path / "s.vec")
        assert np.isfinite(vs).all()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_jobs_manifest_trains_each_job_as_alone(tmp_path, precision):
    """-jobs: the jobs of a manifest train together in one batch; with
    -deterministic 1 each exports the vectors it gets alone (same seed)."""
    lines = []
    for i, (name, seed) in enumerate((("zipf_t1", 0), ("messy_t1", 9))):
        g = load(name)
        (tmp_path / f"c{i}.txt").write_bytes(g["text"])
        common = ["-train", f"c{i}.txt", "-binary", "1", "-seed", str(seed), "-size", str(16 + 24 * i),
                  "-negative", "5"] + _flags(g, drop=("-negative", "-size"))
        lines.append(" ".join(common + ["-output", f"j{i}.vec"]))
        _run(common + ["-output", f"a{i}.vec", "-debug", "0", "-deterministic", "1", "-precision", precision],
             tmp_path)
    (tmp_path / "jobs.txt").write_text("# two jobs\n" + "\n".join(lines) + "\n")
    out = _run(["-jobs", "jobs.txt", "-deterministic", "1", "-precision", precision], tmp_path)
    assert "Job 2 Words:" in out and "Overall Words Per Second:" in out
    for i in range(2):
        assert (tmp_path / f"j{i}.vec").read_bytes() == (tmp_path / f"a{i}.vec").read_bytes()


@pytest.mark.parametrize("name", ["c1_t16", "c2cut_t64"])
def test_parallel_reader_vocab_matches_reference_at_shape(name, tmp_path):
    """The benchmark-shaped corpora (1M and 2M tokens) read by 8 threads: the
    vocabulary file equals the reference program's (digest in
    tests/golden/shape_<name>.json)."""
    import shape_cases as S
    from fw2v import synth
    raw, ends, _ = S.raw_tokens(name)
    (tmp_path / "corpus.txt").write_bytes(synth.text_of(raw, ends))
    f = S.flags_of(name)
    _run(["-train", "corpus.txt", "-debug", "0", "-save-vocab", "v.txt", "-read-threads", "8",
          "-min-count", str(f["min_count"]), "-msl", str(f["msl"])], tmp_path)
    assert _sha(tmp_path / "v.txt") == S.load(name)["vocab_sha256"]
