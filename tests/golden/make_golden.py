"""Generate the golden fixtures in this directory from the reference's own code.

Run from the repository root in a container that has the reference checkout:

    make -C oracle ref          # builds oracle/_ref/fw2v_ref_host from the reference sources
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --shape    # only the benchmark-shaped digests

``oracle/_ref/fw2v_ref_host`` is FULL-W2V-driver.cu (with the two .cpp files it
includes) compiled unmodified and linked against a host-memory CUDA-runtime
stand-in (oracle/ref_shim/cudart_shim.cpp).  Its training kernel is a no-op
that records every batch the reference's host loop ships to the GPU: sentence
lengths, learning rates, kept token ids and the K negatives per kept token.
Together with the reference's vocabulary file (-save-vocab), its exported
initial vectors (-binary 1, untrained because the kernel is a no-op) and its
"Overall Words" count, these pin the oracle and the CUDA sampler bit for bit.

Each fixture stores the synthetic corpus it was made from (seeded generator,
written here), the command-line flags, and the reference's outputs.  The
benchmark-shaped cases of tests/shape_cases.py (corpora of 1M to 12.5M tokens,
up to 3125 sampling threads) store digests of the same outputs instead, in
shape_<name>.json.
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "fw2v_ref_host")
OUT = os.path.dirname(os.path.abspath(__file__))
MAGIC = 0x57325644


def zipf_text(seed: int, n_tokens: int, vocab: int, s: float = 1.0, line_lo: int = 3,
              line_hi: int = 120) -> bytes:
    rng = np.random.default_rng(seed)
    p = 1.0 / np.arange(1, vocab + 1) ** s
    p /= p.sum()
    toks = rng.choice(vocab, size=n_tokens, p=p)
    lines, i = [], 0
    while i < n_tokens:
        n = int(rng.integers(line_lo, line_hi))
        lines.append(" ".join(f"w{t}" for t in toks[i:i + n]))
        i += n
    return ("\n".join(lines) + "\n").encode()


def messy_text(seed: int) -> bytes:
    """Exercises the word reader: CR, tabs, runs of blanks, empty lines, an
    over-long word (truncated at 799 bytes) and rare words cut by min-count."""
    rng = np.random.default_rng(seed)
    base = zipf_text(seed, 14000, 600, 1.1).decode().split("\n")
    out = []
    for k, line in enumerate(base):
        toks = line.split(" ")
        if k % 7 == 3:
            toks.insert(len(toks) // 2, "rare%d" % k)
        sep = ["\t", "  ", " \t ", " "][k % 4]
        line = sep.join(toks)
        if k % 5 == 1:
            line += "\r"
        if k % 11 == 4:
            out.append("")
        if k == 40:
            line += " " + "x" * 1000 + " tail"
        out.append(line)
    del rng
    return ("\n".join(out) + "\n").encode()


def parse_dump(path: str):
    b = np.fromfile(path, dtype=np.int32)
    i, entries = 0, []
    K = msl = None
    while i < len(b):
        assert b[i] == MAGIC, "corrupt dump"
        fresh, K, msl = (int(x) for x in b[i + 1:i + 4])
        i += 4
        for _ in range(fresh):
            L = int(b[i])
            a = b[i + 1:i + 2].view(np.float32)[0]
            i += 2
            ids = b[i:i + L].copy()
            i += L
            negs = b[i:i + L * K].copy()
            i += L * K
            entries.append((L, a, ids, negs))
    # The last entry of a thread's final launch is the extra zero-length block
    # the reference appends after its epoch loop (FULL-W2V-driver.cu:305-308).
    assert entries and entries[-1][0] == 0
    entries = entries[:-1]
    lens = np.array([e[0] for e in entries], np.int32)
    alphas = np.array([e[1] for e in entries], np.float32)
    ids = np.concatenate([e[2] for e in entries]) if entries else np.zeros(0, np.int32)
    negs = np.concatenate([e[3] for e in entries]) if entries else np.zeros(0, np.int32)
    return lens, alphas, ids.astype(np.int32), negs.astype(np.int32)


def run_case(name: str, text: bytes, flags: list[str]):
    tmp = tempfile.mkdtemp(prefix="fw2v_golden_")
    try:
        corpus = os.path.join(tmp, "corpus.txt")
        with open(corpus, "wb") as f:
            f.write(text)
        dump = os.path.join(tmp, "dump")
        os.mkdir(dump)
        vec = os.path.join(tmp, "out.vec")
        vocab = os.path.join(tmp, "out.vocab")
        cmd = [HARNESS, "-train", corpus, "-output", vec, "-save-vocab", vocab, "-debug", "0",
               "-binary", "1", "-streams", "1", "-kernel-batch-size", "4"] + flags
        r = subprocess.run(cmd, env=dict(os.environ, FW2V_REF_DUMP_DIR=dump),
                           capture_output=True, check=True, text=True)
        overall = [ln for ln in r.stdout.splitlines() if ln.startswith("Overall Words:")]
        overall_words = int(overall[0].split(":")[1])
        words, counts = [], []
        for ln in open(vocab, "rb").read().splitlines():
            w, c = ln.rsplit(b" ", 1)
            words.append(w)
            counts.append(int(c))
        raw = open(vec, "rb").read()
        hdr, rest = raw.split(b"\n", 1)
        V, d = (int(x) for x in hdr.split())
        rows, p = [], 0
        for _ in range(V):
            sp = rest.index(b" ", p)
            p = sp + 1
            rows.append(np.frombuffer(rest[p:p + 4 * d], np.float32))
            p += 4 * d + 1
        syn0 = np.stack(rows)
        threads = sorted(f for f in os.listdir(dump) if f.endswith(".bin"))
        per = [parse_dump(os.path.join(dump, f)) for f in threads]
        # The reference's corpus cache and interpreted corpus for the same flags
        # (preprocessing only: no -output).
        cache = os.path.join(tmp, "out.cache")
        interp = os.path.join(tmp, "out.corpus")
        pre = [HARNESS, "-train", corpus, "-debug", "0", "-save-corpus-cache", cache,
               "-save-corpus", interp] + [f for f in flags if f not in ("-output",)]
        subprocess.run(pre, capture_output=True, check=True, text=True)
        cache_bytes = open(cache, "rb").read()
        arrays = {
            "corpus": np.frombuffer(text, np.uint8),
            "corpus_cache": np.frombuffer(cache_bytes, np.uint8),
            "corpus_text_sha256": np.array(hashlib.sha256(open(interp, "rb").read()).hexdigest()),
            "flags": np.array(" ".join(flags)),
            "vocab_words": np.array([w.decode("latin-1") for w in words]),
            "vocab_counts": np.array(counts, np.uint32),
            "overall_words": np.array(overall_words, np.int64),
            "vec_file_sha256": np.array(hashlib.sha256(raw).hexdigest()),
            "syn0_init_sha256": np.array(hashlib.sha256(syn0.tobytes()).hexdigest()),
            "syn0_init_head": syn0[:8].copy(),
            "n_threads": np.array(len(per), np.int32),
        }
        for t, (lens, alphas, ids, negs) in enumerate(per):
            arrays[f"t{t}_lens"] = lens
            arrays[f"t{t}_alphas"] = alphas
            # vocabularies here are < 32768 words: int16 halves the fixture size
            assert V < 32768
            arrays[f"t{t}_ids"] = ids.astype(np.int16)
            arrays[f"t{t}_negs"] = negs.astype(np.int16)
        # The same run fed from the reference's own vocabulary and corpus cache
        # files (ReadVocab + readCorpusCache, improved_driver_functions.cpp:167-196,
        # 320-401): its batches, and the cache it writes back out.
        dump2 = os.path.join(tmp, "dump_cache")
        os.mkdir(dump2)
        recache = os.path.join(tmp, "re.cache")
        cmd2 = [HARNESS, "-read-vocab", vocab, "-read-corpus-cache", cache, "-output", vec, "-debug", "0",
                "-binary", "1", "-streams", "1", "-kernel-batch-size", "4",
                "-save-corpus-cache", recache] + flags
        r2 = subprocess.run(cmd2, env=dict(os.environ, FW2V_REF_DUMP_DIR=dump2), capture_output=True,
                            check=True, text=True)
        ow2 = [ln for ln in r2.stdout.splitlines() if ln.startswith("Overall Words:")]
        arrays["cache_overall_words"] = np.array(int(ow2[0].split(":")[1]), np.int64)
        arrays["recache_sha256"] = np.array(hashlib.sha256(open(recache, "rb").read()).hexdigest())
        per2 = [parse_dump(os.path.join(dump2, f)) for f in sorted(os.listdir(dump2))]
        for t, (lens, alphas, ids, negs) in enumerate(per2):
            arrays[f"c{t}_lens"] = lens
            arrays[f"c{t}_alphas"] = alphas
            arrays[f"c{t}_ids"] = ids.astype(np.int16)
            arrays[f"c{t}_negs"] = negs.astype(np.int16)
        arrays["cache_n_threads"] = np.array(len(per2), np.int32)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
        print(f"{name}: V={V} overall_words={overall_words} threads={len(per)} "
              f"entries={[len(x[0]) for x in per]}")
    finally:
        shutil.rmtree(tmp)


CASES = [
    ("zipf_t1", lambda: zipf_text(11, 16000, 2000),
     "-size 8 -window 3 -negative 5 -sample 1e-3 -iter 2 -threads 1 -min-count 2 -msl 50 -alpha 0.05"),
    ("eos_t1", lambda: zipf_text(12, 14000, 1500, 1.05),
     "-size 8 -window 2 -negative 3 -sample 1e-4 -iter 2 -threads 1 -min-count 1 -msl 60 -cache-eos"),
    ("zipf_t3", lambda: zipf_text(13, 12000, 1500),
     "-size 8 -window 5 -negative 4 -sample 1e-3 -iter 2 -threads 3 -min-count 3 -msl 40"),
    ("nosample_t2", lambda: zipf_text(14, 9000, 800),
     "-size 8 -window 2 -negative 2 -sample 0 -iter 1 -threads 2 -min-count 1 -msl 30"),
    ("k0_t1", lambda: zipf_text(15, 12000, 900),
     "-size 8 -window 4 -negative 0 -sample 1e-3 -iter 2 -threads 1 -min-count 1 -msl 25"),
    ("messy_t1", lambda: messy_text(16),
     "-size 8 -window 3 -negative 5 -sample 1e-3 -iter 1 -threads 1 -min-count 3 -msl 45 -cache-eos"),
]


def run_shape_case(name: str):
    """A benchmark-shaped case (tests/shape_cases.py): the reference's batches
    and files reduced to digests, written to shape_<name>.json."""
    sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "full-w2v_b200")]
    import shape_cases as S
    from fw2v import synth

    case = S.CASES[name]
    raw, ends, _ = S.raw_tokens(name)
    text = synth.text_of(raw, ends)
    tmp = tempfile.mkdtemp(prefix="fw2v_golden_")
    try:
        corpus = os.path.join(tmp, "corpus.txt")
        with open(corpus, "wb") as f:
            f.write(text)
        dump = os.path.join(tmp, "dump")
        os.mkdir(dump)
        vec = os.path.join(tmp, "out.vec")
        vocab = os.path.join(tmp, "out.vocab")
        cmd = [HARNESS, "-train", corpus, "-output", vec, "-save-vocab", vocab, "-debug", "0",
               "-binary", "1", "-streams", "1", "-kernel-batch-size", "4"] + case["flags"].split()
        if case.get("no_export"):
            cmd.append("-no-export")
        r = subprocess.run(cmd, env=dict(os.environ, FW2V_REF_DUMP_DIR=dump),
                           capture_output=True, check=True, text=True)
        overall = [ln for ln in r.stdout.splitlines() if ln.startswith("Overall Words:")]
        vocab_bytes = open(vocab, "rb").read()
        per = [parse_dump(os.path.join(dump, f)) for f in sorted(os.listdir(dump))]
        out = {
            "name": name,
            "generator": case["gen"],
            "flags": case["flags"],
            "text_sha256": hashlib.sha256(text).hexdigest(),
            "vocab_sha256": hashlib.sha256(vocab_bytes).hexdigest(),
            "vocab_size": vocab_bytes.count(b"\n"),
            "overall_words": int(overall[0].split(":")[1]),
            "streams": S.digests([(l, a, i, n) for l, a, i, n in per]),
        }
        if not case.get("no_export"):
            raw_vec = open(vec, "rb").read()
            hdr, rest = raw_vec.split(b"\n", 1)
            V, d = (int(x) for x in hdr.split())
            rows, p = [], 0
            for _ in range(V):
                p = rest.index(b" ", p) + 1
                rows.append(np.frombuffer(rest[p:p + 4 * d], np.float32))
                p += 4 * d + 1
            out["syn0_init_sha256"] = hashlib.sha256(np.stack(rows).tobytes()).hexdigest()
        with open(os.path.join(OUT, f"shape_{name}.json"), "w") as f:
            json.dump(out, f, separators=(",", ":"))
        print(f"shape_{name}: V={out['vocab_size']} overall_words={out['overall_words']} "
              f"threads={len(per)} kept={sum(s[3] for s in out['streams'])}")
    finally:
        shutil.rmtree(tmp)


# The reference's shuffles (-pre-shuffle, -epoch-shuffle: libc rand(), unseeded)
SHUFFLE_CASES = [
    ("shuffle_t2", lambda: zipf_text(17, 12000, 1200),
     "-size 8 -window 3 -negative 4 -sample 1e-3 -iter 3 -threads 2 -min-count 2 -msl 40 -pre-shuffle "
     "-epoch-shuffle"),
]


def run_shuffle_case(name: str, text: bytes, flags: list[str]):
    """The batches of a run with both shuffles: the corpus, the flags and each
    thread's batches in full (the case is small)."""
    tmp = tempfile.mkdtemp(prefix="fw2v_golden_")
    try:
        corpus = os.path.join(tmp, "corpus.txt")
        with open(corpus, "wb") as f:
            f.write(text)
        dump = os.path.join(tmp, "dump")
        os.mkdir(dump)
        cmd = [HARNESS, "-train", corpus, "-output", os.path.join(tmp, "out.vec"), "-debug", "0", "-binary", "1",
               "-streams", "1", "-kernel-batch-size", "4"] + flags
        r = subprocess.run(cmd, env=dict(os.environ, FW2V_REF_DUMP_DIR=dump), capture_output=True, check=True,
                           text=True)
        overall = [ln for ln in r.stdout.splitlines() if ln.startswith("Overall Words:")]
        per = [parse_dump(os.path.join(dump, f)) for f in sorted(os.listdir(dump))]
        arrays = {"corpus": np.frombuffer(text, np.uint8), "flags": np.array(" ".join(flags)),
                  "overall_words": np.array(int(overall[0].split(":")[1]), np.int64),
                  "n_threads": np.array(len(per), np.int32)}
        for t, (lens, alphas, ids, negs) in enumerate(per):
            arrays[f"t{t}_lens"] = lens
            arrays[f"t{t}_alphas"] = alphas
            arrays[f"t{t}_ids"] = ids.astype(np.int16)
            arrays[f"t{t}_negs"] = negs.astype(np.int16)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
        print(f"{name}: overall_words={int(arrays['overall_words'])} threads={len(per)}")
    finally:
        shutil.rmtree(tmp)


def main():
    if not os.path.exists(HARNESS):
        sys.exit(f"missing {HARNESS}: run `make -C oracle ref` first")
    only_shapes = "--shape" in sys.argv[1:]
    if not only_shapes:
        for name, gen, flags in CASES:
            run_case(name, gen(), flags.split())
        for name, gen, flags in SHUFFLE_CASES:
            run_shuffle_case(name, gen(), flags.split())
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import shape_cases
    for name in shape_cases.CASES:
        run_shape_case(name)


if __name__ == "__main__":
    main()
