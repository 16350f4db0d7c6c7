"""Loader for the golden fixtures written by tests/golden/make_golden.py."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["zipf_t1", "eos_t1", "zipf_t3", "nosample_t2", "k0_t1", "messy_t1"]


def parse_flags(flags: str) -> dict:
    toks = flags.split()
    out = {"cache_eos": False}
    i = 0
    while i < len(toks):
        t = toks[i]
        if t == "-cache-eos":
            out["cache_eos"] = True
            i += 1
            continue
        out[t.lstrip("-").replace("-", "_")] = toks[i + 1]
        i += 2
    cfg = {
        "size": int(out.get("size", 100)), "window": int(out.get("window", 5)),
        "negative": int(out.get("negative", 5)), "sample": float(out.get("sample", 1e-3)),
        "iter": int(out.get("iter", 5)), "threads": int(out.get("threads", 12)),
        "min_count": int(out.get("min_count", 5)), "msl": int(out.get("msl", 1000)),
        "alpha": float(out.get("alpha", 0.025)), "cache_eos": out["cache_eos"],
    }
    return cfg


def load(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: z[k] for k in z.files}
    g["cfg"] = parse_flags(str(g["flags"]))
    g["text"] = g["corpus"].tobytes()
    T = int(g["n_threads"])
    g["threads_out"] = [
        {"lens": g[f"t{t}_lens"], "alphas": g[f"t{t}_alphas"],
         "ids": g[f"t{t}_ids"].astype(np.int32), "negs": g[f"t{t}_negs"].astype(np.int32)}
        for t in range(T)
    ]
    C = int(g["cache_n_threads"])
    g["cache_threads_out"] = [
        {"lens": g[f"c{t}_lens"], "alphas": g[f"c{t}_alphas"],
         "ids": g[f"c{t}_ids"].astype(np.int32), "negs": g[f"c{t}_negs"].astype(np.int32)}
        for t in range(C)
    ]
    g["cache_text"] = g["corpus_cache"].tobytes()
    g["vocab_text"] = "".join(f"{w} {c}\n" for w, c in zip(g["vocab_words"], g["vocab_counts"])).encode("latin-1")
    return g
