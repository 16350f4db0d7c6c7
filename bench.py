#!/usr/bin/env python3
"""Benchmark: trained words/sec of SGNS on B200 (one step = one training epoch).

Workload (default): the text-scale corpus — 17M tokens over a 71k vocabulary,
Zipf(1.0) ranks in a 100-topic mixture with Dirichlet(0.1) weights per
1000-token sentence, seeded synthetic data — trained with d=128, window=8,
negative=5, sample=1e-4, alpha=0.025, FP32 tables, on the reference's method.
"Trained words" counts every token read, subsampled-away ones included, as the
reference's "Overall Words Per Second" does (FULL-W2V-driver.cu:205, 450).

Own arm (default): the library's epoch loop through its C ABI.
  value   device time of K epochs (sampler + trainer), inputs resident in HBM,
          L2 flushed (256 MB write) between epochs and not timed.
  e2e     the same through the public API from host buffers: every step copies
          the token stream from pinned host memory (fw2v_load_corpus), trains
          one epoch and reads the word count back.
  reference_gpu  (N=1) the reference's own CUDA program (baseline/_ref/FULL-W2V,
          built unmodified from its sources for sm_100a) and this project's
          plain FP32 kernel, each training the text-scale corpus (C2) for its 5
          epochs on this GPU: the reference's "Overall Words Per Second" beside
          ours.  The reference kernel cannot run the default workload (d=300:
          its 8-float reduce scratch overlaps index_cache for d > 256,
          FULL-W2V-kernels.cu:117-120, and d % 32 != 0 gives partial-warp
          shuffles).
Reference arm (--impl reference): the reference's own program on the same
corpus written as text (c1/c2), its host threads on all host cores; or, where
it cannot run, the CPU restatement of its training path (oracle port).

Multi-GPU (torchrun): replicas only — every rank trains its own copy of the job,
value = words of all ranks / max over ranks of the timed device time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "full-w2v_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "trained words/sec"
UNIT = "words/s"
L2_FLUSH_BYTES = 256 << 20


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            # a reason counts even in a sample whose clocks did not read
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def default_streams(n_chunks: int) -> int:
    """Sampling streams (the reference's -threads): enough for the GPU sampler,
    few enough that each stream's dropped epoch-end partial sentence is a small
    share of its words (each stream spans >= 256 stored sentences)."""
    return int(max(1, min(4096, n_chunks // 256)))


def cpu_baseline(corpus, cfg, threads, seconds_target=15.0):
    """The oracle's CPU restatement (sampling + Hogwild FP32 training) on all host
    cores, on a bounded sample: the first sentences of every stream of one epoch."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    d = cfg["d"]
    V = len(corpus.counts)
    ocorp = O.Corpus(corpus.host_stream(), corpus.host_chunk_off(), corpus.counts, [], corpus.train_words)
    kw = dict(threads=threads, msl=1000, negative=cfg["negative"], epochs=1, alpha0=0.025,
              sample=cfg["sample"], d=d, window=cfg["window"], n_threads=cores)
    syn0 = O.init_syn0(V, d, d)
    syn1 = np.zeros_like(syn0)
    t0 = time.perf_counter()
    per = 1
    wr, wk = O.cpu_sgns(ocorp, syn0, syn1, max_entries_per_stream=per, **kw)
    dt = time.perf_counter() - t0
    # grow the sample to ~seconds_target of CPU work
    per = int(max(1, min(10_000, per * seconds_target / max(dt, 1e-3))))
    t0 = time.perf_counter()
    wr, wk = O.cpu_sgns(ocorp, syn0, syn1, max_entries_per_stream=per, **kw)
    dt = time.perf_counter() - t0
    return {"value": wr / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {per} sentences of each of {threads} streams of one epoch "
                      f"({wr} words read, {wk} kept) in {dt:.1f} s; oracle/fw2v_cpu_sgns.c, "
                      f"FP32 Hogwild on {cores} threads"}


def make_corpus(args):
    """(corpus, held-out stream or None, config) of the workload: the numpy
    generator for c1/c2 (the reference program reads the same corpus as text),
    the device generators for c3 (800M tokens) and c4 (walks on a 1M-node
    graph, 800M tokens)."""
    from fw2v import synth
    if args.config == "c3":
        return synth.make_topic_corpus_gpu(args.config, n_tokens=args.tokens, heldout_tokens=args.heldout)
    if args.config == "c4":
        g = dict(synth.GRAPH_CONFIGS["c4"])
        if args.tokens:
            g["nodes"] = max(1000, args.tokens // (g["walks_per_node"] * (g["walk_len"] + 1)))
        corpus, held = synth.sbm_corpus_gpu(g["nodes"], g["blocks"], g["degree"], g["p_ratio"],
                                            g["walks_per_node"], g["walk_len"], seed=1234 + 4,
                                            heldout_walks=max(1, args.heldout // (g["walk_len"] + 1)))
        cfg = dict(g, n_tokens=len(corpus.stream) - 1, min_count=1)
        return corpus, held, cfg
    corpus, cfg = synth.make_topic_corpus(args.config, n_tokens=args.tokens)
    return corpus, None, cfg


def job_config(args, cfg, T, epochs, precision):
    import fw2v
    return fw2v.default_config(layer_size=cfg["d"], window=cfg["window"], negative=cfg["negative"], epochs=epochs,
                               threads=T, msl=1000, alpha=0.025, sample=cfg["sample"], precision=precision)


def timed_epochs(args, world, dev, run_epochs, flush, stream, back_to_back):
    """W untimed epochs, then K timed ones bracketed by barrier + synchronize.
    run_epochs(n) trains n epochs -> (words read, words kept, device ms,
    kernel launches, training-kernel ms, training-kernel launches).
    back_to_back: the K epochs run as one call, so that every epoch's
    sampling overlaps the training before it as in a real run (inputs larger
    than L2); otherwise one call per epoch with L2 flushed (untimed) before
    each."""
    import torch
    for _ in range(args.warmup):
        run_epochs(1)
    barrier(world)
    torch.cuda.synchronize(dev)
    res = []
    if back_to_back:
        res.append(run_epochs(args.steps))
    else:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)  # L2 flush, not timed
            torch.cuda.synchronize(dev)
            res.append(run_epochs(1))
    torch.cuda.synchronize(dev)
    barrier(world)
    return res


def single_job_epochs(tr, n, dev, tstream):
    """n epochs of a single-job handle timed on the device: an event before
    the first, and one recorded once the device is idle after the last (the
    handle samples the next epoch on a second stream while one trains)."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(tstream)
    words = kept = 0
    train_ms = 0.0
    for _ in range(n):
        st = tr.train_epoch()
        words += st.words_read
        kept += st.words_kept
        train_ms += st.train_ms
    torch.cuda.synchronize(dev)
    e1.record(tstream)
    e1.synchronize()
    return words, kept, e0.elapsed_time(e1), 4 * n, train_ms, n


def heldout(tr_cls, corpus, cfg, pairs, syn0, syn1):
    """Mean held-out SGNS loss per pair of tables (FP32 evaluation of the values)."""
    import fw2v
    from fw2v import evaluate
    c = fw2v.default_config(layer_size=cfg["d"], window=cfg["window"], negative=cfg["negative"], epochs=1,
                            threads=1, msl=1000, sample=0.0)
    with tr_cls(c) as t:
        t.set_vocab(corpus.counts, corpus.train_words)
        t.set_tables(syn0, syn1)
        return evaluate.heldout_loss(t, pairs)


def run_own(args, world, rank, local):
    import torch

    import fw2v
    from fw2v import evaluate

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    corpus, held, cfg = make_corpus(args)
    T = args.streams or default_streams(len(corpus.chunk_off))
    d, W, K = cfg["d"], cfg["window"], cfg["negative"]
    epochs = args.warmup + args.steps
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    form = args.form
    # tables and corpus far larger than L2 (C3, C4): time the epochs back to back
    back_to_back = args.config in ("c3", "c4") and not args.per_epoch
    bf16 = form.startswith("bf16")
    prec = fw2v.BF16 if bf16 else fw2v.FP32
    pairs = None
    if held is not None and len(held) > 0:
        pairs = evaluate.heldout_pairs(corpus.counts, corpus.train_words, held, window=W, negative=K)
    tune_cache = os.path.join(tempfile.mkdtemp(prefix="fw2v_tune_"), "tune.json")
    tuned = None

    with ClockSampler(local) as clk:
        if form.endswith("batched"):
            b = fw2v.Batch(precision=prec, device=local, group_bytes=args.group_bytes)
            b.add_job(job_config(args, cfg, T, epochs, prec), corpus.counts, corpus.train_words, corpus.stream,
                      corpus.chunk_off)
            if args.shape:  # a given shape instead of the tuner's
                b.set_shape(0, *[int(x) for x in args.shape.split(",")])
                if args.wpb:
                    for f in range(3):
                        b.set_launch(f, min(args.wpb, (8, 6, 4)[f]))
                tuned = {"given": args.shape, "warps_per_block": args.wpb}
            else:
                tuned = b.tune(cache=tune_cache)

            def run_epochs(n):
                # per round: sampler, negatives, entry prefix, job bookkeeping, trainer
                st = b.train_epochs(n)
                return st.words_read, st.words_kept, st.ms, 5 * st.rounds * n, st.train_ms, st.train_launches

            res = timed_epochs(args, world, dev, run_epochs, flush, stream, back_to_back)
            shape = b.shape(0)
            b.close()
        else:
            tr = fw2v.Trainer(job_config(args, cfg, T, epochs, prec))
            tr.set_vocab(corpus.counts, corpus.train_words)
            tr.load_corpus(corpus.stream, corpus.chunk_off)
            tstream = torch.cuda.ExternalStream(tr.stream_handle(), device=dev)

            # per epoch: sampler, negatives, entry prefix, trainer
            res = timed_epochs(args, world, dev, lambda n: single_job_epochs(tr, n, dev, tstream), flush, stream,
                               back_to_back)
            shape = None
            tr.close()
    words = sum(r[0] for r in res)  # res: (read, kept, epoch ms, launches, train ms, train launches)
    kept = sum(r[1] for r in res)
    total_s = max_over_ranks(world, sum(r[2] for r in res) / 1e3)
    value = sum_over_ranks(world, float(words)) / total_s

    def quality(s0, s1):
        """Held-out loss and precision@10 of tables trained for exactly one
        epoch (the configurations' epoch count)."""
        loss = heldout(fw2v.Trainer, corpus, cfg, pairs, s0, s1) if pairs is not None else None
        p10 = None
        if corpus.purity is not None:
            p10, _ = evaluate.precision_at_10(s0, corpus.label, corpus.counts, purity=corpus.purity, device=dev)
        return loss, p10

    # e2e: through the public API from pinned host buffers, every step
    pinned = torch.empty(len(corpus.stream), dtype=torch.int32, pin_memory=True)
    pinned.numpy()[:] = corpus.host_stream()
    host_chunks = corpus.host_chunk_off()
    host_stream = pinned.numpy()
    e2e_steps = max(1, min(args.steps, 2))
    e2e_words, e2e_s = 0, 0.0
    for i in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xFF)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        if form.endswith("batched"):
            with fw2v.Batch(precision=prec, device=local, group_bytes=args.group_bytes) as eb:
                eb.add_job(job_config(args, cfg, T, 1, prec), corpus.counts, corpus.train_words, host_stream,
                           host_chunks)
                if args.shape:
                    eb.set_shape(0, *[int(x) for x in args.shape.split(",")])
                    if args.wpb:
                        for f in range(3):
                            eb.set_launch(f, min(args.wpb, (8, 6, 4)[f]))
                else:
                    eb.tune(cache=tune_cache)  # the shapes chosen above, from the cache
                st = eb.train_epochs(1)
                e2e_words += st.words_read
                e2e_s += time.perf_counter() - t0
                if i == 0:  # a fresh one-epoch model of the value's form: its quality (untimed)
                    loss, p10 = quality(eb.syn0(0), eb.syn1neg(0))
        else:
            with fw2v.Trainer(job_config(args, cfg, T, 1, prec)) as et:
                et.set_vocab(corpus.counts, corpus.train_words)
                et.load_corpus(host_stream, host_chunks)
                et.sample_epoch()
                e2e_words += et.train_sampled().words_read
                e2e_s += time.perf_counter() - t0
                if i == 0:
                    loss, p10 = quality(et.syn0(), et.syn1neg())
    e2e_s = max_over_ranks(world, e2e_s)
    e2e_value = sum_over_ranks(world, float(e2e_words)) / e2e_s
    h2d = 4 * len(corpus.stream) + 8 * len(corpus.chunk_off) + corpus.counts.nbytes
    d2h = 8 * T + 16

    # the plain FP32 kernel on the same workload, for the form's speed-up
    compare = None
    if form != "fp32" and not args.no_compare:
        # speed: one untimed epoch, then min(K, 2) timed the same way as the value's
        n_cmp = min(args.steps, 2)
        with fw2v.Trainer(job_config(args, cfg, T, 1 + n_cmp, fw2v.FP32)) as tr:
            tr.set_vocab(corpus.counts, corpus.train_words)
            tr.load_corpus(corpus.stream, corpus.chunk_off)
            tstream = torch.cuda.ExternalStream(tr.stream_handle(), device=dev)
            tr.train_epoch()
            torch.cuda.synchronize(dev)
            if back_to_back:
                cres = [single_job_epochs(tr, n_cmp, dev, tstream)]
            else:
                cres = []
                for i in range(n_cmp):
                    with torch.cuda.stream(stream):
                        flush.fill_(i & 0xFF)
                    torch.cuda.synchronize(dev)
                    cres.append(single_job_epochs(tr, 1, dev, tstream))
        cw, ms = sum(r[0] for r in cres), sum(r[2] for r in cres)
        cval = sum_over_ranks(world, float(cw)) / max_over_ranks(world, ms / 1e3)
        # quality: a fresh one-epoch FP32 model
        with fw2v.Trainer(job_config(args, cfg, T, 1, fw2v.FP32)) as tq:
            tq.set_vocab(corpus.counts, corpus.train_words)
            tq.load_corpus(corpus.stream, corpus.chunk_off)
            tq.train_epoch()
            closs, cp10 = quality(tq.syn0(), tq.syn1neg())
        compare = {"form": "fp32 (single-job kernel, untuned)", "value": cval, "unit": UNIT,
                   "epochs_timed": n_cmp, "heldout_loss": closs, "precision_at_10": cp10,
                   "speedup": value / cval,
                   "heldout_loss_rel_diff": (loss - closs) / closs if loss is not None and closs else None}

    hbm, peak_kind = peaks()
    elem = 2 if bf16 else 4
    kept_per_epoch = kept / args.steps
    epoch_ms = total_s * 1e3 / args.steps
    bytes_per_epoch = kept_per_epoch * (2 * d * elem * (K + 2) + 4 * (1 + K))
    # the training kernel's own launches: CUDA events around each one on its stream
    n_launch = sum(r[5] for r in res)
    train_ms = sum(r[4] for r in res)
    timed_launches = n_launch > 0 and all(r[4] > 0 for r in res)
    launch_ms = train_ms / n_launch if timed_launches else epoch_ms
    bytes_per_launch = bytes_per_epoch * args.steps / n_launch if timed_launches else bytes_per_epoch
    achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr_map = json.load(f)
        key = f"{args.config}:{args.tokens or cfg['n_tokens']}:{form}"
        if key in tr_map:
            traffic = tr_map[key]["dram_bytes_per_launch"]
    kernel = "sgns_batch_kernel" if form.endswith("batched") else "sgns_train_kernel"
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": epoch_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16-tables/f32-math" if bf16 else "f32",
        "data": "synthetic (seeded " + ("random walks on a stochastic block model" if args.config == "c4"
                                         else "topic-mixture corpus") + ", generated in-process)",
        "config": {"workload": f"{args.config}: {cfg['n_tokens']/1e6:.0f}M-token "
                               f"{'walk' if args.config == 'c4' else 'topic'} corpus, "
                               f"V={len(corpus.counts)}, d={d}, window={W}, negative={K}, sample={cfg['sample']}, "
                               f"msl=1000, {T} sampling streams; form {form}",
                   "form": form, "tokens_per_epoch": int(len(corpus.stream) - 1), "vocab": len(corpus.counts),
                   "layer_size": d, "window": W, "negative": K, "streams": T, "shape": shape,
                   "tuning": tuned,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": ("tables and corpus exceed L2; the K timed epochs run back to back in one call"
                          if back_to_back else "flushed between steps (256 MB write, untimed)"),
                   "quality": "held-out loss and precision@10 of fresh one-epoch models of each form"},
        "heldout_loss": loss,
        "precision_at_10": p10,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "gpu_launches": int(sum(r[3] for r in res)),  # all of this library's kernels in the timed epochs
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "kernel": kernel, "peak_kind": peak_kind,
                     "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms, "launches": n_launch,
                     "note": "algorithmic bytes of a training launch (rows of 1+K targets and one context per "
                             "kept word, read and written, plus its ids) over the launch's device time (CUDA "
                             "events on its stream); epoch_ms includes sampling"},
        "epoch_ms": epoch_ms,
        "breakdown": {"kept_fraction": kept / max(words, 1)},
    }
    if compare is not None:
        out["fp32_plain"] = compare
    clocks = clk.summary()
    if clocks:
        out["clocks"] = clocks
    if args.config == "c3":
        out["config"]["notes"] = (
            "subsampling is inactive at this corpus shape (kept_fraction 1.0): the 1000-topic mixture flattens "
            "every word's marginal frequency below the sample=1e-4 threshold; same-topic precision@10 after one "
            "epoch is at chance for both precisions (about 1% of context pairs share a topic), so the held-out "
            "SGNS loss is the quality gate here")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(corpus, cfg, T)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        del corpus, held, pairs
        out["reference_gpu"] = reference_gpu(local, args.reference_gpu, args.ref_walks_per_node)
    return out


def safe_reference_threads(corpus, cfg, epochs, cores, streams=4, batch=200):
    """Host threads for the reference program under which every launch reads
    only buffers it has filled: each thread must ship more than streams x
    batch sentences over the run, or its final launch (FULL-W2V-driver.cu:
    305-318, all `batch` blocks of stream S-1) replays unfilled buffers.
    Sentences per thread come from this library's sampler, which reproduces
    the reference's batch builder bit for bit."""
    import fw2v
    threads = min(cores, len(corpus.chunk_off))
    while threads >= 1:
        c = fw2v.default_config(layer_size=8, window=cfg["window"], negative=cfg["negative"], epochs=1,
                                threads=threads, msl=1000, alpha=0.025, sample=cfg["sample"])
        with fw2v.Trainer(c) as t:
            t.set_vocab(corpus.counts, corpus.train_words)
            t.load_corpus(corpus.stream, corpus.chunk_off)
            t.sample_epoch()
            least = min(len(r[0]) for r in t.epoch_samples())
        if least * epochs >= streams * batch + 1:
            return threads
        threads //= 2
    return 0


def run_reference_program(binary, text, cfg, epochs, threads, streams=4, batch=200, extra=()):
    """FULL-W2V on a text corpus; (words/s, overall seconds) or a reason string."""
    cmd = [binary, "-train", text] + list(extra) + [ "-size", str(cfg["d"]), "-window", str(cfg["window"]),
           "-negative", str(cfg["negative"]), "-sample", str(cfg["sample"]), "-iter", str(epochs),
           "-alpha", "0.025", "-min-count", str(cfg["min_count"]), "-threads", str(threads),
           "-streams", str(streams), "-kernel-batch-size", str(batch), "-msl", "1000",
           "-debug", "0", "-no-export", "-output", os.devnull]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        return f"reference exited {r.returncode}: {r.stderr[-300:]}"
    wps = [ln for ln in r.stdout.splitlines() if ln.startswith("Overall Words Per Second:")]
    tim = [ln for ln in r.stdout.splitlines() if ln.startswith("Overall time:")]
    if not wps:
        return "no words/sec line from the reference"
    return float(wps[0].split(":")[1]), (float(tim[0].split(":")[1]) if tim else None)


def write_walk_text(corpus, path, walk_len):
    """A walk corpus as text, one walk per line, each word its vocabulary id:
    the reference's text front end builds the same vocabulary from it (counts,
    ties by first occurrence) and, with -cache-eos, the same sentences."""
    ids = corpus.host_stream()[:-1].reshape(-1, walk_len + 1)[:, :walk_len]
    with open(path, "w") as f:
        for s0 in range(0, len(ids), 100_000):
            np.savetxt(f, ids[s0:s0 + 100_000], fmt="%d", delimiter=" ")


def reference_gpu(local, which="c2", walks_per_node=1):
    """The reference's CUDA program and the plain FP32 kernel of this library on
    the same corpus, one after the other on this GPU.  c2: the text-scale
    corpus (17M tokens, V=71k after min-count 5, d=128, window 8, negative 5,
    sample 1e-4, 5 epochs).  c4: the 1M-node stochastic-block-model graph
    with `walks_per_node` walks of 80 per node (C4 has 10), written one walk
    per line and read with -cache-eos (d=128, window 10, sample 1e-3, 1
    epoch).  Each rate is the implementation's own: the reference's "Overall
    Words Per Second" (its clock runs from after set-up to its final device
    sync, FULL-W2V-driver.cu:162, 324, 450); ours, words read over the device
    time of the epochs (sampler and trainer, CUDA events)."""
    import torch

    import fw2v
    from fw2v import synth
    binary = os.path.join(ROOT, "baseline", "_ref", "FULL-W2V")
    if not os.path.exists(binary):
        return {"unavailable": "baseline/_ref/FULL-W2V not built (make -C baseline with the reference checkout)"}
    dev = torch.device("cuda", local)
    tmp = tempfile.mkdtemp(prefix="fw2v_ref_")
    text = os.path.join(tmp, "corpus.txt")
    try:
        if which == "c2":
            cfg = dict(synth.CONFIGS["c2"])
            raw, planted, _ = synth.topic_tokens(cfg["n_tokens"], cfg["vocab"], cfg["topics"], cfg["zipf_s"],
                                                 seed=1236)
            ends = np.arange(1000, len(raw) + 1000, 1000)
            ends[-1] = len(raw)
            corpus = synth.build_stream(raw, ends, planted, min_count=cfg["min_count"], msl=1000)
            with open(text, "wb") as f:
                f.write(synth.text_of(raw, ends))
            del raw
            extra = ()
            workload = (f"c2: {cfg['n_tokens'] / 1e6:.0f}M-token topic corpus, V={len(corpus.counts)}, d={cfg['d']}, "
                        f"window={cfg['window']}, negative={cfg['negative']}, sample={cfg['sample']}, msl=1000, "
                        f"{cfg['epochs']} epochs")
        else:
            g = dict(synth.GRAPH_CONFIGS["c4"])
            corpus, _ = synth.sbm_corpus_gpu(g["nodes"], g["blocks"], g["degree"], g["p_ratio"], walks_per_node,
                                             g["walk_len"], seed=1234 + 4)
            write_walk_text(corpus, text, g["walk_len"])
            cfg = dict(g, min_count=1)
            extra = ("-cache-eos",)
            workload = (f"c4 graph ({g['nodes']} nodes, {g['blocks']} blocks), {walks_per_node} walk(s) of "
                        f"{g['walk_len']} per node ({len(corpus.stream) - 1} tokens with </s>), V={len(corpus.counts)}, "
                        f"d={g['d']}, window={g['window']}, negative={g['negative']}, sample={g['sample']}, "
                        f"-cache-eos, {g['epochs']} epoch")
        epochs = cfg["epochs"]
        cores = os.cpu_count() or 1
        threads = safe_reference_threads(corpus, cfg, epochs, cores)
        if threads < 1:
            return {"unavailable": "corpus too small for the reference's launch pattern"}
        ref = run_reference_program(binary, text, cfg, epochs, threads, extra=extra)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if isinstance(ref, str):
        return {"unavailable": ref}
    T = default_streams(len(corpus.chunk_off))
    c = fw2v.default_config(layer_size=cfg["d"], window=cfg["window"], negative=cfg["negative"], epochs=epochs,
                            threads=T, msl=1000, alpha=0.025, sample=cfg["sample"])
    with fw2v.Trainer(c) as t:
        t.set_vocab(corpus.counts, corpus.train_words)
        t.load_corpus(corpus.stream, corpus.chunk_off)
        ts = torch.cuda.ExternalStream(t.stream_handle(), device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(ts)
        words = t.train()
        e1.record(ts)
        e1.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
    ours = words / secs
    return {"workload": workload + "; both on this GPU, one after the other",
            "reference": {"value": ref[0], "unit": UNIT, "overall_time_s": ref[1], "host_threads": threads,
                          "streams": 4, "kernel_batch_size": 200,
                          "program": "baseline/_ref/FULL-W2V: the reference's FULL-W2V-driver.cu and "
                                     "FULL-W2V-kernels.cu, unmodified, nvcc -O3 -Xptxas -dlcm=ca for sm_100a"},
            "fp32_plain": {"value": ours, "unit": UNIT, "device_time_s": secs, "words": int(words),
                           "sampling_streams": T, "kernel": "sgns_train_kernel, default shape"},
            "speedup": ours / ref[0]}


def run_c5(args, world, rank, local):
    """The batched configuration: 256 independent graph jobs (synth.c5_job_specs,
    node counts times --scale).  Each job is generated on the device, trained
    alone with the plain FP32 single-job kernel (timed, scored), then added to
    one batch that trains all of them in the value's form (tuned, one CUDA
    graph).  value = words of all jobs / the batch's device time; fp32_alone =
    the same words / the sum of the jobs' own device times.  On N ranks the jobs
    are partitioned by token count (fw2v.shard.assign_jobs); each rank trains
    its share, and the words of all ranks count over the slowest rank's time."""
    import torch

    import fw2v
    from fw2v import evaluate, synth
    from fw2v.shard import combine_ranks, rank_share

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    all_specs = synth.c5_job_specs(scale=args.scale)
    specs = [all_specs[j] for j in rank_share(all_specs, world, rank)]
    prec = fw2v.BF16 if args.form.startswith("bf16") else fw2v.FP32
    batch = fw2v.Batch(precision=prec, device=local, group_bytes=args.group_bytes)
    labels, alone_p10, alone_ms, alone_words = [], [], 0.0, 0
    for j, s in enumerate(specs):
        corpus, _ = synth.sbm_corpus_gpu(s["nodes"], s["blocks"], s["degree"], s["p_ratio"], s["walks_per_node"],
                                         s["walk_len"], seed=s["seed"])
        T = default_streams(len(corpus.chunk_off))
        cfg = fw2v.default_config(layer_size=s["d"], window=s["window"], negative=s["negative"], epochs=s["epochs"],
                                  threads=T, msl=1000, alpha=0.025, sample=s["sample"], seed=s["seed"])
        if not args.no_compare:
            with fw2v.Trainer(cfg) as t:
                t.set_vocab(corpus.counts, corpus.train_words)
                t.load_corpus(corpus.stream, corpus.chunk_off)
                ts = torch.cuda.ExternalStream(t.stream_handle(), device=dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(ts)
                alone_words += t.train()
                e1.record(ts)
                e1.synchronize()
                alone_ms += e0.elapsed_time(e1)
                alone_p10.append(evaluate.precision_at_10(t.syn0(), corpus.label, corpus.counts,
                                                          purity=corpus.purity, device=dev)[0])
        batch.add_job(cfg, corpus.counts, corpus.train_words, corpus.stream, corpus.chunk_off)
        labels.append((corpus.label, corpus.counts, corpus.purity))
        del corpus
    tuned = batch.tune()
    barrier(world)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        st = batch.train()
        torch.cuda.synchronize(dev)
    barrier(world)
    tot = combine_ranks(st.words_read, st.ms / 1e3, alone_words, alone_ms / 1e3, device=dev)
    batch_s, words_all, value = tot["seconds"], tot["words"], tot["value"]
    p10 = [evaluate.precision_at_10(batch.syn0(j), *labels[j][:2], purity=labels[j][2], device=dev)[0]
           for j in range(len(specs))]
    batch.close()
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 0,
           "ms_per_step": batch_s * 1e3, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
           "vs_baseline": None,
           "dtype": "bf16-tables/f32-math" if prec == fw2v.BF16 else "f32",
           "data": "synthetic (seeded random walks on 256 stochastic block models, generated in-process)",
           "config": {"workload": f"c5: {len(all_specs)} graph jobs, {words_all / 1e9:.2f}B tokens, one batch per "
                                  f"rank; form {args.form}", "form": args.form, "jobs": len(all_specs),
                      "jobs_this_rank": len(specs), "scale": args.scale,
                      "parallelism": f"jobs partitioned over {world} ranks" if world > 1 else "single GPU",
                      "rounds": st.rounds, "group_bytes": args.group_bytes, "tuning": tuned},
           "precision_at_10": {"mean": float(np.nanmean(p10)), "min": float(np.nanmin(p10))},
           "gpu_launches": 5 * st.rounds}
    if alone_p10:
        diff = np.array(p10) - np.array(alone_p10)
        alone_value = tot["alone_value"]
        out["fp32_alone"] = {"form": "each job alone, fp32 single-job kernel", "value": alone_value,
                             "unit": UNIT, "speedup": value / alone_value,
                             "precision_at_10_mean": float(np.nanmean(alone_p10)),
                             "p10_diff_mean": float(np.nanmean(diff)), "p10_diff_min": float(np.nanmin(diff)),
                             "jobs_within_1_point": int(np.sum(diff >= -0.01))}
    clocks = clk.summary()
    if clocks:
        out["clocks"] = clocks
    return out


def run_reference(args, world, rank):
    """The reference program (oracle/_ref/FULL-W2V) on the same corpus, or the
    CPU port where it cannot run."""
    from fw2v import synth
    from oracle import oracle as O

    if world > 1 and rank != 0:
        return None
    if args.config == "c5":
        return {"impl": "reference", "unavailable": "the reference trains one corpus per process; the batched "
                                                    "configuration has no reference form (use --config c3)"}
    corpus, _, cfg = make_corpus(args)
    T_stream = args.streams or default_streams(len(corpus.chunk_off))
    cores = os.cpu_count() or 1
    binary = os.path.join(ROOT, "baseline", "_ref", "FULL-W2V")
    reason = None
    if args.config not in ("c1", "c2"):
        reason = f"{args.config} is generated on the device and is not written as text for the reference program"
    elif cfg["d"] > 256 or cfg["d"] % 32:
        reason = f"reference kernel unsupported at d={cfg['d']} (shared-memory overlap / partial warp)"
    elif not os.path.exists(binary):
        reason = "baseline/_ref/FULL-W2V not built"
    if reason is None:
        res = reference_program(args, corpus, cfg, binary, cores)
        if isinstance(res, dict):
            return res
        reason = res
    base = cpu_baseline(corpus, cfg, T_stream)
    base["sample"] += f"; reference program not run: {reason}"
    return {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config}, "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def reference_program(args, corpus, cfg, binary, cores):
    """FULL-W2V on the workload's corpus written as text, with host threads
    under which every launch reads only buffers it has filled
    (safe_reference_threads)."""
    epochs = args.steps
    threads = safe_reference_threads(corpus, cfg, epochs, cores)
    if threads < 1:
        return "corpus too small for the reference's launch pattern"
    raw_text = synth_text(args, cfg)
    if raw_text is None:
        return "could not write the corpus as text"
    try:
        res = run_reference_program(binary, raw_text, cfg, epochs, threads)
    finally:
        shutil.rmtree(os.path.dirname(raw_text), ignore_errors=True)
    if isinstance(res, str):
        return res
    value, secs = res
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": epochs,
            "warmup": 0, "ms_per_step": secs * 1e3 / epochs if secs else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (same seeded corpus, written as text)", "impl": "reference",
            "config": {"workload": f"{args.config} as text, reference FULL-W2V sm_100a",
                       "threads": threads, "streams": 4, "kernel_batch_size": 200},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{epochs} epochs of the full corpus; the reference's "
                                       f"host threads on {threads} cores feed its sm_100a kernel"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def synth_text(args, cfg):
    from fw2v import synth
    n = args.tokens or cfg["n_tokens"]
    seed = 1234 + int(args.config[1:])
    raw, _, _ = synth.topic_tokens(n, cfg["vocab"], cfg["topics"], cfg["zipf_s"], seed=seed)
    ends = np.arange(1000, len(raw) + 1000, 1000)
    ends[-1] = len(raw)
    tmp = tempfile.mkdtemp(prefix="fw2v_ref_")
    path = os.path.join(tmp, "corpus.txt")
    with open(path, "wb") as f:
        s = 0
        for e in ends:
            f.write((" ".join(f"w{t}" for t in raw[s:e]) + "\n").encode())
            s = e
    return path


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fw2v", choices=["fw2v", "reference"])
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--scale", type=float, default=1.0, help="c5: node counts of the jobs times this")
    ap.add_argument("--tokens", type=int, default=None, help="override the corpus size")
    ap.add_argument("--streams", type=int, default=None, help="sampling streams (-threads)")
    ap.add_argument("--form", default="bf16-batched", choices=["bf16-batched", "fp32-batched", "bf16", "fp32"],
                    help="tables and kernel: batched (persistent multi-job kernel, tuned, CUDA graph) or the "
                         "single-job kernel")
    ap.add_argument("--heldout", type=int, default=1_000_000, help="held-out tokens (c3)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP32 comparison run")
    ap.add_argument("--shape", default=None, help="batched forms: lane_vec,lane_nv,stages,prefetch instead of tuning")
    ap.add_argument("--wpb", type=int, default=0, help="batched forms with --shape: warps per block")
    ap.add_argument("--group-bytes", type=int, default=0,
                    help="batched forms: table bytes per group of interleaved jobs (0: half of L2, -1: one group)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--per-epoch", action="store_true",
                    help="c3/c4: time one call per epoch with L2 flushed between them instead of back to back")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's CUDA program against the plain FP32 kernel")
    ap.add_argument("--reference-gpu", default="c2", choices=["c2", "c4"],
                    help="corpus of that comparison: c2 (text scale) or c4 (the 1M-node walk graph)")
    ap.add_argument("--ref-walks-per-node", type=int, default=1, help="c4 comparison: walks per node (C4: 10)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.config == "c5":
        out = run_c5(args, world, rank, local)
    else:
        out = run_own(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
