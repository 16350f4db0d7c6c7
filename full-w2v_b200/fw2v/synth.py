"""Seeded synthetic corpora standing in for the reference's text8 / 1-Billion-Word
/ graph-walk corpora (not available offline): a topic-mixture corpus with
Zipf-distributed words, and random walks on a stochastic block model.  Both
come with a planted label per word (topic or block) for precision@10.

`build_stream` turns raw token ids into what the reference's text front end
would build from the same tokens written one sentence per line: a vocabulary
sorted by count (ties in first-occurrence order, "</s>" at index 0 with one
count per line but the last), the min-count cut, and the global token stream
cut into chunks of `msl` (improved_driver_functions.cpp:136-164, 244-281).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class SynthCorpus:
    counts: np.ndarray       # uint32, vocab order, index 0 = </s>
    train_words: int
    stream: object           # int32 vocab ids, trailing 0: numpy, or a CUDA tensor (device generators)
    chunk_off: object        # int64 chunk starts: numpy, or a CUDA tensor
    label: np.ndarray        # planted topic/block per vocab id (-1 for </s>)
    raw_of_vocab: np.ndarray  # raw id per vocab id (-1 for </s>)
    # share of a word's expected count that its planted topic contributes
    # (1 for graph nodes); words above 1/2 carry a recoverable planted label
    purity: np.ndarray | None = None

    def host_stream(self) -> np.ndarray:
        """The token stream in host memory (copied once from the device)."""
        if not isinstance(self.stream, np.ndarray):
            self.stream_host = getattr(self, "stream_host", None)
            if self.stream_host is None:
                self.stream_host = self.stream.cpu().numpy()
            return self.stream_host
        return self.stream

    def host_chunk_off(self) -> np.ndarray:
        return self.chunk_off if isinstance(self.chunk_off, np.ndarray) else self.chunk_off.cpu().numpy()

    @property
    def n_chunks(self) -> int:
        return len(self.chunk_off)

    @property
    def n_stream(self) -> int:
        return len(self.stream)


def topic_tokens(n_tokens: int, vocab: int, topics: int, zipf_s: float, *, sentence_len: int = 1000,
                 dirichlet: float = 0.1, seed: int = 0, chunk: int = 512):
    """Raw token ids of a topic-mixture corpus, and each raw word's planted topic.

    Every sentence draws topic weights from Dirichlet(dirichlet); every token
    draws a topic from them and a word from that topic's Zipf(zipf_s) law over
    its own random permutation of the vocabulary.  A word's planted topic is the
    topic under which it is most probable (its lowest rank).
    """
    rng = np.random.default_rng(seed)
    perm = np.stack([rng.permutation(vocab) for _ in range(topics)]).astype(np.int32)
    rank_p = 1.0 / np.arange(1, vocab + 1, dtype=np.float64) ** zipf_s
    cdf = np.cumsum(rank_p)
    cdf /= cdf[-1]
    n_sent = (n_tokens + sentence_len - 1) // sentence_len
    out = np.empty(n_sent * sentence_len, np.int32)
    for s0 in range(0, n_sent, chunk):
        s1 = min(n_sent, s0 + chunk)
        theta = rng.dirichlet(np.full(topics, dirichlet), size=s1 - s0)
        ctheta = np.cumsum(theta, axis=1)
        ctheta[:, -1] = 1.0
        u = rng.random((s1 - s0, sentence_len))
        z = np.empty((s1 - s0, sentence_len), np.int32)
        for i in range(s1 - s0):
            z[i] = np.searchsorted(ctheta[i], u[i], side="right")
        np.minimum(z, topics - 1, out=z)
        r = np.searchsorted(cdf, rng.random((s1 - s0, sentence_len)), side="right")
        np.minimum(r, vocab - 1, out=r)
        out[s0 * sentence_len:s1 * sentence_len] = perm[z, r].ravel()
    ranks = np.empty((topics, vocab), np.int32)
    ranks[np.arange(topics)[:, None], perm] = np.arange(vocab)[None, :]
    planted = np.argmin(ranks, axis=0).astype(np.int32)
    p = (ranks + 1.0) ** -zipf_s
    purity = p.max(0) / p.sum(0)
    return out[:n_tokens], planted, purity


def sbm_graph(nodes: int, blocks: int, degree: float, p_ratio: float, rng: np.random.Generator):
    """A stochastic block model multigraph in CSR form.

    Nodes are split into `blocks` equal blocks (node i in block
    i * blocks // nodes); a node's expected degree is `degree`, and an edge
    inside its block is p_ratio times as likely as one to any given node of
    another block: p_in (bsize - 1) + p_out (nodes - bsize) = degree with
    p_in = p_ratio p_out.  Edge counts are Poisson; an in-block edge joins a
    uniform node and a uniform other node of its block, a cross-block edge a
    uniform node and a uniform node of a uniform other block.  Returns
    (offsets int64 [nodes + 1], neighbours int32, block of each node int32).
    """
    block = (np.arange(nodes) * blocks // nodes).astype(np.int32)
    bsize = nodes / blocks
    p_out = degree / (p_ratio * (bsize - 1) + (nodes - bsize))
    n_in = rng.poisson(p_ratio * p_out * (bsize - 1) * nodes / 2)
    n_out = rng.poisson(p_out * (nodes - bsize) * nodes / 2) if blocks > 1 else 0
    a = rng.integers(0, nodes, n_in)
    lo = (block[a].astype(np.int64) * nodes) // blocks
    size = ((block[a].astype(np.int64) + 1) * nodes) // blocks - lo
    b = lo + (a - lo + 1 + (rng.random(n_in) * (size - 1)).astype(np.int64)) % size
    c = rng.integers(0, nodes, n_out)
    other = (block[c].astype(np.int64) + 1 + rng.integers(0, max(blocks - 1, 1), n_out)) % blocks
    lo2 = (other * nodes) // blocks
    dd = lo2 + (rng.random(n_out) * (((other + 1) * nodes) // blocks - lo2)).astype(np.int64)
    src = np.concatenate([a, b, c, dd])
    dst = np.concatenate([b, a, dd, c])
    ok = src != dst  # blocks of one node have no in-block partner
    src, dst = src[ok], dst[ok]
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order].astype(np.int32)
    offs = np.zeros(nodes + 1, np.int64)
    np.add.at(offs, src + 1, 1)
    return np.cumsum(offs), dst, block


def sbm_walks(nodes: int, blocks: int, degree: float, p_ratio: float, walks_per_node: int,
              walk_len: int, *, seed: int = 0):
    """Uniform random walks on a stochastic block model graph (sbm_graph).
    Returns (walks as an int32 [n_walks, walk_len] array of node ids, block of
    each node)."""
    rng = np.random.default_rng(seed)
    offs, dst, block = sbm_graph(nodes, blocks, degree, p_ratio, rng)
    deg = np.diff(offs)
    starts = np.repeat(np.arange(nodes, dtype=np.int32), walks_per_node)
    walks = np.empty((len(starts), walk_len), np.int32)
    cur = starts.copy()
    walks[:, 0] = cur
    for t in range(1, walk_len):
        dcur = deg[cur]
        nxt = cur.copy()
        has = dcur > 0
        pick = (rng.random(has.sum()) * dcur[has]).astype(np.int64)
        nxt[has] = dst[offs[cur[has]] + pick]
        cur = nxt
        walks[:, t] = cur
    return walks, block


def build_stream(raw: np.ndarray, sentence_ends: np.ndarray, raw_label: np.ndarray, *,
                 min_count: int, msl: int, cache_eos: bool = False) -> SynthCorpus:
    """Vocabulary, stream and chunks for raw ids written one sentence per line.

    sentence_ends: exclusive end offset of each line in `raw`.
    """
    n_raw = int(raw.max()) + 1 if len(raw) else 0
    cnt = np.bincount(raw, minlength=n_raw)
    first = np.full(n_raw, len(raw), np.int64)
    np.minimum.at(first, raw, np.arange(len(raw)))
    seen = np.nonzero(cnt)[0]
    order = seen[np.lexsort((first[seen], -cnt[seen]))]
    order = order[cnt[order] >= min_count]
    n_lines = len(sentence_ends)
    eos = max(n_lines - 1, 0)  # the final newline is read at EOF and not counted
    counts = np.concatenate([[eos], cnt[order]]).astype(np.uint32)
    vocab_of_raw = np.full(n_raw, -1, np.int64)
    vocab_of_raw[order] = np.arange(1, len(order) + 1)
    vid = vocab_of_raw[raw]
    if cache_eos:
        parts = []
        bounds = np.concatenate([[0], sentence_ends])
        for i in range(n_lines):
            seg = vid[bounds[i]:bounds[i + 1]]
            parts.append(seg[seg >= 0])
            parts.append(np.zeros(1, np.int64))
        ids = np.concatenate(parts).astype(np.int32)
        # chunk at EOS or msl (improved_driver_functions.cpp:270)
        offs, n = [], 0
        start = True
        for i, w in enumerate(ids):
            if start:
                offs.append(i)
                start = False
                n = 0
            n += 1
            if w == 0 or n >= msl:
                start = True
        chunk_off = np.array(offs, np.int64)
    else:
        ids = vid[vid >= 0].astype(np.int32)
        chunk_off = np.arange(0, len(ids), msl, dtype=np.int64)
    stream = np.concatenate([ids, np.zeros(1, np.int32)]).astype(np.int32)
    train_words = int(counts.sum()) + 1
    label = np.concatenate([[-1], raw_label[order]]).astype(np.int32)
    raw_of_vocab = np.concatenate([[-1], order]).astype(np.int64)
    return SynthCorpus(counts, train_words, stream, chunk_off, label, raw_of_vocab)


def text_of(raw: np.ndarray, sentence_ends: np.ndarray) -> bytes:
    """The corpus as a text file: tokens w<raw id>, one sentence per line."""
    lines, s = [], 0
    for e in sentence_ends:
        lines.append(" ".join(f"w{t}" for t in raw[s:e]))
        s = e
    return ("\n".join(lines) + "\n").encode()


# Workloads of the benchmark configurations (sizes and laws as specified there).
CONFIGS = {
    "c1": dict(n_tokens=1_000_000, vocab=10_000, topics=20, zipf_s=1.0, d=100, window=5,
               negative=5, sample=1e-4, epochs=1, min_count=1),
    "c2": dict(n_tokens=17_000_000, vocab=71_000, topics=100, zipf_s=1.0, d=128, window=8,
               negative=5, sample=1e-4, epochs=5, min_count=5),
    "c3": dict(n_tokens=800_000_000, vocab=555_000, topics=1000, zipf_s=1.05, d=300, window=5,
               negative=5, sample=1e-4, epochs=1, min_count=5),
}


def make_topic_corpus(name: str, *, n_tokens: int | None = None, seed: int | None = None,
                      msl: int = 1000) -> tuple[SynthCorpus, dict]:
    cfg = dict(CONFIGS[name])
    if n_tokens is not None:
        cfg["n_tokens"] = n_tokens
    seed = 1234 + int(name[1:]) if seed is None else seed
    raw, planted, purity = topic_tokens(cfg["n_tokens"], cfg["vocab"], cfg["topics"], cfg["zipf_s"],
                                        seed=seed)
    ends = np.arange(1000, len(raw) + 1000, 1000)
    ends[-1] = len(raw)
    corpus = build_stream(raw, ends, planted, min_count=cfg["min_count"], msl=msl)
    corpus.purity = np.concatenate([[0.0], purity[corpus.raw_of_vocab[1:]]])
    return corpus, cfg


# ---------------------------------------------------------------------------
# Device-side generation for the large configurations (seeded torch RNG on the
# GPU; the same seed gives the same corpus on the same device and software).
# ---------------------------------------------------------------------------

def _affine_perms(vocab: int, topics: int, rng: np.random.Generator):
    """Per-topic permutations r -> (a*r + b) mod V with gcd(a, V) = 1."""
    a, b = [], []
    while len(a) < topics:
        x = int(rng.integers(1, vocab))
        if np.gcd(x, vocab) == 1:
            a.append(x)
            b.append(int(rng.integers(0, vocab)))
    return np.array(a, np.int64), np.array(b, np.int64)


def topic_corpus_gpu(n_tokens: int, vocab: int, topics: int, zipf_s: float, *, min_count: int,
                     msl: int = 1000, sentence_len: int = 1000, dirichlet: float = 0.1, seed: int = 0,
                     device="cuda", heldout_tokens: int = 0):
    """The topic-mixture corpus of topic_tokens(), generated with torch on a
    device (each topic's Zipf law runs over an affine permutation of the
    vocabulary instead of a random one, so no V x topics table is needed).

    Returns (SynthCorpus, held-out stream as int32 vocab ids or None); the
    held-out tokens continue the same generator after the training tokens and
    drop words outside the training vocabulary.
    """
    import torch

    rng = np.random.default_rng(seed)
    a, b = _affine_perms(vocab, topics, rng)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    dev = torch.device(device)
    cdf = torch.cumsum(torch.arange(1, vocab + 1, device=dev, dtype=torch.float64).pow(-zipf_s), 0)
    cdf = cdf / cdf[-1]
    ta = torch.from_numpy(a).to(dev)
    tb = torch.from_numpy(b).to(dev)
    total = n_tokens + heldout_tokens
    n_sent = (total + sentence_len - 1) // sentence_len
    raw = torch.empty(n_sent * sentence_len, dtype=torch.int32, device=dev)
    conc = torch.full((topics,), dirichlet, device=dev)
    chunk = max(1, (1 << 27) // (topics * 4))
    for s0 in range(0, n_sent, chunk):
        s1 = min(n_sent, s0 + chunk)
        g = torch._standard_gamma(conc.expand(s1 - s0, topics).contiguous(), generator=gen)
        theta = g / g.sum(1, keepdim=True).clamp_min(1e-30)
        z = torch.multinomial(theta, sentence_len, replacement=True, generator=gen)
        u = torch.rand((s1 - s0, sentence_len), device=dev, generator=gen, dtype=torch.float64)
        r = torch.searchsorted(cdf, u).clamp_(max=vocab - 1)
        raw[s0 * sentence_len:s1 * sentence_len] = ((ta[z] * r + tb[z]) % vocab).reshape(-1).to(torch.int32)
    raw = raw[:total]
    # planted topic: the one under which a word's rank (a_z^-1 (w - b_z) mod V) is lowest
    inv = torch.from_numpy(np.array([pow(int(x), -1, vocab) for x in a], np.int64)).to(dev)
    words = torch.arange(vocab, device=dev, dtype=torch.int64)
    best = torch.full((vocab,), vocab, device=dev, dtype=torch.int64)
    planted = torch.zeros(vocab, device=dev, dtype=torch.int64)
    psum = torch.zeros(vocab, device=dev, dtype=torch.float64)
    for zt in range(topics):
        rk = (inv[zt] * ((words - tb[zt]) % vocab)) % vocab
        better = rk < best
        best = torch.where(better, rk, best)
        planted = torch.where(better, torch.full_like(planted, zt), planted)
        psum += (rk + 1.0).pow(-zipf_s)
    purity_raw = (best + 1.0).pow(-zipf_s) / psum
    train_raw = raw[:n_tokens].long()
    # vocabulary: count descending, ties by first occurrence, min-count cut
    cnt = torch.bincount(train_raw, minlength=vocab)
    first = torch.full((vocab,), n_tokens, device=dev, dtype=torch.int64)
    first.scatter_reduce_(0, train_raw, torch.arange(n_tokens, device=dev, dtype=torch.int64), reduce="amin")
    seen = torch.nonzero(cnt).flatten()
    order = seen[torch.argsort(first[seen], stable=True)]
    order = order[torch.argsort(-cnt[order], stable=True)]
    order = order[cnt[order] >= min_count]
    n_lines = (n_tokens + sentence_len - 1) // sentence_len
    counts = torch.cat([torch.tensor([max(n_lines - 1, 0)], device=dev), cnt[order]])
    vocab_of_raw = torch.full((vocab,), -1, device=dev, dtype=torch.int64)
    vocab_of_raw[order] = torch.arange(1, len(order) + 1, device=dev)
    vid = vocab_of_raw[train_raw]
    ids = vid[vid >= 0].to(torch.int32)
    # the stream and its chunks stay on the device (fw2v_load_corpus_device)
    stream = torch.cat([ids, torch.zeros(1, dtype=torch.int32, device=dev)])
    chunk_off = torch.arange(0, len(ids), msl, dtype=torch.int64, device=dev)
    counts_np = counts.cpu().numpy().astype(np.uint32)
    label = np.concatenate([[-1], planted[order].cpu().numpy()]).astype(np.int32)
    raw_of_vocab = np.concatenate([[-1], order.cpu().numpy()]).astype(np.int64)
    purity = np.concatenate([[0.0], purity_raw[order].cpu().numpy()])
    corpus = SynthCorpus(counts_np, int(counts_np.sum()) + 1, stream, chunk_off, label, raw_of_vocab, purity)
    held = None
    if heldout_tokens:
        hv = vocab_of_raw[raw[n_tokens:].long()]
        held = hv[hv >= 0].to(torch.int32).cpu().numpy()
    del raw, train_raw, vid
    if dev.type == "cuda":
        torch.cuda.empty_cache()
    return corpus, held


def make_topic_corpus_gpu(name: str, *, n_tokens: int | None = None, heldout_tokens: int = 0,
                          msl: int = 1000, device="cuda"):
    """A named configuration's topic corpus from topic_corpus_gpu:
    (corpus, held-out stream, config)."""
    cfg = dict(CONFIGS[name])
    if n_tokens is not None:
        cfg["n_tokens"] = n_tokens
    corpus, held = topic_corpus_gpu(cfg["n_tokens"], cfg["vocab"], cfg["topics"], cfg["zipf_s"],
                                    min_count=cfg["min_count"], msl=msl, seed=1234 + int(name[1:]),
                                    device=device, heldout_tokens=heldout_tokens)
    return corpus, held, cfg


def sbm_graph_torch(nodes: int, blocks: int, degree: float, p_ratio: float, rng: np.random.Generator,
                    gen, dev):
    """sbm_graph() with torch on device `dev` (edge counts from the numpy
    `rng`, endpoints from the torch generator `gen`): (offsets int64
    [nodes + 1], neighbours int32, block of each node int64), as tensors."""
    import torch
    block = (torch.arange(nodes, device=dev, dtype=torch.int64) * blocks) // nodes
    bsize = nodes / blocks
    p_out = degree / (p_ratio * (bsize - 1) + (nodes - bsize))
    n_in = int(rng.poisson(p_ratio * p_out * (bsize - 1) * nodes / 2))
    n_out = int(rng.poisson(p_out * (nodes - bsize) * nodes / 2)) if blocks > 1 else 0
    a = torch.randint(0, nodes, (n_in,), device=dev, generator=gen)
    lo = (block[a] * nodes) // blocks
    size = ((block[a] + 1) * nodes) // blocks - lo
    u = torch.rand(n_in, device=dev, generator=gen, dtype=torch.float64)
    b = lo + (a - lo + 1 + (u * (size - 1)).long()) % size
    c = torch.randint(0, nodes, (n_out,), device=dev, generator=gen)
    other = (block[c] + 1 + torch.randint(0, max(blocks - 1, 1), (n_out,), device=dev, generator=gen)) % blocks
    lo2 = (other * nodes) // blocks
    u2 = torch.rand(n_out, device=dev, generator=gen, dtype=torch.float64)
    d = lo2 + (u2 * (((other + 1) * nodes) // blocks - lo2)).long()
    src = torch.cat([a, b, c, d])
    dst = torch.cat([b, a, d, c])
    del a, b, c, d, lo, size, u, other, lo2, u2
    ok = src != dst  # blocks of one node have no in-block partner
    src, dst = src[ok], dst[ok]
    order = torch.argsort(src, stable=True)
    src, dst = src[order], dst[order].to(torch.int32).contiguous()
    deg = torch.bincount(src, minlength=nodes)
    offs = torch.zeros(nodes + 1, device=dev, dtype=torch.int64)
    offs[1:] = torch.cumsum(deg, 0)
    return offs, dst, block


def sbm_corpus_gpu(nodes: int, blocks: int, degree: float, p_ratio: float, walks_per_node: int, walk_len: int, *,
                   seed: int = 0, device="cuda", min_count: int = 1, heldout_walks: int = 0):
    """sbm_walks() generated on a device, written as the reference's text
    front end would read the walks one per line with -cache-eos: every walk is
    a sentence ending in </s> and a stored chunk of its own.  The graph is
    built with torch; the walks come from this library's walk kernel
    (fw2v_random_walks, counter-based per (seed, walk, step)) straight into the
    token stream, which stays on the device.  The vocabulary is the visited
    nodes by count (ties by first occurrence).

    Returns (SynthCorpus with each node's block as its label and purity 1,
    held-out walks as int32 vocab ids with a 0 after each, or None).
    """
    import torch

    from . import lib
    if min_count > 1:
        raise ValueError("walk corpora keep every visited node (min_count 1)")
    dev = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    offs, dst, block = sbm_graph_torch(nodes, blocks, degree, p_ratio, np.random.default_rng(seed), gen, dev)
    cs = torch.cuda.current_stream(dev)

    def walks(starts, wseed):
        """Walks from `starts` as a stream: walk w at w * (walk_len + 1), raw
        node ids, a -1 after each walk, one trailing slot."""
        out = torch.empty(len(starts) * (walk_len + 1) + 1, device=dev, dtype=torch.int32)
        st = lib().fw2v_random_walks(offs.data_ptr(), dst.data_ptr(), nodes, starts.data_ptr(), len(starts),
                                     walk_len, wseed, out.data_ptr(), cs.cuda_stream)
        if st != 0:
            raise RuntimeError(f"fw2v_random_walks failed: status {st}")
        out[-1] = -1
        return out

    starts = torch.arange(nodes, device=dev, dtype=torch.int32).repeat_interleave(walks_per_node).contiguous()
    stream = walks(starts, seed)
    n_walks = len(starts)
    body = stream[:-1].view(n_walks, walk_len + 1)[:, :walk_len]
    flat = body.reshape(-1).long()
    n = flat.numel()
    cnt = torch.bincount(flat, minlength=nodes)
    first = torch.full((nodes,), n, device=dev, dtype=torch.int64)
    first.scatter_reduce_(0, flat, torch.arange(n, device=dev, dtype=torch.int64), reduce="amin")
    del flat
    seen = torch.nonzero(cnt).flatten()
    vorder = seen[torch.argsort(first[seen], stable=True)]
    vorder = vorder[torch.argsort(-cnt[vorder], stable=True)]
    vocab_of = torch.zeros(nodes, device=dev, dtype=torch.int32)
    vocab_of[vorder] = torch.arange(1, len(vorder) + 1, device=dev, dtype=torch.int32)
    counts = torch.cat([torch.tensor([max(n_walks - 1, 0)], device=dev), cnt[vorder]]).cpu().numpy().astype(np.uint32)

    def relabel(t):
        st = lib().fw2v_relabel_stream(t.data_ptr(), t.numel(), vocab_of.data_ptr(), nodes, cs.cuda_stream)
        if st != 0:
            raise RuntimeError(f"fw2v_relabel_stream failed: status {st}")
        return t

    relabel(stream)  # node ids -> vocabulary ids, the separators and the trailing slot -> 0
    chunk_off = torch.arange(n_walks, device=dev, dtype=torch.int64) * (walk_len + 1)
    label = np.concatenate([[-1], block[vorder].cpu().numpy()]).astype(np.int32)
    raw_of_vocab = np.concatenate([[-1], vorder.cpu().numpy()]).astype(np.int64)
    purity = np.concatenate([[0.0], np.ones(len(vorder))])
    corpus = SynthCorpus(counts, int(counts.sum()) + 1, stream, chunk_off, label, raw_of_vocab, purity)
    held = None
    if heldout_walks:
        hs = torch.randint(0, nodes, (heldout_walks,), device=dev, generator=gen).to(torch.int32).contiguous()
        held = relabel(walks(hs, seed ^ 0x48454C44))[:-1].cpu().numpy()
    if dev.type == "cuda":
        torch.cuda.empty_cache()
    return corpus, held


# Graph-walk workloads: C4 (one 1M-node graph) and the jobs of C5 (256 graphs of
# log-uniform size), as specified for the benchmark configurations.
GRAPH_CONFIGS = {
    "c4": dict(nodes=1_000_000, blocks=64, degree=20.0, p_ratio=20.0, walks_per_node=10, walk_len=80, d=128,
               window=10, negative=5, sample=1e-3, epochs=1),
}


def c5_job_specs(n_jobs: int = 256, seed: int = 5, scale: float = 1.0):
    """Per-job specifications of the batched configuration: log-uniform 1k-200k
    nodes (times `scale`), 4-64 blocks, average degree 10-30, 10 walks of 40-80
    per node, d in {64, 128}, window in {5, 10}, negative 5, its own seed."""
    rng = np.random.default_rng(seed)
    out = []
    for j in range(n_jobs):
        nodes = int(round(np.exp(rng.uniform(np.log(1_000), np.log(200_000))) * scale))
        out.append(dict(nodes=max(nodes, 64), blocks=int(rng.integers(4, 65)), degree=float(rng.uniform(10, 30)),
                        p_ratio=20.0, walks_per_node=10, walk_len=int(rng.integers(40, 81)),
                        d=int(rng.choice([64, 128])), window=int(rng.choice([5, 10])), negative=5, sample=1e-3,
                        epochs=1, seed=int(rng.integers(1, 2**31))))
    return out
