/*
 * TEST / BENCHMARK INFRASTRUCTURE ONLY.
 *
 * Multi-threaded CPU restatement of the reference's training path, used as the
 * timed CPU baseline of bench.py ("port"): each host thread owns sampling
 * streams exactly as a reference thread does (FULL-W2V-driver.cu:80-354), builds
 * each sentence with the oracle's batch builder and trains it at once with the
 * FULL-W2V method (per-position context copies reused for the whole window
 * lifetime, one fresh read and one write-back per target row) on tables shared
 * by all threads without locks (Hogwild, like word2vec).  FP32, dot products
 * with eight partial sums and elementwise loops that the compiler vectorises.
 * The product never calls this file.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "fw2v_oracle.h"

typedef struct {
  const orc_sampler_cfg* scfg;
  const orc_train_cfg* tcfg;
  float* syn0;
  float* syn1;
  int tid, n_threads;
  int64_t max_entries_per_stream;
  uint64_t words_read, words_kept;
  int rc;
} worker_t;

/* The hot loops are compiled for AVX-512, AVX2 + FMA and the baseline ISA,
 * and the loader picks the widest the host supports (GCC function clones). */
#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__)
#define HOT __attribute__((target_clones("arch=skylake-avx512", "arch=haswell", "default")))
#else
#define HOT
#endif

HOT static float dot8(const float* restrict a, const float* restrict b, int d) {
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int e = 0;
  for (; e + 8 <= d; e += 8)
    for (int j = 0; j < 8; j++) s[j] += a[e + j] * b[e + j];
  float t = ((s[0] + s[4]) + (s[1] + s[5])) + ((s[2] + s[6]) + (s[3] + s[7]));
  for (; e < d; e++) t += a[e] * b[e];
  return t;
}

/* v += g*o and o += g*v_old */
HOT static void update2(float* restrict v, float* restrict o, float g, int d) {
  for (int e = 0; e < d; e++) {
    const float vo = v[e];
    v[e] = vo + g * o[e];
    o[e] += g * vo;
  }
}

/* row += a - b */
HOT static void add_delta(float* restrict row, const float* restrict a, const float* restrict b, int d) {
  for (int e = 0; e < d; e++) row[e] += a[e] - b[e];
}

static float grad(const orc_train_cfg* c, float x, int label, float alpha) {
  if (c->sigmoid == ORC_SIGMOID_TABLE) {
    float s = (x + 6.0f) * (1.0f / 12.0f);
    if (!(s > 0.0f)) s = 0.0f;
    if (s > 1.0f) s = 1.0f;
    int idx = (int)(s * 999.0f);
    return label ? alpha * c->exp_table[ORC_EXP_TABLE_SIZE - 1 - idx] : -alpha * c->exp_table[idx];
  }
  return label ? alpha / (1.0f + expf(x)) : -alpha / (1.0f + expf(-x));
}

static void train_sentence(const orc_train_cfg* c, float* syn0, float* syn1, int L, const int32_t* ids,
                           const int32_t* negs, float alpha, float* cur, float* orig, float* o, float* o0) {
  const int d = c->d, W = c->window, K = c->negative, D = 2 * W + 1;
  const int64_t P = c->pitch;
  int nin = W + 1 < L ? W + 1 : L;
  for (int p = 0; p < nin; p++) {
    memcpy(cur + (int64_t)p * d, syn0 + (int64_t)ids[p] * P, sizeof(float) * d);
    memcpy(orig + (int64_t)p * d, cur + (int64_t)p * d, sizeof(float) * d);
  }
  for (int w = 0; w < L; w++) {
    int base = w - W, ctx[32], n = 0;
    for (int r = 0; r < D; r++) {
      int p = base + ((r - base) % D + D) % D;
      if (p != w && p >= 0 && p < L) ctx[n++] = p;
    }
    if (n > 0) {
      for (int k = 0; k <= K; k++) {
        int32_t t = k == 0 ? ids[w] : negs[(int64_t)w * K + k - 1];
        float* row = syn1 + (int64_t)t * P;
        memcpy(o, row, sizeof(float) * d);
        memcpy(o0, row, sizeof(float) * d);
        for (int j = 0; j < n; j++) {
          float* v = cur + (int64_t)ctx[j] * d;
          float g = grad(c, dot8(v, o, d), k == 0, alpha);
          update2(v, o, g, d);
        }
        add_delta(row, o, o0, d);
      }
    }
    if (w - W >= 0) {
      int p = w - W;
      add_delta(syn0 + (int64_t)ids[p] * P, cur + (int64_t)p * d, orig + (int64_t)p * d, d);
    }
    if (w + W + 1 < L) {
      int p = w + W + 1;
      memcpy(cur + (int64_t)p * d, syn0 + (int64_t)ids[p] * P, sizeof(float) * d);
      memcpy(orig + (int64_t)p * d, cur + (int64_t)p * d, sizeof(float) * d);
    }
  }
  for (int p = L - W > 0 ? L - W : 0; p < L; p++)
    add_delta(syn0 + (int64_t)ids[p] * P, cur + (int64_t)p * d, orig + (int64_t)p * d, d);
}

static void* worker(void* arg) {
  worker_t* wk = (worker_t*)arg;
  const orc_sampler_cfg* sc = wk->scfg;
  const orc_train_cfg* tc = wk->tcfg;
  const int K = sc->negative, d = tc->d, msl = sc->msl;
  float* cur = (float*)malloc(sizeof(float) * (size_t)(msl + 1) * d);
  float* orig = (float*)malloc(sizeof(float) * (size_t)(msl + 1) * d);
  float* o = (float*)malloc(sizeof(float) * d);
  float* o0 = (float*)malloc(sizeof(float) * d);
  wk->rc = 0;
  for (int s = wk->tid; s < sc->threads && wk->rc == 0; s += wk->n_threads) {
    int64_t es, ee;
    orc_stream_range(sc, s, &es, &ee);
    int64_t cap = (ee < sc->n_chunks ? sc->chunk_off[ee] : sc->stream_len) - sc->chunk_off[es] + 2;
    int32_t* lens = (int32_t*)malloc(sizeof(int32_t) * cap);
    float* alphas = (float*)malloc(sizeof(float) * cap);
    int32_t* ids = (int32_t*)malloc(sizeof(int32_t) * cap);
    int32_t* negs = (int32_t*)malloc(sizeof(int32_t) * cap * (K > 0 ? K : 1));
    orc_stream_state st;
    orc_stream_init(sc, s, &st);
    for (int e = 0; e < sc->epochs && wk->rc == 0; e++) {
      int64_t ne = 0, nk = 0;
      uint64_t wr = 0;
      /* a bounded sample samples only the sentences it trains */
      if (wk->max_entries_per_stream > 0)
        wk->rc = orc_sample_epoch_prefix(sc, s, &st, wk->max_entries_per_stream, cap, lens, alphas, cap, ids, negs,
                                         &ne, &nk, &wr);
      else
        wk->rc = orc_sample_epoch(sc, s, &st, cap, lens, alphas, cap, ids, negs, &ne, &nk, &wr);
      if (wk->rc) break;
      int64_t off = 0;
      for (int64_t i = 0; i < ne; i++) {
        if (lens[i] > 0)
          train_sentence(tc, wk->syn0, wk->syn1, lens[i], ids + off, negs + off * K, alphas[i], cur, orig, o, o0);
        off += lens[i];
        wk->words_kept += (uint64_t)lens[i];
      }
      wk->words_read += wr;
    }
    free(lens);
    free(alphas);
    free(ids);
    free(negs);
  }
  free(cur);
  free(orig);
  free(o);
  free(o0);
  return NULL;
}

/* Train `scfg->epochs` epochs of every stream on n_threads host threads.
 * max_entries_per_stream > 0 bounds the sentences sampled and trained per
 * stream and epoch (a sample of the workload); words_read counts the tokens
 * those sentences consumed. */
int orc_cpu_sgns(const orc_sampler_cfg* scfg, const orc_train_cfg* tcfg, float* syn0, float* syn1neg,
                 int n_threads, int64_t max_entries_per_stream, uint64_t* words_read, uint64_t* words_kept) {
  if (n_threads < 1) n_threads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * n_threads);
  worker_t* wk = (worker_t*)calloc(n_threads, sizeof(worker_t));
  for (int t = 0; t < n_threads; t++) {
    wk[t].scfg = scfg;
    wk[t].tcfg = tcfg;
    wk[t].syn0 = syn0;
    wk[t].syn1 = syn1neg;
    wk[t].tid = t;
    wk[t].n_threads = n_threads;
    wk[t].max_entries_per_stream = max_entries_per_stream;
    pthread_create(&th[t], NULL, worker, &wk[t]);
  }
  int rc = 0;
  uint64_t wr = 0, kept = 0;
  for (int t = 0; t < n_threads; t++) {
    pthread_join(th[t], NULL);
    if (wk[t].rc) rc = wk[t].rc;
    wr += wk[t].words_read;
    kept += wk[t].words_kept;
  }
  free(th);
  free(wk);
  *words_read = wr;
  *words_kept = kept;
  return rc;
}
