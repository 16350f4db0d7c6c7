/*
 * TEST INFRASTRUCTURE ONLY — see fw2v_oracle.h.  CPU restatement of the FULL-W2V
 * hot path; the product library never links or calls this file.
 *
 * Build with -ffp-contract=off: the FP32 mode reproduces the CUDA kernel's
 * operation order exactly and must not let the C compiler fuse a*b+c on its own.
 */
#include "fw2v_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LCG_MUL 25214903917ULL
#define LCG_ADD 11ULL

uint64_t orc_lcg_next(uint64_t r) { return r * LCG_MUL + LCG_ADD; }

/* generate_expTable_h.cpp:46-55: val = exp((i/size*2-1)*MAX_EXP) in float,
 * val/(val+1); the first entry is printed as 0 and the last as 1. */
void orc_exp_table(float* t) {
  const int size = ORC_EXP_TABLE_SIZE;
  for (int i = 0; i < size; i++) {
    float x = ((float)i / (float)size * 2.0f - 1.0f) * 6.0f;
    float val = expf(x);
    val = val / (val + 1.0f);
    if (i == 0) val = 0.0f;
    if (i + 1 == size) val = 1.0f;
    t[i] = val;
  }
}

/* improved_driver_functions.cpp:27-31, from LCG state `start` (1 there) */
void orc_init_syn0_from(float* syn0, int64_t V, int d, int64_t pitch, uint64_t start) {
  uint64_t r = start;
  for (int64_t row = 0; row < V; row++) {
    for (int c = 0; c < d; c++) {
      r = orc_lcg_next(r);
      syn0[row * pitch + c] = (((float)(r & 0xFFFF) / 65536.0f) - 0.5f) / (float)d;
    }
    for (int64_t c = d; c < pitch; c++) syn0[row * pitch + c] = 0.0f;
  }
}

void orc_init_syn0(float* syn0, int64_t V, int d, int64_t pitch) { orc_init_syn0_from(syn0, V, d, pitch, 1); }

/* improved_driver_functions.cpp:71-77: base = (float)(sample * train_words),
 * ratio = base / count, keep threshold = sqrtf(ratio) + ratio, all in float. */
void orc_subsample_table(const uint32_t* counts, int64_t V, float sample, uint64_t train_words,
                         float* p_keep) {
  float base = sample * (float)train_words;
  for (int64_t i = 0; i < V; i++) {
    float ratio = base / (float)counts[i];
    p_keep[i] = sqrtf(ratio) + ratio;
  }
}

/* improved_driver_functions.cpp:44-58.  The power sum is sequential (the
 * reference's OpenMP reduction is sequential when built without OpenMP).  The
 * fill starts from word 1 with the running share initialised to word 0's share
 * (the outer `i` is still 0 at :50), so word 1 receives </s>'s share. */
int64_t orc_unigram_runs(const uint32_t* counts, int64_t V, int64_t table_size, int64_t* run_start,
                         int32_t* run_word, int32_t* table) {
  if (V < 2) return 0;
  double total = 0.0;
  for (int64_t i = 0; i < V; i++) total += pow((double)counts[i], 0.75);
  double d1 = pow((double)counts[0], 0.75) / total;
  int32_t i = 1;
  int64_t n_runs = 0;
  run_start[0] = 0;
  run_word[0] = 1;
  n_runs = 1;
  for (int64_t a = 0; a < table_size; a++) {
    if (table) table[a] = i;
    if ((double)a / (double)table_size > d1) {
      if (i < V - 1) {
        i++;
        if (a + 1 < table_size) {
          run_start[n_runs] = a + 1;
          run_word[n_runs] = i;
          n_runs++;
        }
      }
      d1 += pow((double)counts[i], 0.75) / total;
    }
  }
  run_start[n_runs] = table_size;
  return n_runs;
}

int32_t orc_unigram_lookup(const int64_t* run_start, const int32_t* run_word, int64_t n_runs,
                           int64_t index) {
  int64_t lo = 0, hi = n_runs - 1;
  while (lo < hi) {
    int64_t mid = (lo + hi + 1) / 2;
    if (run_start[mid] <= index) lo = mid;
    else hi = mid - 1;
  }
  return run_word[lo];
}

/* FULL-W2V-driver.cu:103-110: contiguous chunk ranges, the remainder spread one
 * each over the lowest stream ids. */
void orc_stream_range(const orc_sampler_cfg* cfg, int stream_id, int64_t* first, int64_t* end) {
  int64_t per = cfg->n_chunks / cfg->threads, left = cfg->n_chunks % cfg->threads;
  int64_t start = 0;
  for (int64_t i = 0; i < stream_id; i++) start += per + (i < left ? 1 : 0);
  *first = start;
  *end = start + per + (stream_id < left ? 1 : 0);
}

/* FULL-W2V-driver.cu:113-114: next_random starts at the thread id. */
void orc_stream_init(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st) {
  st->lcg = (uint64_t)stream_id;
  st->wca_own = 0;
  st->alpha = cfg->alpha0;
}

/* FULL-W2V-driver.cu:168-190: the learning rate follows the global word count.
 * With T streams that advance together the global count is T times this
 * stream's own contribution (exactly the reference for T = 1). */
static void refresh_alpha(const orc_sampler_cfg* cfg, orc_stream_state* st) {
  uint64_t global = (uint64_t)cfg->threads * st->wca_own;
  float denom = (float)((uint64_t)cfg->epochs * cfg->train_words + 1);
  st->alpha = cfg->alpha0 * (1 - (float)global / denom);
  if (st->alpha < cfg->alpha0 * 0.0001f) st->alpha = cfg->alpha0 * 0.0001f;
}

/* FULL-W2V-driver.cu:166-302 for one stream and one epoch. */
/* One epoch of a stream, or its first stop_after entries (stop_after > 0):
 * the entries are the same as the full epoch's first ones and *words_read
 * counts the tokens those entries consumed. */
static int sample_epoch(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st, int64_t stop_after,
                        int64_t cap_entries, int32_t* lens, float* alphas, int64_t cap_kept, int32_t* ids,
                        int32_t* negs, int64_t* n_entries, int64_t* n_kept, uint64_t* words_read) {
  int64_t es, ee;
  orc_stream_range(cfg, stream_id, &es, &ee);
  const int K = cfg->negative;
  uint64_t word_count = 0, last_word_count = 0;
  int64_t ss = es, cur = 0;
  int64_t ne = 0, nk = 0;
  for (;;) {
    if (word_count - last_word_count > 10000) {
      st->wca_own += word_count - last_word_count;
      last_word_count = word_count;
      refresh_alpha(cfg, st);
    }
    int32_t L = 0;
    while (L < cfg->msl) {
      if (cur >= cfg->msl) {
        ss++;
        cur = 0;
        if (ss >= ee) break;
      }
      if (ss >= cfg->n_chunks) return -2;
      int64_t pos = cfg->chunk_off[ss] + cur;
      if (pos < 0 || pos >= cfg->stream_len) return -2;
      int32_t w = cfg->stream[pos];
      cur++;
      word_count++;
      if (w == 0 || ss >= ee) {
        ss++;
        cur = 0;
        break;
      }
      if (cfg->sample > 0) {
        st->lcg = orc_lcg_next(st->lcg);
        if (cfg->p_keep[w] < (float)(st->lcg & 0xFFFF) / 65536.0f) continue;
      }
      if (nk + L >= cap_kept) return -1;
      ids[nk + L] = w;
      for (int k = 0; k < K; k++) {
        st->lcg = orc_lcg_next(st->lcg);
        int64_t idx = (int64_t)((st->lcg >> 16) % (uint64_t)cfg->table_size);
        negs[(nk + L) * K + k] = orc_unigram_lookup(cfg->run_start, cfg->run_word, cfg->n_runs, idx);
      }
      L++;
    }
    if (ne >= cap_entries) return -1;
    if (ss >= ee) {
      /* Epoch end (:233-277): flush the count, drop the partial sentence. */
      st->wca_own += word_count - last_word_count;
      lens[ne] = 0;
      alphas[ne] = st->alpha;
      ne++;
      break;
    }
    lens[ne] = L;
    alphas[ne] = st->alpha;
    ne++;
    nk += L;
    if (stop_after > 0 && ne >= stop_after) break;
  }
  *n_entries = ne;
  *n_kept = nk;
  *words_read = word_count;
  return 0;
}

int orc_sample_epoch(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st,
                     int64_t cap_entries, int32_t* lens, float* alphas, int64_t cap_kept,
                     int32_t* ids, int32_t* negs, int64_t* n_entries, int64_t* n_kept,
                     uint64_t* words_read) {
  return sample_epoch(cfg, stream_id, st, 0, cap_entries, lens, alphas, cap_kept, ids, negs, n_entries, n_kept,
                      words_read);
}

int orc_sample_epoch_prefix(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st,
                            int64_t max_entries, int64_t cap_entries, int32_t* lens, float* alphas,
                            int64_t cap_kept, int32_t* ids, int32_t* negs, int64_t* n_entries,
                            int64_t* n_kept, uint64_t* words_read) {
  return sample_epoch(cfg, stream_id, st, max_entries > 0 ? max_entries : 1, cap_entries, lens, alphas, cap_kept,
                      ids, negs, n_entries, n_kept, words_read);
}

/* ---------------- SGNS update ---------------- */

static int table_index_f32(float x) {
  /* FULL-W2V-kernels.cu:92-99 */
  const float dilute = 1.0f / 12.0f;
  float s = (x + 6.0f) * dilute;
  if (!(s > 0.0f)) s = 0.0f; /* __saturatef: NaN -> 0 */
  if (s > 1.0f) s = 1.0f;
  return (int)(s * 999.0f);
}

static float grad_f32(const orc_train_cfg* cfg, float x, int label, float alpha) {
  if (cfg->sigmoid == ORC_SIGMOID_TABLE) {
    int idx = table_index_f32(x);
    /* positive: +alpha * nexpTable[idx] = expTable[999-idx]; negatives: -alpha * expTable[idx] */
    return label ? alpha * cfg->exp_table[ORC_EXP_TABLE_SIZE - 1 - idx]
                 : (-alpha) * cfg->exp_table[idx];
  }
  return label ? alpha / (1.0f + expf(x)) : (-alpha) / (1.0f + expf(-x));
}

static double grad_f64(const orc_train_cfg* cfg, double x, int label, float alpha) {
  if (cfg->sigmoid == ORC_SIGMOID_TABLE) {
    double s = (x + 6.0) / 12.0;
    if (!(s > 0.0)) s = 0.0;
    if (s > 1.0) s = 1.0;
    int idx = (int)(s * 999.0);
    return label ? (double)alpha * cfg->exp_table[ORC_EXP_TABLE_SIZE - 1 - idx]
                 : -(double)alpha * cfg->exp_table[idx];
  }
  return label ? (double)alpha / (1.0 + exp(x)) : -(double)alpha / (1.0 + exp(-x));
}

/* Dot product with the CUDA kernel's order: lane l of 32 holds elements
 * ((i*32+l)*vec + j), i < nv, j < vec, and keeps two running sums, "even"
 * (j = 0, 2) and "odd" (j = 1, 3), each first a product then FMAs in (i, j)
 * order (the kernel's packed FP32x2 FMAs); the lane's partial is even + odd,
 * and lanes are combined by the xor tree with masks 16, 8, 4, 2, 1 (zero
 * beyond d). */
static float dot_f32(const orc_train_cfg* cfg, const float* a, const float* b) {
  float part[32];
  for (int l = 0; l < 32; l++) {
    float pe = 0.0f, po = 0.0f;
    int first = 1;
    for (int i = 0; i < cfg->nv; i++) {
      for (int j = 0; j < cfg->vec; j += 2) {
        int e = (i * 32 + l) * cfg->vec + j;
        float x0 = e < cfg->d ? a[e] : 0.0f, y0 = e < cfg->d ? b[e] : 0.0f;
        float x1 = e + 1 < cfg->d ? a[e + 1] : 0.0f, y1 = e + 1 < cfg->d ? b[e + 1] : 0.0f;
        if (first) {
          pe = x0 * y0;
          po = x1 * y1;
          first = 0;
        } else {
          pe = fmaf(x0, y0, pe);
          po = fmaf(x1, y1, po);
        }
      }
    }
    part[l] = pe + po;
  }
  /* Lanes l and l^m add the same two values, so after each level the lanes of
   * a group agree and lane 0's sums are the tree: part[l] + part[l + m]. */
  for (int m = 16; m >= 1; m >>= 1)
    for (int l = 0; l < m; l++) part[l] = part[l] + part[l + m];
  return part[0];
}

/* Context positions of centre w in ring-slot order: ascending (p mod (2W+1))
 * over the window [w-W, w+W] clipped to the sentence, centre excluded
 * (the steady-state order of FULL-W2V-kernels.cu:170-182). */
static int context_list(int w, int W, int L, int* ctx) {
  int D = 2 * W + 1, n = 0, base = w - W;
  for (int r = 0; r < D; r++) {
    int off = ((r - base) % D + D) % D;
    int p = base + off;
    if (p != w && p >= 0 && p < L) ctx[n++] = p;
  }
  return n;
}

#define DEFINE_TRAIN(NAME, T, DOT, GRAD, UPD_V, UPD_O, ZERO)                                         \
  static int NAME##_sentence(const orc_train_cfg* cfg, T* syn0, T* syn1, int64_t V, int32_t L,     \
                             const int32_t* ids, const int32_t* negs, float alpha, T* cur,        \
                             T* orig, T* o, T* o0, int* ctx) {                                    \
    const int d = cfg->d, W = cfg->window, K = cfg->negative;                                     \
    const int64_t P = cfg->pitch;                                                                  \
    for (int32_t p = 0; p < L; p++)                                                               \
      if (ids[p] < 0 || ids[p] >= V) return -3;                                                    \
    for (int64_t q = 0; q < (int64_t)L * K; q++)                                                  \
      if (negs[q] < 0 || negs[q] >= V) return -3;                                                  \
    int n_enter = W + 1 < L ? W + 1 : L;                                                           \
    for (int p = 0; p < n_enter; p++)                                                             \
      for (int e = 0; e < d; e++) cur[(int64_t)p * d + e] = orig[(int64_t)p * d + e] =            \
          syn0[(int64_t)ids[p] * P + e];                                                           \
    for (int w = 0; w < L; w++) {                                                                  \
      int n = context_list(w, W, L, ctx);                                                         \
      if (n > 0) {                                                                                 \
        for (int k = 0; k <= K; k++) {                                                            \
          int32_t t = k == 0 ? ids[w] : negs[(int64_t)w * K + k - 1];                             \
          int label = k == 0;                                                                      \
          for (int e = 0; e < d; e++) o0[e] = o[e] = syn1[(int64_t)t * P + e];                    \
          for (int j = 0; j < n; j++) {                                                            \
            T* v = cur + (int64_t)ctx[j] * d;                                                      \
            T x = DOT(cfg, v, o);                                                                  \
            T g = GRAD(cfg, x, label, alpha);                                                      \
            for (int e = 0; e < d; e++) {                                                          \
              T vo = v[e];                                                                         \
              v[e] = UPD_V(g, o[e], vo);                                                           \
              o[e] = UPD_O(g, vo, o[e]);                                                           \
            }                                                                                      \
          }                                                                                        \
          for (int e = 0; e < d; e++) {                                                            \
            T delta = o[e] - o0[e];                                                                \
            syn1[(int64_t)t * P + e] = syn1[(int64_t)t * P + e] + delta;                          \
          }                                                                                        \
        }                                                                                          \
      }                                                                                            \
      if (w - W >= 0) {                                                                            \
        int p = w - W;                                                                             \
        for (int e = 0; e < d; e++) {                                                              \
          T delta = cur[(int64_t)p * d + e] - orig[(int64_t)p * d + e];                           \
          syn0[(int64_t)ids[p] * P + e] = syn0[(int64_t)ids[p] * P + e] + delta;                  \
        }                                                                                          \
      }                                                                                            \
      if (w + W + 1 < L) {                                                                         \
        int p = w + W + 1;                                                                         \
        for (int e = 0; e < d; e++) cur[(int64_t)p * d + e] = orig[(int64_t)p * d + e] =          \
            syn0[(int64_t)ids[p] * P + e];                                                         \
      }                                                                                            \
    }                                                                                              \
    for (int p = L - W > 0 ? L - W : 0; p < L; p++) {                                              \
      for (int e = 0; e < d; e++) {                                                                \
        T delta = cur[(int64_t)p * d + e] - orig[(int64_t)p * d + e];                             \
        syn0[(int64_t)ids[p] * P + e] = syn0[(int64_t)ids[p] * P + e] + delta;                    \
      }                                                                                            \
    }                                                                                              \
    (void)ZERO;                                                                                    \
    return 0;                                                                                      \
  }                                                                                                \
  int NAME(const orc_train_cfg* cfg, T* syn0, T* syn1, int64_t V, int64_t n_sent,                 \
           const int64_t* starts, const int32_t* lens, const float* alphas, const int32_t* ids,    \
           const int32_t* negs) {                                                                  \
    int32_t maxL = 0;                                                                              \
    for (int64_t s = 0; s < n_sent; s++)                                                           \
      if (lens[s] > maxL) maxL = lens[s];                                                          \
    const int d = cfg->d;                                                                          \
    T* cur = (T*)malloc(sizeof(T) * ((size_t)maxL + 1) * d);                                       \
    T* orig = (T*)malloc(sizeof(T) * ((size_t)maxL + 1) * d);                                      \
    T* o = (T*)malloc(sizeof(T) * d);                                                              \
    T* o0 = (T*)malloc(sizeof(T) * d);                                                             \
    int* ctx = (int*)malloc(sizeof(int) * (2 * cfg->window + 1));                                  \
    int rc = 0;                                                                                    \
    for (int64_t s = 0; s < n_sent && rc == 0; s++) {                                              \
      if (lens[s] <= 0) continue;                                                                  \
      rc = NAME##_sentence(cfg, syn0, syn1, V, lens[s], ids + starts[s],                          \
                           negs + starts[s] * cfg->negative, alphas[s], cur, orig, o, o0, ctx);   \
    }                                                                                              \
    free(cur);                                                                                     \
    free(orig);                                                                                    \
    free(o);                                                                                       \
    free(o0);                                                                                      \
    free(ctx);                                                                                     \
    return rc;                                                                                     \
  }

static double dot_f64(const orc_train_cfg* cfg, const double* a, const double* b) {
  double s = 0.0;
  for (int e = 0; e < cfg->d; e++) s += a[e] * b[e];
  return s;
}
#define UPD_F32(g, y, x) fmaf((g), (y), (x))
#define UPD_F64(g, y, x) ((x) + (g) * (y))

DEFINE_TRAIN(orc_train_f32, float, dot_f32, grad_f32, UPD_F32, UPD_F32, 0)
DEFINE_TRAIN(orc_train_f64, double, dot_f64, grad_f64, UPD_F64, UPD_F64, 0)

/* ---- bfloat16 tables (FP32 math, stochastic-rounded write-back) ---- */
static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}
/* The library's stochastic-rounding bits: a key per sentence, then 32-bit
 * mixing per event and per vector of a row. */
static uint64_t sr_sentence_key(uint64_t seed, uint64_t uid) {
  return mix64(seed ^ mix64(uid * 0x9E3779B97F4A7C15ULL));
}
static uint64_t sr_event_key(uint64_t skey, uint64_t event) {
  return (skey & 0xFFFFFFFF00000000ULL) | (uint32_t)((uint32_t)skey ^ fmix32((uint32_t)event * 0x9E3779B9u + 1u));
}
static uint64_t sr_vector_bits(uint64_t key, uint64_t row, uint64_t vec) {
  uint32_t lo = fmix32((uint32_t)key ^ ((uint32_t)row * 0x27D4EB2Fu) ^ ((uint32_t)vec * 0x165667B1u));
  uint32_t hi = (lo ^ (uint32_t)(key >> 32)) * 0x9E3779B9u;
  hi ^= hi >> 15;
  return ((uint64_t)hi << 32) | lo;
}
static float bf16_f(uint16_t h) {
  uint32_t b = (uint32_t)h << 16;
  float x;
  memcpy(&x, &b, 4);
  return x;
}
static uint16_t bf16_sr(float x, uint32_t r16) {
  uint32_t b;
  memcpy(&b, &x, 4);
  if ((b & 0x7F800000u) == 0x7F800000u) return (uint16_t)((b >> 16) | ((b & 0x007FFFFFu) ? 0x40 : 0));
  return (uint16_t)((b + (r16 & 0xFFFFu)) >> 16);
}
uint16_t orc_bf16_nearest(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  if ((b & 0x7F800000u) == 0x7F800000u) return (uint16_t)((b >> 16) | ((b & 0x007FFFFFu) ? 0x40 : 0));
  return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
}

/* One element of the write-back of a row that moved from b to a: the
 * increment SR(a) - b, rounded to bfloat16, added to the stored value with
 * round-to-nearest-even.  Both addends are bfloat16, so their float sum rounds
 * to the same bfloat16 as the exact sum. */
uint16_t orc_bf16_writeback1(uint16_t stored, float a, float b, uint32_t r16) {
  float inc = bf16_f(orc_bf16_nearest(bf16_f(bf16_sr(a, r16)) - b));
  return orc_bf16_nearest(bf16_f(stored) + inc);
}

static void bf16_writeback(uint16_t* row, const float* a, const float* b, int d, int vec, uint64_t key,
                           uint64_t row_id) {
  for (int e = 0; e < d; e++) {
    uint64_t bits = sr_vector_bits(key, row_id, (uint64_t)(e / vec));
    row[e] = orc_bf16_writeback1(row[e], a[e], b[e], (uint32_t)(bits >> (16 * (e % vec))) & 0xFFFFu);
  }
}

/* Serial SGNS on bfloat16 tables with the kernel's FP32 order (orc_train_f32)
 * and its stochastic rounding: sentence s is uid s, target k of centre w is
 * event w*(K+1)+k, the leaving position q is event L*(K+1)+q. */
int orc_train_bf16(const orc_train_cfg* cfg, uint16_t* syn0, uint16_t* syn1, int64_t V, int64_t n_sent,
                   const int64_t* starts, const int32_t* lens, const float* alphas, const int32_t* ids,
                   const int32_t* negs, uint64_t seed) {
  const int d = cfg->d, W = cfg->window, K = cfg->negative;
  const int64_t P = cfg->pitch;
  int32_t maxL = 0;
  for (int64_t s = 0; s < n_sent; s++)
    if (lens[s] > maxL) maxL = lens[s];
  float* cur = (float*)malloc(sizeof(float) * ((size_t)maxL + 1) * d);
  float* orig = (float*)malloc(sizeof(float) * ((size_t)maxL + 1) * d);
  float* o = (float*)malloc(sizeof(float) * d);
  float* o0 = (float*)malloc(sizeof(float) * d);
  int* ctx = (int*)malloc(sizeof(int) * (2 * W + 1));
  int rc = 0;
  for (int64_t s = 0; s < n_sent && rc == 0; s++) {
    const int L = lens[s];
    if (L <= 0) continue;
    const uint64_t skey = sr_sentence_key(seed, (uint64_t)s);
    const int32_t* sid = ids + starts[s];
    const int32_t* sneg = negs + starts[s] * K;
    for (int p = 0; p < L; p++)
      if (sid[p] < 0 || sid[p] >= V) rc = -3;
    for (int64_t q = 0; q < (int64_t)L * K; q++)
      if (sneg[q] < 0 || sneg[q] >= V) rc = -3;
    if (rc) break;
    int n_enter = W + 1 < L ? W + 1 : L;
    for (int p = 0; p < n_enter; p++)
      for (int e = 0; e < d; e++) cur[(int64_t)p * d + e] = orig[(int64_t)p * d + e] = bf16_f(syn0[(int64_t)sid[p] * P + e]);
    for (int w = 0; w < L; w++) {
      int n = context_list(w, W, L, ctx);
      if (n > 0) {
        for (int k = 0; k <= K; k++) {
          int32_t t = k == 0 ? sid[w] : sneg[(int64_t)w * K + k - 1];
          for (int e = 0; e < d; e++) o0[e] = o[e] = bf16_f(syn1[(int64_t)t * P + e]);
          for (int j = 0; j < n; j++) {
            float* v = cur + (int64_t)ctx[j] * d;
            float x = dot_f32(cfg, v, o);
            float g = grad_f32(cfg, x, k == 0, alphas[s]);
            for (int e = 0; e < d; e++) {
              float vo = v[e];
              v[e] = fmaf(g, o[e], vo);
              o[e] = fmaf(g, vo, o[e]);
            }
          }
          bf16_writeback(syn1 + (int64_t)t * P, o, o0, d, cfg->vec,
                         sr_event_key(skey, (uint64_t)w * (K + 1) + k), (uint64_t)t);
        }
      }
      if (w - W >= 0) {
        int p = w - W;
        bf16_writeback(syn0 + (int64_t)sid[p] * P, cur + (int64_t)p * d, orig + (int64_t)p * d, d, cfg->vec,
                       sr_event_key(skey, (uint64_t)L * (K + 1) + p), (uint64_t)sid[p]);
      }
      if (w + W + 1 < L) {
        int p = w + W + 1;
        for (int e = 0; e < d; e++) cur[(int64_t)p * d + e] = orig[(int64_t)p * d + e] = bf16_f(syn0[(int64_t)sid[p] * P + e]);
      }
    }
    for (int p = L - W > 0 ? L - W : 0; p < L; p++) {
      bf16_writeback(syn0 + (int64_t)sid[p] * P, cur + (int64_t)p * d, orig + (int64_t)p * d, d, cfg->vec,
                     sr_event_key(skey, (uint64_t)L * (K + 1) + p), (uint64_t)sid[p]);
    }
  }
  free(cur);
  free(orig);
  free(o);
  free(o0);
  free(ctx);
  return rc;
}

static double log_sigmoid(double x) {
  return x >= 0 ? -log1p(exp(-x)) : x - log1p(exp(x));
}

double orc_heldout_loss(const float* syn0, const float* syn1neg, int64_t pitch, int d, int window,
                        int negative, int64_t n_sent, const int64_t* starts, const int32_t* lens,
                        const int32_t* ids, const int32_t* negs, int64_t* pairs) {
  double total = 0.0;
  int64_t np = 0;
  int* ctx = (int*)malloc(sizeof(int) * (2 * window + 1));
  for (int64_t s = 0; s < n_sent; s++) {
    const int32_t* sid = ids + starts[s];
    const int32_t* sneg = negs + starts[s] * negative;
    int L = lens[s];
    for (int w = 0; w < L; w++) {
      int n = context_list(w, window, L, ctx);
      for (int j = 0; j < n; j++) {
        const float* v = syn0 + (int64_t)sid[ctx[j]] * pitch;
        for (int k = 0; k <= negative; k++) {
          int32_t t = k == 0 ? sid[w] : sneg[(int64_t)w * negative + k - 1];
          const float* o = syn1neg + (int64_t)t * pitch;
          double x = 0.0;
          for (int e = 0; e < d; e++) x += (double)v[e] * (double)o[e];
          total -= k == 0 ? log_sigmoid(x) : log_sigmoid(-x);
        }
        np++;
      }
    }
  }
  free(ctx);
  *pairs = np;
  return total;
}
