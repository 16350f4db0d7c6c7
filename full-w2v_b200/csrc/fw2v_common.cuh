// Shared device helpers of libfw2v: the word2vec LCG with jump-ahead, the
// per-lane row layout used by the training kernel, and the parameter blocks
// the kernels take.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace fw2v {

constexpr uint64_t kLcgMul = 25214903917ULL;  // FULL-W2V-driver.cu:217
constexpr uint64_t kLcgAdd = 11ULL;
constexpr int64_t kUnigramTableSize = 100000000LL;  // FULL-W2V-driver.cu:61
constexpr int kExpTableSize = 1000;                 // FULL-W2V-driver.cu:17
constexpr int kMaxWindow = 15;                      // ring of 2W+1 <= 32 slots, one per lane
constexpr int kMaxNegative = 31;
constexpr int kWarpsPerBlock = 4;
constexpr unsigned kFull = 0xffffffffu;

__host__ __device__ __forceinline__ uint64_t lcg_next(uint64_t r) { return r * kLcgMul + kLcgAdd; }

// r -> a*r + c, the LCG applied n times (all arithmetic mod 2^64).
struct Affine {
  uint64_t a, c;
};

__host__ __device__ __forceinline__ Affine lcg_jump(uint64_t n) {
  Affine res{1, 0};
  Affine base{kLcgMul, kLcgAdd};
  while (n) {
    if (n & 1) res = Affine{base.a * res.a, base.a * res.c + base.c};
    base = Affine{base.a * base.a, base.a * base.c + base.c};
    n >>= 1;
  }
  return res;
}

// Counter-based random bits for stochastic rounding.  A training launch
// (seed) and a sentence (uid) give a 64-bit sentence key, once per sentence;
// an event within the sentence (a target row's or a leaving context row's
// write-back) and each vector of the row then draw their bits with 32-bit
// multiply-xorshift steps: 32 bits per vector of 2 elements, 64 per vector of
// 4, 16 per element.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
// Offset of every LCG start state and stochastic-rounding seed for a
// configuration's seed (0 for seed 0: the reference's seeds).
__host__ __device__ __forceinline__ uint64_t seed_offset(uint64_t seed) { return seed ? mix64(seed) : 0; }
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}
__host__ __device__ __forceinline__ uint64_t sr_sentence_key(uint64_t seed, uint64_t uid) {
  return mix64(seed ^ mix64(uid * 0x9E3779B97F4A7C15ULL));
}
// Key of event `event` of a sentence: the low word mixed with the event number.
__host__ __device__ __forceinline__ uint64_t sr_event_key(uint64_t skey, uint64_t event) {
  return (skey & 0xFFFFFFFF00000000ULL) | (uint32_t)((uint32_t)skey ^ fmix32((uint32_t)event * 0x9E3779B9u + 1u));
}
__host__ __device__ __forceinline__ uint64_t sr_vector_bits(uint64_t key, uint64_t row, uint64_t vec) {
  const uint32_t lo = fmix32((uint32_t)key ^ ((uint32_t)row * 0x27D4EB2Fu) ^ ((uint32_t)vec * 0x165667B1u));
  uint32_t hi = (lo ^ (uint32_t)(key >> 32)) * 0x9E3779B9u;
  hi ^= hi >> 15;
  return ((uint64_t)hi << 32) | lo;
}
// x (finite) rounded to bfloat16 up or down in magnitude with probability
// equal to its distance from the truncated value, widened back to float: 16
// random bits r16 (uniform in [0, 65536)) carry into the kept bits and the 16
// discarded bits are cleared.
__device__ __forceinline__ float bf16_stochastic_value(float x, uint32_t r16) {
  return __uint_as_float((__float_as_uint(x) + r16) & 0xFFFF0000u);
}
__host__ __device__ __forceinline__ float bf16_value(uint16_t h) {
  const uint32_t b = (uint32_t)h << 16;
  float x;
  memcpy(&x, &b, 4);
  return x;
}
// Round to nearest even (table initialisation and host conversions).
__host__ __device__ __forceinline__ uint16_t bf16_nearest(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  if ((b & 0x7F800000u) == 0x7F800000u) return (uint16_t)((b >> 16) | ((b & 0x007FFFFFu) ? 0x40 : 0));
  return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
}

// Learning-rate refresh (FULL-W2V-driver.cu:188-189) with the global word count
// taken as T x this stream's own flushed count.
__host__ __device__ __forceinline__ float refreshed_alpha(float alpha0, uint64_t wca_own, int threads,
                                                          int epochs, uint64_t train_words) {
  uint64_t global = (uint64_t)threads * wca_own;
  float denom = (float)((uint64_t)epochs * train_words + 1);
#ifdef __CUDA_ARCH__
  float a = __fmul_rn(alpha0, __fsub_rn(1.0f, __fdiv_rn(__ull2float_rn(global), denom)));
  float floor_a = __fmul_rn(alpha0, 0.0001f);
#else
  float a = alpha0 * (1 - (float)global / denom);
  float floor_a = alpha0 * 0.0001f;
#endif
  return a < floor_a ? floor_a : a;
}

// ---------------------------------------------------------------------------
// Sampler: one reference "thread" (an LCG stream over a contiguous chunk range)
// ---------------------------------------------------------------------------
struct SamplerParams {
  const int32_t* stream;
  int64_t stream_len;
  const int64_t* chunk_off;
  int64_t n_chunks;
  const int64_t* stream_base;  // threads + 1: where each stream's kept ids start
  int64_t vocab;
  const int32_t* keep_thr;  // keep a token iff (lcg & 0xFFFF) <= keep_thr[word]
  float sample;
  const int32_t* unigram;         // the table, or null: search unigram_firsts
  const int64_t* unigram_firsts;  // first table index of words 1..n_firsts (non-decreasing)
  int64_t n_firsts;
  int64_t table_size;
  const uint64_t* jump_a;   // r -> jump_a[m] * r + jump_c[m] is m LCG steps
  const uint64_t* jump_c;
  int threads, msl, negative, epochs;
  float alpha0;
  uint64_t train_words;
  // state carried across epochs, one per stream
  uint64_t* lcg;
  uint64_t* wca_own;
  float* alpha;
  // outputs; entries of stream s start at entry_base(s), kept ids at kept_base(s)
  int64_t* ent_start;
  int32_t* ent_len;
  float* ent_alpha;
  int32_t* kept_ids;
  uint64_t* kept_state;     // LCG state after a kept token's keep decision
  int32_t* kept_negs;
  int64_t* n_entries;
  int64_t* n_kept;
  uint64_t* words;
  int* error_flag;
};

// Unigram table entry `a` (FULL-W2V-driver.cu:224-227): the table itself, or
// the same value from the run boundaries: the word whose run [firsts[j],
// firsts[j+1]) holds a is j+1 (the search the table fill uses).
__device__ __forceinline__ int32_t unigram_pick(const SamplerParams& p, int64_t a) {
  if (p.unigram) return __ldg(p.unigram + a);
  int64_t lo = 0, hi = p.n_firsts - 1;  // last j with firsts[j] <= a (firsts[0] == 0)
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(p.unigram_firsts + mid) <= a) lo = mid;
    else hi = mid - 1;
  }
  return (int32_t)(lo + 1);
}

__host__ __device__ __forceinline__ void stream_range(int64_t n_chunks, int threads, int s,
                                                      int64_t* first, int64_t* end) {
  int64_t per = n_chunks / threads, left = n_chunks % threads;
  int64_t ss = (int64_t)s;
  *first = ss * per + (ss < left ? ss : left);
  *end = *first + per + (ss < left ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Trainer
// ---------------------------------------------------------------------------
enum SentenceSource : int {
  kSourceEpoch = 0,     // entries written by the sampler, indexed through entry_prefix
  kSourceExplicit = 1,  // starts / lens / alphas arrays
  kSourceBlocks = 2     // reference batch layout: sentence b at b*msl
};

struct TrainParams {
  void* syn0;     // float or bfloat16 (uint16) rows, by the kernel's element type
  void* syn1neg;
  int64_t pitch;  // elements per row, also the float stride of shared-memory rows
  int64_t vocab;
  int d, window, negative, sigmoid;
  const int32_t* ids;
  const int32_t* negs;
  int source;
  // kSourceEpoch
  const int64_t* entry_prefix;  // threads + 1
  const int64_t* stream_base;   // threads + 1
  int threads;
  const int64_t* ent_start;
  const int32_t* ent_len;
  const float* ent_alpha;
  // kSourceExplicit
  const int64_t* starts;
  const int32_t* lens;
  const float* alphas;
  int64_t n_sentences;
  // kSourceBlocks
  int msl;
  unsigned long long* work_counter;
  int deterministic;
  int* error_flag;
  const float* exp_table;
  // per-warp scratch, (2W+1) * pitch elements for each of scratch_warps warps:
  // the value every ring row had when it entered the window
  void* orig_scratch;
  int64_t scratch_warps;
  uint64_t sr_seed;  // stochastic rounding of bfloat16 write-backs
  int bf16;          // tables hold bfloat16
  int prefetch;      // copy each group's target rows while the previous group trains
  int bulk;          // stage the entering and leaving context rows by bulk copies
  // batched launches: lane vector width (2 or 4), vectors per lane (1 to 3)
  // and pipeline stages of this job's sentences
  int lane_vec, lane_nv, stages;
};

// A round of a batched epoch: n sampling streams of any jobs.  Stream g of the
// round is stream local[g] of job job[g], whose carried state is at index
// gstream[g] of the batch's state arrays; its kept ids start at kbase[g] and
// its entries at kbase[g] + 2g of the round's buffers (kbase has n + 1 entries).
struct BatchRound {
  const int32_t* job;
  const int32_t* local;
  const int64_t* gstream;
  const int64_t* kbase;
  int n;
};

// A parameter block copied into shared memory by the lanes t = 0..n-1 of a
// warp or block, one 32-bit word each, so that per-job parameters read from
// there in a kernel's inner loops (global stores cannot alias them).
template <typename P>
__device__ __forceinline__ void copy_params(P* dst, const P* src, int t, int n) {
  static_assert(sizeof(P) % 4 == 0, "parameter blocks are word-sized");
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  for (int i = t; i < (int)(sizeof(P) / 4); i += n) d[i] = s[i];
}

// Sampler output layout: stream s keeps its kept ids at [stream_base[s],
// stream_base[s+1]) and its batch entries from stream_base[s] + 2s (one more
// entry than kept ids at most, plus the epoch-end entry).
__host__ __device__ __forceinline__ int64_t entry_base(const int64_t* stream_base, int s) {
  return stream_base[s] + 2 * (int64_t)s;
}

}  // namespace fw2v
