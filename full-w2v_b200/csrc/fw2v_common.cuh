// Shared device helpers of libfw2v: the word2vec LCG with jump-ahead, the
// per-lane row layout used by the training kernel, and the parameter blocks
// the kernels take.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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
  const int32_t* unigram;
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
  float* syn0;
  float* syn1neg;
  int64_t pitch;  // floats per row
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
  // per-warp scratch, (2W+1) * pitch floats for each of scratch_warps warps:
  // the value every ring row had when it entered the window
  float* orig_scratch;
  int64_t scratch_warps;
};

// Sampler output layout: stream s keeps its kept ids at [stream_base[s],
// stream_base[s+1]) and its batch entries from stream_base[s] + 2s (one more
// entry than kept ids at most, plus the epoch-end entry).
__host__ __device__ __forceinline__ int64_t entry_base(const int64_t* stream_base, int s) {
  return stream_base[s] + 2 * (int64_t)s;
}

}  // namespace fw2v
