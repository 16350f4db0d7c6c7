// InitNet on the device (improved_driver_functions.cpp:1-83): syn0 from the
// LCG, the subsampling thresholds and the 1e8-entry unigram table.  The
// 1000-entry sigmoid table is built on the host (fw2v_exp_table) because the
// reference's values come from the host libm's expf.
//
// The unigram table's run boundaries are computed on the host in double
// precision with the reference's sequential power sum and running share (the
// values depend on libm's pow, which the reference calls on the host), then the
// table itself is filled on the device.  The boundary walk visits one table
// index per word instead of all 1e8, and evaluates the reference's predicate
// (a / 1e8 > running share) at the same indices with the same doubles, so the
// table is identical to the reference's sequential fill.
#include <cmath>
#include <vector>

#include "fw2v_common.cuh"

namespace fw2v {

// improved_driver_functions.cpp:27-31; element i = row*d + c uses the
// (i+1)-th LCG state from `start` (1 in the reference).  One thread per row,
// started by jump-ahead.  Bfloat16 tables take the FP32 value rounded to nearest.
template <typename T>
__global__ void init_syn0_kernel(T* syn0, int64_t V, int d, int64_t pitch, uint64_t start) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= V) return;
  const Affine j = lcg_jump((uint64_t)row * (uint64_t)d);
  uint64_t r = j.a * start + j.c;  // state after row*d steps from `start`
  T* out = syn0 + row * pitch;
  const float fd = (float)d;
  for (int c = 0; c < d; c++) {
    r = lcg_next(r);
    const float u = __uint2float_rn((unsigned)(r & 0xFFFF)) / 65536.0f;
    const float x = __fdiv_rn(__fsub_rn(u, 0.5f), fd);
    if constexpr (sizeof(T) == 4) out[c] = x;
    else out[c] = bf16_nearest(x);
  }
}

// improved_driver_functions.cpp:71-77, as an integer threshold: the reference
// drops a token iff p < u/65536 (FULL-W2V-driver.cu:218), u = lcg & 0xFFFF;
// p*65536 is exact in float, so it keeps iff u <= floor(p*65536).
__global__ void subsample_kernel(const uint32_t* counts, int64_t V, float sample, uint64_t train_words,
                                 int32_t* keep_thr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const float base = __fmul_rn(sample, __ull2float_rn(train_words));
  const float ratio = __fdiv_rn(base, __uint2float_rn(counts[i]));
  const float pk = __fadd_rn(__fsqrt_rn(ratio), ratio);
  const float scaled = __fmul_rn(pk, 65536.0f);
  keep_thr[i] = (isnan(pk) || scaled >= 65535.0f) ? 65535 : (int32_t)floorf(scaled);
}

// firsts[j] = first table index of word j+1 (j < n), non-decreasing.
__global__ void unigram_fill_kernel(const int64_t* firsts, int n, int32_t* table, int64_t size) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < size; a += stride) {
    int lo = 0, hi = n - 1;  // last j with firsts[j] <= a (firsts[0] == 0)
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(firsts + mid) <= a) lo = mid;
      else hi = mid - 1;
    }
    table[a] = lo + 1;
  }
}

}  // namespace fw2v

// generate_expTable_h.cpp:46-55: float expf on the host, first entry 0, last 1.
extern "C" void fw2v_exp_table(float* t) {
  for (int i = 0; i < fw2v::kExpTableSize; i++) {
    float x = ((float)i / (float)fw2v::kExpTableSize * 2.0f - 1.0f) * 6.0f;
    float val = std::exp(x);
    val = val / (val + 1.0f);
    if (i == 0) val = 0.0f;
    if (i + 1 == fw2v::kExpTableSize) val = 1.0f;
    t[i] = val;
  }
}

// Host: first table index of every word 1..V-1 (words never reached get
// `size`).  firsts must hold V-1 entries.  Returns 0, or -1 if V < 2.
extern "C" int fw2v_unigram_firsts(const uint32_t* counts, int64_t V, int64_t size, int64_t* firsts) {
  if (V < 2) return -1;
  double total = 0.0;
  for (int64_t i = 0; i < V; i++) total += std::pow((double)counts[i], 0.75);
  const double dsize = (double)size;
  auto pred = [&](int64_t a, double d1) { return (double)a / dsize > d1; };
  double d1 = std::pow((double)counts[0], 0.75) / total;
  int64_t word = 1;
  int64_t a = 0;
  firsts[0] = 0;
  for (int64_t j = 1; j < V - 1; j++) firsts[j] = size;
  while (a < size && word < V - 1) {
    // smallest x >= a with x / size > d1: entries [a, x] hold `word`, and the
    // fill moves to the next word right after x (one step per entry at most).
    double guess = std::floor(d1 * dsize);
    int64_t x = guess < (double)a ? a : (guess > dsize ? size : (int64_t)guess);
    while (x > a && pred(x - 1, d1)) x--;
    while (x < size && !pred(x, d1)) x++;
    if (x >= size) break;
    word++;
    if (x + 1 < size) firsts[word - 1] = x + 1;
    d1 += std::pow((double)counts[word], 0.75) / total;
    a = x + 1;
  }
  return 0;
}

namespace fw2v {

cudaError_t launch_init_tables(void* syn0, bool bf16, int64_t V, int d, int64_t pitch, const uint32_t* d_counts,
                               float sample, uint64_t train_words, int32_t* keep_thr,
                               const int64_t* d_firsts, int n_firsts, int32_t* unigram,
                               int64_t table_size, uint64_t start, cudaStream_t st) {
  const int b = 256;
  if (bf16) init_syn0_kernel<<<(unsigned)((V + b - 1) / b), b, 0, st>>>((uint16_t*)syn0, V, d, pitch, start);
  else init_syn0_kernel<<<(unsigned)((V + b - 1) / b), b, 0, st>>>((float*)syn0, V, d, pitch, start);
  subsample_kernel<<<(unsigned)((V + b - 1) / b), b, 0, st>>>(d_counts, V, sample, train_words, keep_thr);
  if (unigram) unigram_fill_kernel<<<148 * 16, 256, 0, st>>>(d_firsts, n_firsts, unigram, table_size);
  return cudaGetLastError();
}

}  // namespace fw2v

namespace fw2v {

__global__ void validate_ids_kernel(const int32_t* ids, int64_t n, int64_t vocab, int* flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t t = __ldg(ids + i);
    bad |= t < 0 || (int64_t)t >= vocab;
  }
  if (bad) atomicExch(flag, 1);
}

cudaError_t launch_validate_ids(const int32_t* ids, int64_t n, int64_t vocab, int* flag, cudaStream_t st) {
  validate_ids_kernel<<<148 * 8, 256, 0, st>>>(ids, n, vocab, flag);
  return cudaGetLastError();
}

// A device-resident corpus: the stream ends with the 0 after its last word and
// every chunk starts inside it (the checks fw2v_load_corpus makes on the host).
__global__ void check_corpus_kernel(const int32_t* stream, int64_t len, const int64_t* chunk_off, int64_t n,
                                    int* flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = t == 0 && stream[len - 1] != 0;
  for (int64_t i = t; i < n; i += stride) {
    const int64_t o = chunk_off[i];
    bad |= o < 0 || o >= len;
  }
  if (bad) atomicExch(flag, 1);
}

// Seeded Fisher-Yates over n chunk offsets, on the device: for i = n-1 down
// to 1, j = the high 64 bits of mix64(key ^ mix64(i)) * (i + 1), swap a[i]
// and a[j].  The draws do not depend on the array, and the swaps are applied
// in order by one thread, on a copy in shared memory when the array fits
// there (use_smem), in place otherwise.
__global__ void fisher_yates_kernel(int64_t* a, int64_t n, uint64_t key, int use_smem) {
  extern __shared__ int64_t sa[];
  if (use_smem) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) sa[i] = a[i];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int64_t* x = use_smem ? sa : a;
    for (int64_t i = n - 1; i > 0; i--) {
      const int64_t j = (int64_t)__umul64hi(mix64(key ^ mix64((uint64_t)i)), (uint64_t)(i + 1));
      const int64_t t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  if (use_smem) {
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) a[i] = sa[i];
  }
}

cudaError_t launch_fisher_yates(int64_t* a, int64_t n, uint64_t key, cudaStream_t st) {
  if (n < 2) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  const size_t bytes = (size_t)n * sizeof(int64_t);
  const int use_smem = bytes <= (size_t)optin;
  if (use_smem) {
    e = cudaFuncSetAttribute(fisher_yates_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
  }
  fisher_yates_kernel<<<1, 1024, use_smem ? bytes : 0, st>>>(a, n, key, use_smem);
  return cudaGetLastError();
}

cudaError_t launch_check_corpus(const int32_t* stream, int64_t len, const int64_t* chunk_off, int64_t n, int* flag,
                                cudaStream_t st) {
  check_corpus_kernel<<<148 * 2, 256, 0, st>>>(stream, len, chunk_off, n, flag);
  return cudaGetLastError();
}

}  // namespace fw2v
