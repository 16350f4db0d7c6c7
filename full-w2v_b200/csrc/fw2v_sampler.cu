// On-device batch builder: the sentence / subsampling / negative-sampling loop
// of Train_SGNS (FULL-W2V-driver.cu:166-302).  Every reference "thread" is a
// sampling stream: a contiguous range of stored chunks (FULL-W2V-driver.cu:
// 103-110) and an LCG seeded with its id (:114) that persists across epochs.
//
// The LCG chain of a stream is inherently serial (a kept token advances it by
// 1+K steps, a dropped one by 1), but its decisions only depend on the low 16
// bits of the state, and the low 32 bits of an LCG mod 2^64 form an LCG mod
// 2^32 of their own.  So one warp runs a stream: the 32 lanes load 32 tokens
// and their keep thresholds at once, then walk them in order with a 32-bit
// state (one multiply-add per step, the K negatives' steps folded into one
// precomputed K-step map).  Each lane records the step at which its own token
// was kept; the full 64-bit state there follows from the state at the start of
// the 32-token block by one jump-ahead multiply-add (table of r -> A_m r + C_m).
// A second, fully parallel kernel turns each kept token's state into its K
// negative ids (FULL-W2V-driver.cu:224-227).
//
// Output of one epoch, per stream s (kept_base(s) = stream_base[s], the sum of
// the readable lengths of the chunks before the stream's range in chunk-table
// order; entry_base(s) = kept_base(s) + 2s):
//   entries  ent_{start,len,alpha}[entry_base(s) + e], e < n_entries[s]: every
//            batch entry the reference records, zero-length ones included
//   kept     kept_ids / kept_state[kept_base(s) + k], k < n_kept[s], and
//            kept_negs[(kept_base(s) + k) * K + j]
//   words[s] tokens read this epoch (EOS and subsampled-away tokens included).
#include "fw2v_common.cuh"

namespace fw2v {

namespace {

constexpr uint32_t kLcgMul32 = (uint32_t)kLcgMul;
constexpr uint32_t kLcgAdd32 = (uint32_t)kLcgAdd;

}  // namespace

// One stream's epoch: the chunks [es, ee) of the job's chunk table, kept ids
// from kept_base (at most kept_cap), entries from entry_b; the stream's
// carried state is at index `st` of p.lcg / wca_own / alpha, its counts at
// index `so` of p.n_entries / n_kept / words.
__device__ __forceinline__ void sample_stream(const SamplerParams& p, int64_t es, int64_t ee, int64_t kept_base,
                                              int64_t kept_cap, int64_t entry_b, int64_t st, int64_t so,
                                              int lane) {
  const int64_t entry_cap = kept_cap + 2;
  const int K = p.negative;
  const int msl = p.msl;
  const bool subsample = p.sample > 0.0f;
  const uint32_t aK = (uint32_t)p.jump_a[K];
  const uint32_t cK = (uint32_t)p.jump_c[K];

  uint64_t r_blk = p.lcg[st];  // full state at the start of the current block
  uint32_t r32 = (uint32_t)r_blk;
  uint64_t wca_own = p.wca_own[st];
  float alpha = p.alpha[st];
  uint64_t word_count = 0, last_word_count = 0;
  int64_t nk = 0, ne = 0;
  int L = 0;
  bool fail = false;

  // Record a batch entry of `len` kept words, then the learning-rate refresh the
  // reference performs before building the next sentence (FULL-W2V-driver.cu:168-190).
  auto record = [&](int len, bool refresh) {
    if (ne >= entry_cap) {
      fail = true;
      return;
    }
    if (lane == 0) {
      p.ent_start[entry_b + ne] = kept_base + nk;
      p.ent_len[entry_b + ne] = len;
      p.ent_alpha[entry_b + ne] = alpha;
    }
    ne++;
    nk += len;
    if (refresh && word_count - last_word_count > 10000) {
      wca_own += word_count - last_word_count;
      last_word_count = word_count;
      alpha = refreshed_alpha(p.alpha0, wca_own, p.threads, p.epochs, p.train_words);
    }
  };

  for (int64_t ss = es; ss < ee && !fail; ss++) {
    const int64_t off = p.chunk_off[ss];
    bool chunk_done = false;
    for (int cur0 = 0; cur0 < msl && !chunk_done && !fail; cur0 += 32) {
      // A chunk is read from its start until msl tokens or its first 0 (EOS).
      const int cur = cur0 + lane;
      const int64_t pos = off + cur;
      const bool inb = cur < msl && pos < p.stream_len;
      const int w = inb ? __ldg(p.stream + pos) : -1;
      const unsigned zmask = __ballot_sync(kFull, inb && w == 0);
      int nvalid = msl - cur0 < 32 ? msl - cur0 : 32;
      if (zmask) {
        const int z = __ffs(zmask);
        if (z < nvalid) nvalid = z;
      }
      const bool bad = lane < nvalid && (!inb || w < 0 || (int64_t)w >= p.vocab);
      if (__any_sync(kFull, bad)) {
        fail = true;
        break;
      }
      const int thr = (lane < nvalid && w > 0) ? __ldg(p.keep_thr + w) : 0;
      bool my_keep = false;
      int my_m = 0;
      int64_t my_slot = 0;
      int m = 0;  // LCG steps taken in this block
      for (int i = 0; i < nvalid; i++) {
        const int wi = __shfl_sync(kFull, w, i);
        const int ti = __shfl_sync(kFull, thr, i);
        word_count++;
        if (wi == 0) {
          // EOS ends the chunk; it ends the sentence unless it closes the
          // stream's range, where the partial sentence is dropped (:233-247).
          chunk_done = true;
          if (ss + 1 < ee) {
            record(L, true);
            L = 0;
          }
          break;
        }
        bool keep = true;
        if (subsample) {
          r32 = r32 * kLcgMul32 + kLcgAdd32;
          m++;
          keep = (int)(r32 & 0xFFFFu) <= ti;
        }
        if (keep) {
          if (lane == i) {
            my_keep = true;
            my_m = m;
            my_slot = nk + L;
          }
          r32 = r32 * aK + cK;
          m += K;
          L++;
          if (L == msl) {
            record(L, true);
            L = 0;
          }
        }
      }
      bool lfail = false;
      if (my_keep) {
        if (my_slot >= kept_cap) {
          lfail = true;
        } else {
          p.kept_ids[kept_base + my_slot] = w;
          p.kept_state[kept_base + my_slot] = p.jump_a[my_m] * r_blk + p.jump_c[my_m];
        }
      }
      fail |= __any_sync(kFull, lfail);
      r_blk = p.jump_a[m] * r_blk + p.jump_c[m];
    }
  }
  if (!fail) {
    // Epoch end (FULL-W2V-driver.cu:233-277): flush the count, drop the partial
    // sentence (recorded with length 0).
    wca_own += word_count - last_word_count;
    record(0, false);
  }
  if (fail) {
    if (lane == 0) atomicExch(p.error_flag, 1);
    ne = 0;
    nk = 0;
  }
  if (lane == 0) {
    p.lcg[st] = r_blk;
    p.wca_own[st] = wca_own;
    p.alpha[st] = alpha;
    p.n_entries[so] = ne;
    p.n_kept[so] = nk;
    p.words[so] = word_count;
  }
}

__global__ void __launch_bounds__(128) sampler_warp_kernel(SamplerParams p) {
  const int lane = threadIdx.x & 31;
  const int s = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (s >= p.threads) return;
  int64_t es, ee;
  stream_range(p.n_chunks, p.threads, s, &es, &ee);
  const int64_t kept_base = p.stream_base[s];
  sample_stream(p, es, ee, kept_base, p.stream_base[s + 1] - kept_base, entry_base(p.stream_base, s), s, s, lane);
}

// K negatives of every kept token from its LCG state: the reference draws them
// right after the token's keep decision, one LCG step each, and indexes the
// unigram table with (state >> 16) % table_size (FULL-W2V-driver.cu:224-227).
__device__ __forceinline__ void draw_negatives(const SamplerParams& p, int64_t slot) {
  uint64_t r = p.kept_state[slot];
  int32_t* out = p.kept_negs + slot * p.negative;
  for (int j = 0; j < p.negative; j++) {
    r = lcg_next(r);
    out[j] = unigram_pick(p, (int64_t)((r >> 16) % (uint64_t)p.table_size));
  }
}

__global__ void __launch_bounds__(256) negatives_kernel(SamplerParams p) {
  const int s = blockIdx.y;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p.threads || k >= p.n_kept[s]) return;
  draw_negatives(p, p.stream_base[s] + k);
}

// Exclusive prefix sum of n_entries over streams (one block), so that the
// trainer can map a global sentence number to (stream, entry).
__global__ void __launch_bounds__(1024) entry_prefix_kernel(const int64_t* n_entries, int threads,
                                                            int64_t* prefix) {
  __shared__ int64_t partial[1024];
  const int t = threadIdx.x;
  const int per = (threads + 1023) / 1024;
  const int lo = t * per;
  int64_t sum = 0;
  for (int i = lo; i < lo + per && i < threads; i++) sum += n_entries[i];
  partial[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int64_t v = t >= off ? partial[t - off] : 0;
    __syncthreads();
    partial[t] += v;
    __syncthreads();
  }
  int64_t run = t > 0 ? partial[t - 1] : 0;
  for (int i = lo; i < lo + per && i < threads; i++) {
    prefix[i] = run;
    run += n_entries[i];
  }
  if (t == 1023) prefix[threads] = partial[1023];
}

// Readable length of every stored chunk: its tokens up to msl or up to and
// including its first 0 (the reader stops there, FULL-W2V-driver.cu:196-212),
// clipped at the end of the stream.  One warp per chunk.
__global__ void __launch_bounds__(256) chunk_length_kernel(const int32_t* stream, int64_t stream_len,
                                                           const int64_t* chunk_off, int64_t n_chunks, int msl,
                                                           int64_t* len) {
  const int lane = threadIdx.x & 31;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (c >= n_chunks) return;
  const int64_t off = chunk_off[c];
  int n = msl;
  for (int cur0 = 0; cur0 < msl; cur0 += 32) {
    const int cur = cur0 + lane;
    const int64_t pos = off + cur;
    const bool inb = cur < msl && pos < stream_len;
    const unsigned end = __ballot_sync(kFull, !inb || stream[pos] == 0);
    if (end) {
      const int z = __ffs(end) - 1;  // first lane out of the stream or holding a 0
      const int64_t zpos = off + cur0 + z;
      n = cur0 + z + (zpos < stream_len ? 1 : 0);
      if (n > msl) n = msl;
      break;
    }
  }
  if (lane == 0) len[c] = n;
}

// In-place exclusive prefix sum of n int64 values followed by their total at
// index n (one block; the vectors here are chunk or stream counts).
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(int64_t* v, int64_t n) {
  __shared__ int64_t partial[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + 1023) / 1024;
  const int64_t lo = t * per;
  int64_t sum = 0;
  for (int64_t i = lo; i < lo + per && i < n; i++) sum += v[i];
  partial[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int64_t x = t >= off ? partial[t - off] : 0;
    __syncthreads();
    partial[t] += x;
    __syncthreads();
  }
  int64_t run = t > 0 ? partial[t - 1] : 0;
  for (int64_t i = lo; i < lo + per && i < n; i++) {
    const int64_t x = v[i];
    v[i] = run;
    run += x;
  }
  if (t == 1023) v[n] = partial[1023];
}

// stream_base[s] = chunk_base[first chunk of s]; stream_base[T] = total.
__global__ void stream_base_kernel(const int64_t* chunk_base, int64_t n_chunks, int threads, int64_t* stream_base) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s > threads) return;
  if (s == threads) {
    stream_base[s] = chunk_base[n_chunks];
    return;
  }
  int64_t first, end;
  stream_range(n_chunks, threads, s, &first, &end);
  stream_base[s] = chunk_base[first];
}

// ---- batched jobs: one launch over a round's (job, stream) list ----

// One warp per stream of the round; jobs past their epoch count record nothing.
__global__ void __launch_bounds__(128) sampler_batch_kernel(const SamplerParams* jobs, BatchRound r, int epoch) {
  __shared__ __align__(8) SamplerParams sp[4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= r.n) return;
  copy_params(&sp[warp], &jobs[r.job[g]], lane, 32);
  __syncwarp();
  const SamplerParams& p = sp[warp];
  if (epoch >= p.epochs) {
    if (lane == 0) {
      p.n_entries[g] = 0;
      p.n_kept[g] = 0;
      p.words[g] = 0;
    }
    return;
  }
  int64_t es, ee;
  stream_range(p.n_chunks, p.threads, r.local[g], &es, &ee);
  const int64_t kb = r.kbase[g];
  sample_stream(p, es, ee, kb, r.kbase[g + 1] - kb, kb + 2 * g, r.gstream[g], g, lane);
}

// blockIdx.y = stream of the round.
__global__ void __launch_bounds__(256) negatives_batch_kernel(const SamplerParams* jobs, BatchRound r) {
  __shared__ __align__(8) SamplerParams sp;
  const int g = blockIdx.y;
  copy_params(&sp, &jobs[r.job[g]], threadIdx.x, blockDim.x);
  __syncthreads();
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= sp.n_kept[g]) return;
  draw_negatives(sp, r.kbase[g] + k);
}

// One thread per job: the number of the job's first sentence in each of its
// round streams (its sentences are numbered in stream order over the epoch,
// as a single job's are), and the job's words read and kept.
__global__ void round_jobs_kernel(BatchRound r, const int64_t* n_entries, const int64_t* n_kept,
                                  const uint64_t* words, int n_jobs, int64_t* job_uid, int64_t* uid_base,
                                  unsigned long long* job_words, unsigned long long* job_kept) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_jobs) return;
  int64_t run = job_uid[j];
  unsigned long long w = 0, k = 0;
  for (int g = 0; g < r.n; g++) {
    if (r.job[g] != j) continue;
    uid_base[g] = run;
    run += n_entries[g];
    w += words[g];
    k += (unsigned long long)n_kept[g];
  }
  job_uid[j] = run;
  job_words[j] += w;
  job_kept[j] += k;
}

cudaError_t launch_sampler_round(const SamplerParams* d_jobs, const BatchRound& r, int epoch, int64_t max_region,
                                 bool any_negatives, const int64_t* n_entries, const int64_t* n_kept,
                                 const uint64_t* words, int n_jobs, int64_t* job_uid, int64_t* uid_base,
                                 unsigned long long* job_words, unsigned long long* job_kept,
                                 int64_t* entry_prefix, cudaStream_t st) {
  if (r.n < 1 || r.n > 65535) return cudaErrorInvalidValue;
  sampler_batch_kernel<<<(r.n + 3) / 4, 128, 0, st>>>(d_jobs, r, epoch);
  if (any_negatives && max_region > 0) {
    const dim3 grid((unsigned)((max_region + 255) / 256), (unsigned)r.n);
    negatives_batch_kernel<<<grid, 256, 0, st>>>(d_jobs, r);
  }
  entry_prefix_kernel<<<1, 1024, 0, st>>>(n_entries, r.n, entry_prefix);
  round_jobs_kernel<<<(n_jobs + 127) / 128, 128, 0, st>>>(r, n_entries, n_kept, words, n_jobs, job_uid, uid_base,
                                                        job_words, job_kept);
  return cudaGetLastError();
}

cudaError_t launch_corpus_layout(const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                                 int64_t n_chunks, int msl, int threads, int64_t* chunk_base,
                                 int64_t* stream_base, cudaStream_t st) {
  chunk_length_kernel<<<(unsigned)((n_chunks * 32 + 255) / 256), 256, 0, st>>>(stream, stream_len, chunk_off,
                                                                             n_chunks, msl, chunk_base);
  exclusive_scan_kernel<<<1, 1024, 0, st>>>(chunk_base, n_chunks);
  stream_base_kernel<<<(threads + 1 + 255) / 256, 256, 0, st>>>(chunk_base, n_chunks, threads, stream_base);
  return cudaGetLastError();
}

cudaError_t launch_sampler(const SamplerParams& p, int64_t max_region, int64_t* entry_prefix,
                           cudaStream_t st) {
  const int warps_per_block = 4;
  const int grid = (p.threads + warps_per_block - 1) / warps_per_block;
  sampler_warp_kernel<<<grid, warps_per_block * 32, 0, st>>>(p);
  if (p.negative > 0) {
    const dim3 ngrid((unsigned)((max_region + 255) / 256), (unsigned)p.threads);
    negatives_kernel<<<ngrid, 256, 0, st>>>(p);
  }
  entry_prefix_kernel<<<1, 1024, 0, st>>>(p.n_entries, p.threads, entry_prefix);
  return cudaGetLastError();
}

}  // namespace fw2v
