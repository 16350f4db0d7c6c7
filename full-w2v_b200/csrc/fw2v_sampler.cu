// On-device batch builder: the sentence/subsampling/negative-sampling loop of
// Train_SGNS (FULL-W2V-driver.cu:166-302), one CUDA thread per reference
// "thread" (LCG stream).  Every stream owns a contiguous range of stored
// chunks (FULL-W2V-driver.cu:103-110), an LCG seeded with its id (:114) that
// persists across epochs, and its own learning-rate state.
//
// Output of one epoch, per stream s:
//   entries  ent_{start,len,alpha}[entry_base(s) + e], e < n_entries[s]
//            (every batch entry the reference records, zero-length ones too)
//   kept ids kept_ids[kept_base(s) + k], k < n_kept[s], and K negatives each
//            at kept_negs[(kept_base(s) + k) * K + j]
//   words[s] tokens read this epoch (EOS and subsampled-away tokens included).
// kept_base(s) = chunk_off[first chunk of s]; entry_base(s) = kept_base(s) + 2s.
// Capacities follow from the region of stream s in the token stream; a stream
// that would overflow them (possible only with chunk tables whose chunks are
// shorter than msl without a closing 0) stops and raises the error flag.
#include "fw2v_common.cuh"

namespace fw2v {

__global__ void __launch_bounds__(128) sampler_epoch_kernel(SamplerParams p) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p.threads) return;
  int64_t es, ee;
  stream_range(p.n_chunks, p.threads, s, &es, &ee);
  const int64_t kept_base = p.chunk_off[es];
  const int64_t region_end = ee < p.n_chunks ? p.chunk_off[ee] : p.stream_len;
  const int64_t kept_cap = region_end - kept_base;
  const int64_t entry_b = kept_base + 2 * (int64_t)s;
  const int64_t entry_cap = kept_cap + 2;
  const int K = p.negative;
  const int msl = p.msl;

  uint64_t lcg = p.lcg[s];
  uint64_t wca_own = p.wca_own[s];
  float alpha = p.alpha[s];
  uint64_t word_count = 0, last_word_count = 0;
  int64_t ss = es, cur = 0;
  int64_t ne = 0, nk = 0;
  bool fail = false;

  for (;;) {
    if (word_count - last_word_count > 10000) {
      wca_own += word_count - last_word_count;
      last_word_count = word_count;
      alpha = refreshed_alpha(p.alpha0, wca_own, p.threads, p.epochs, p.train_words);
    }
    int32_t L = 0;
    while (L < msl) {
      if (cur >= msl) {
        ss++;
        cur = 0;
        if (ss >= ee) break;
      }
      const int64_t pos = p.chunk_off[ss] + cur;
      if (pos >= p.stream_len) {
        fail = true;
        break;
      }
      const int32_t w = __ldg(p.stream + pos);
      cur++;
      word_count++;
      if (w == 0 || ss >= ee) {
        ss++;
        cur = 0;
        break;
      }
      if (p.sample > 0.0f) {
        lcg = lcg_next(lcg);
        const float u = __uint2float_rn((unsigned)(lcg & 0xFFFF)) / 65536.0f;
        if (__ldg(p.p_keep + w) < u) continue;
      }
      if (nk + L >= kept_cap) {
        fail = true;
        break;
      }
      const int64_t slot = kept_base + nk + L;
      p.kept_ids[slot] = w;
      for (int k = 0; k < K; k++) {
        lcg = lcg_next(lcg);
        const int64_t idx = (int64_t)((lcg >> 16) % (uint64_t)p.table_size);
        p.kept_negs[slot * K + k] = __ldg(p.unigram + idx);
      }
      L++;
    }
    if (fail || ne >= entry_cap) {
      fail = true;
      break;
    }
    const int64_t e = entry_b + ne;
    if (ss >= ee) {
      // Epoch end (FULL-W2V-driver.cu:233-277): flush the count, drop the
      // partial sentence (recorded with length 0).
      wca_own += word_count - last_word_count;
      p.ent_start[e] = kept_base + nk;
      p.ent_len[e] = 0;
      p.ent_alpha[e] = alpha;
      ne++;
      break;
    }
    p.ent_start[e] = kept_base + nk;
    p.ent_len[e] = L;
    p.ent_alpha[e] = alpha;
    ne++;
    nk += L;
  }
  if (fail) {
    atomicExch(p.error_flag, 1);
    ne = 0;
    nk = 0;
  }
  p.lcg[s] = lcg;
  p.wca_own[s] = wca_own;
  p.alpha[s] = alpha;
  p.n_entries[s] = ne;
  p.n_kept[s] = nk;
  p.words[s] = word_count;
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

cudaError_t launch_sampler(const SamplerParams& p, int64_t* entry_prefix, cudaStream_t st) {
  const int block = 128;
  const int grid = (p.threads + block - 1) / block;
  sampler_epoch_kernel<<<grid, block, 0, st>>>(p);
  entry_prefix_kernel<<<1, 1024, 0, st>>>(p.n_entries, p.threads, entry_prefix);
  return cudaGetLastError();
}

}  // namespace fw2v
