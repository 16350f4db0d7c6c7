// Nearest neighbours by cosine similarity among rows of an embedding table:
// the evaluator behind same-label precision@10 (the reference scores its
// vectors with word-similarity sets offline, analysis/hyperwords; here the
// planted topics or blocks of the synthetic corpora are the labels).
//
// For each query (an index into a candidate list of table rows) the k most
// similar other candidates, most similar first.  Ranking is by
// <q, c> / |c| in FP32 (the query's own norm does not change its ranking);
// the reported similarity is the cosine <q, c> / (|q| |c|).  Ties go to the
// lower candidate index.
//
// Kernels:
//   inv_norm_kernel    one warp per candidate: 1 / |c|, FP32 (and the query
//                      norms through the same list)
//   neighbours_kernel  a block takes QB queries and one slice of the
//                      candidates; each warp streams candidate rows (lane l
//                      holds elements l + 32 i, coalesced), multiplies each
//                      by the QB query rows held in registers and reduces the
//                      QB dot products together with a transposing shuffle
//                      tree; the lane that ends with a query's sum keeps that
//                      query's running top-k in shared memory (a fast reject
//                      against the k-th best first).  The warps' lists are
//                      merged into the slice's top-k.
//   merge_kernel       one warp per query merges the slices' lists.
// All arithmetic is CUDA-core FP32: the work is a few hundred thousand rows
// times a few thousand queries, and the ranking must not move under a
// reduced-precision product.
#include <cuda_bf16.h>

#include <cfloat>

#include "../../include/fw2v.h"
#include "fw2v_common.cuh"

namespace fw2v {
namespace {

constexpr int kQB = 8;        // queries per block
constexpr int kNbrWarps = 8;  // warps per block
constexpr int kMaxK = 32;

template <typename T>
__device__ __forceinline__ float elem(const T* row, int e);
template <>
__device__ __forceinline__ float elem<float>(const float* row, int e) {
  return __ldg(row + e);
}
template <>
__device__ __forceinline__ float elem<uint16_t>(const uint16_t* row, int e) {
  return bf16_value(__ldg(row + e));
}

// (sim, idx) ranks above (s2, i2): larger similarity, then lower index.
__device__ __forceinline__ bool better(float s, int i, float s2, int i2) { return s > s2 || (s == s2 && i < i2); }

template <typename T>
__global__ void inv_norm_kernel(const T* table, int64_t pitch, int d, const int32_t* cand, int64_t n,
                                float* inv) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = w; c < n; c += nw) {
    const T* row = table + (int64_t)cand[c] * pitch;
    float s = 0.0f;
    for (int e = lane; e < d; e += 32) {
      const float x = elem(row, e);
      s = __fmaf_rn(x, x, s);
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(kFull, s, m);
    if (lane == 0) inv[c] = s > 0.0f ? 1.0f / sqrtf(s) : 0.0f;
  }
}

// Lane l of a warp ends the transposing reduction of kQB values with the sum
// of value ((l >> 4) & 1) * 4 + ((l >> 3) & 1) * 2 + ((l >> 2) & 1).
__device__ __forceinline__ int query_of_lane(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

__device__ __forceinline__ float reduce8(float (&a)[kQB], int lane) {
  {
    const bool hi = lane & 16;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float send = hi ? a[j] : a[j + 4];
      const float keep = hi ? a[j + 4] : a[j];
      a[j] = keep + __shfl_xor_sync(kFull, send, 16);
    }
  }
  {
    const bool hi = lane & 8;
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const float send = hi ? a[j] : a[j + 2];
      const float keep = hi ? a[j + 2] : a[j];
      a[j] = keep + __shfl_xor_sync(kFull, send, 8);
    }
  }
  const bool hi = lane & 4;
  const float send = hi ? a[0] : a[1];
  const float keep = hi ? a[1] : a[0];
  float r = keep + __shfl_xor_sync(kFull, send, 4);
  r += __shfl_xor_sync(kFull, r, 2);
  r += __shfl_xor_sync(kFull, r, 1);
  return r;
}

// The best (s, i) over the warp, and the lane it came from, on every lane.
__device__ __forceinline__ void warp_best(float& s, int& i, int& src) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) {
    const float os = __shfl_xor_sync(kFull, s, m);
    const int oi = __shfl_xor_sync(kFull, i, m);
    const int osrc = __shfl_xor_sync(kFull, src, m);
    if (better(os, oi, s, i) || (os == s && oi == i && osrc < src)) {
      s = os;
      i = oi;
      src = osrc;
    }
  }
}

// Insert (s, i) into a descending list of k entries (the caller checked that
// it beats the last one).
__device__ __forceinline__ void list_insert(float* ls, int* li, int k, float s, int i) {
  int p = k - 1;
  while (p > 0 && better(s, i, ls[p - 1], li[p - 1])) {
    ls[p] = ls[p - 1];
    li[p] = li[p - 1];
    p--;
  }
  ls[p] = s;
  li[p] = i;
}

// NE: elements per lane (rows of up to 32 * NE elements).
template <typename T, int NE>
__global__ void __launch_bounds__(kNbrWarps * 32) neighbours_kernel(const T* table, int64_t pitch, int d,
                                                                  const int32_t* cand, int64_t n_cand,
                                                                  const float* inv, const int32_t* queries,
                                                                  int64_t n_q, int k, int64_t slice,
                                                                  float* part_s, int32_t* part_i) {
  __shared__ float ls[kNbrWarps][kQB][kMaxK];
  __shared__ int li[kNbrWarps][kQB][kMaxK];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t q0 = (int64_t)blockIdx.x * kQB;
  const int64_t c_begin = (int64_t)blockIdx.y * slice;
  const int64_t c_end = c_begin + slice < n_cand ? c_begin + slice : n_cand;
  // the block's query rows, in registers (zero past d and past the last query)
  float qv[kQB][NE];
  int qself[kQB];
#pragma unroll
  for (int j = 0; j < kQB; j++) {
    const bool real = q0 + j < n_q;
    qself[j] = real ? queries[q0 + j] : -1;
    const T* row = table + (real ? (int64_t)cand[qself[j]] * pitch : 0);
#pragma unroll
    for (int i = 0; i < NE; i++) {
      const int e = lane + 32 * i;
      qv[j][i] = real && e < d ? elem(row, e) : 0.0f;
    }
  }
  for (int t = lane; t < kQB * kMaxK; t += 32) {
    ls[warp][t / kMaxK][t % kMaxK] = -FLT_MAX;
    li[warp][t / kMaxK][t % kMaxK] = INT32_MAX;
  }
  __syncwarp();
  const int myq = query_of_lane(lane);
  const bool leader = (lane & 3) == 0;
  int my_self = -1;  // the leader's query's own candidate, never its neighbour
#pragma unroll
  for (int j = 0; j < kQB; j++)
    if (j == myq) my_self = qself[j];
  float thr_s = -FLT_MAX;  // the leader's k-th best so far
  int thr_i = INT32_MAX;
  for (int64_t c = c_begin + warp; c < c_end; c += kNbrWarps) {
    const T* row = table + (int64_t)__ldg(cand + c) * pitch;
    float x[NE];
#pragma unroll
    for (int i = 0; i < NE; i++) {
      const int e = lane + 32 * i;
      x[i] = e < d ? elem(row, e) : 0.0f;
    }
    float a[kQB];
#pragma unroll
    for (int j = 0; j < kQB; j++) {
      float s = 0.0f;
#pragma unroll
      for (int i = 0; i < NE; i++) s = __fmaf_rn(qv[j][i], x[i], s);
      a[j] = s;
    }
    const float score = reduce8(a, lane) * __ldg(inv + c);
    const int ci = (int)c;
    if (leader && ci != my_self && better(score, ci, thr_s, thr_i)) {
      list_insert(ls[warp][myq], li[warp][myq], k, score, ci);
      thr_s = ls[warp][myq][k - 1];
      thr_i = li[warp][myq][k - 1];
    }
  }
  __syncthreads();
  // the slice's best k of query j: warp j merges the warps' sorted lists,
  // lane w < kNbrWarps walking list w
  if (warp < kQB && q0 + warp < n_q) {
    const int j = warp;
    const int64_t out = ((q0 + j) * gridDim.y + blockIdx.y) * k;
    int head = 0;
    for (int r = 0; r < k; r++) {
      float bs = -FLT_MAX;
      int bi = INT32_MAX, src = lane;
      if (lane < kNbrWarps && head < k) {
        bs = ls[lane][j][head];
        bi = li[lane][j][head];
      }
      warp_best(bs, bi, src);
      if (lane == src) head++;
      if (lane == 0) {
        part_s[out + r] = bs;
        part_i[out + r] = bi;
      }
    }
  }
}

// One warp per query: the best k of its slices' sorted lists (lane s walking
// slice s), and the cosine of each (score times the query's inverse norm).
__global__ void merge_kernel(const float* part_s, const int32_t* part_i, int slices, int k, int64_t n_q,
                             const int32_t* queries, const float* inv, int32_t* out_i, float* out_s) {
  const int lane = threadIdx.x & 31;
  const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (q >= n_q) return;
  const float* ps = part_s + q * slices * k;
  const int32_t* pi = part_i + q * slices * k;
  const float qinv = inv[queries[q]];
  int head = 0;
  for (int r = 0; r < k; r++) {
    float bs = -FLT_MAX;
    int bi = INT32_MAX, src = lane;
    if (lane < slices && head < k) {
      bs = ps[lane * k + head];
      bi = pi[lane * k + head];
    }
    warp_best(bs, bi, src);
    if (lane == src) head++;
    if (lane == 0) {
      out_i[q * k + r] = bi;
      out_s[q * k + r] = bi == INT32_MAX ? -2.0f : bs * qinv;
    }
  }
}

template <typename T, int NE>
cudaError_t launch_neighbours(const T* table, int64_t pitch, int d, const int32_t* cand, int64_t n_cand,
                              const float* inv, const int32_t* queries, int64_t n_q, int k, int slices,
                              int64_t slice, float* part_s, int32_t* part_i, cudaStream_t st) {
  const dim3 grid((unsigned)((n_q + kQB - 1) / kQB), (unsigned)slices);
  neighbours_kernel<T, NE><<<grid, kNbrWarps * 32, 0, st>>>(table, pitch, d, cand, n_cand, inv, queries, n_q, k,
                                                             slice, part_s, part_i);
  return cudaGetLastError();
}

template <typename T>
cudaError_t run(const T* table, int64_t pitch, int d, const int32_t* cand, int64_t n_cand, const int32_t* queries,
                int64_t n_q, int k, int32_t* out_i, float* out_s, cudaStream_t st) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  // slices of the candidates so that the grid covers the GPU a few times over;
  // at most 32 (one merge lane each)
  const int64_t qblocks = (n_q + kQB - 1) / kQB;
  int slices = (int)((4 * (int64_t)sms * 2 + qblocks - 1) / qblocks);
  if (slices < 1) slices = 1;
  if (slices > 32) slices = 32;
  if ((int64_t)slices > n_cand) slices = (int)n_cand;
  const int64_t slice = (n_cand + slices - 1) / slices;
  float* inv = nullptr;
  float* part_s = nullptr;
  int32_t* part_i = nullptr;
  e = cudaMallocAsync((void**)&inv, (size_t)n_cand * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&part_s, (size_t)n_q * slices * k * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&part_i, (size_t)n_q * slices * k * sizeof(int32_t), st);
  if (e == cudaSuccess) {
    inv_norm_kernel<T><<<sms * 8, 256, 0, st>>>(table, pitch, d, cand, n_cand, inv);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    if (d <= 128) e = launch_neighbours<T, 4>(table, pitch, d, cand, n_cand, inv, queries, n_q, k, slices, slice,
                                              part_s, part_i, st);
    else if (d <= 256) e = launch_neighbours<T, 8>(table, pitch, d, cand, n_cand, inv, queries, n_q, k, slices,
                                                   slice, part_s, part_i, st);
    else if (d <= 384) e = launch_neighbours<T, 12>(table, pitch, d, cand, n_cand, inv, queries, n_q, k, slices,
                                                    slice, part_s, part_i, st);
    else e = launch_neighbours<T, 16>(table, pitch, d, cand, n_cand, inv, queries, n_q, k, slices, slice, part_s,
                                      part_i, st);
  }
  if (e == cudaSuccess) {
    merge_kernel<<<(unsigned)((n_q * 32 + 255) / 256), 256, 0, st>>>(part_s, part_i, slices, k, n_q, queries, inv,
                                                                     out_i, out_s);
    e = cudaGetLastError();
  }
  if (inv) cudaFreeAsync(inv, st);
  if (part_s) cudaFreeAsync(part_s, st);
  if (part_i) cudaFreeAsync(part_i, st);
  return e;
}

}  // namespace
}  // namespace fw2v

extern "C" fw2v_status fw2v_neighbours(const void* table, int32_t precision, int64_t pitch, int32_t layer_size,
                                       const int32_t* cand, int64_t n_cand, const int32_t* queries,
                                       int64_t n_queries, int32_t k, int32_t* out_idx, float* out_sim,
                                       void* stream) {
  if (!table || !cand || !queries || !out_idx || !out_sim || layer_size < 1 || layer_size > 512 ||
      pitch < layer_size || (precision != FW2V_FP32 && precision != FW2V_BF16) || n_cand < 2 ||
      n_cand > INT32_MAX || n_queries < 0 || k < 1 || k > fw2v::kMaxK || k >= n_cand)
    return FW2V_ERR_ARGUMENT;
  if (n_queries == 0) return FW2V_OK;
  const cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e =
      precision == FW2V_FP32
          ? fw2v::run<float>((const float*)table, pitch, layer_size, cand, n_cand, queries, n_queries, k, out_idx,
                             out_sim, st)
          : fw2v::run<uint16_t>((const uint16_t*)table, pitch, layer_size, cand, n_cand, queries, n_queries, k,
                                out_idx, out_sim, st);
  if (e == cudaErrorMemoryAllocation) return FW2V_ERR_NOMEM;
  return e == cudaSuccess ? FW2V_OK : FW2V_ERR_CUDA;
}
