// Uniform random walks on a graph in CSR form, written straight into a
// training token stream on the device: the generator of the graph-embedding
// corpora (random walks written one per line and read with -cache-eos, so a
// walk is a sentence ending in </s>; the reference reads such corpora as text,
// improved_driver_functions.cpp:244-281).
//
//   walks_kernel    one thread per walk: start node, then each step a
//                   uniform neighbour (a node without neighbours stays put);
//                   the step's neighbour index comes from a counter-based
//                   hash of (seed, walk, step), so a walk does not depend on
//                   which thread runs it or when.  Writes raw node ids, walk w
//                   at w * (len + 1), followed by one separator slot.
//   relabel_kernel  raw node ids -> vocabulary ids (a node's id in the
//                   corpus vocabulary), the separator slots -> 0 (</s>).
#include "../../include/fw2v.h"
#include "fw2v_common.cuh"

namespace fw2v {
namespace {

// Uniform integer in [0, n) from 64 random bits (multiply-high; bias below
// n / 2^64).
__device__ __forceinline__ int64_t uniform_below(uint64_t r, int64_t n) {
  return (int64_t)__umul64hi(r, (uint64_t)n);
}

__device__ __forceinline__ uint64_t walk_bits(uint64_t key, uint64_t walk, uint64_t step) {
  return mix64(key ^ mix64(walk * 0x9E3779B97F4A7C15ULL + step));
}

// Node ids outside [0, nodes) (a malformed graph) end the walk in place: the
// kernel reads only offs[0..nodes] and dst[offs[0]..offs[nodes]).
__global__ void walks_kernel(const int64_t* offs, const int32_t* dst, int64_t nodes, const int32_t* starts,
                             int64_t n_walks, int len, uint64_t key, int32_t* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t e_lo = offs[0], e_hi = offs[nodes];
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_walks; w += stride) {
    int32_t cur = starts[w];
    if ((uint64_t)cur >= (uint64_t)nodes) cur = 0;
    int32_t* o = out + w * (int64_t)(len + 1);
    o[0] = cur;
    for (int t = 1; t < len; t++) {
      const int64_t b = offs[cur], deg = offs[cur + 1] - b;
      if (deg > 0 && b >= e_lo && b + deg <= e_hi) {
        const int32_t nxt = dst[b + uniform_below(walk_bits(key, (uint64_t)w, (uint64_t)t), deg)];
        if ((uint64_t)nxt < (uint64_t)nodes) cur = nxt;
      }
      o[t] = cur;
    }
    o[len] = -1;  // separator slot
  }
}

__global__ void relabel_kernel(int32_t* stream, int64_t n, const int32_t* vocab_of, int64_t nodes) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t x = stream[i];
    stream[i] = x < 0 || x >= nodes ? 0 : vocab_of[x];
  }
}

}  // namespace
}  // namespace fw2v

extern "C" fw2v_status fw2v_random_walks(const int64_t* offs, const int32_t* dst, int64_t nodes,
                                         const int32_t* starts, int64_t n_walks, int32_t walk_len, uint64_t seed,
                                         int32_t* out, void* stream) {
  if (!offs || !dst || !starts || !out || nodes < 1 || nodes > INT32_MAX || n_walks < 0 || walk_len < 1)
    return FW2V_ERR_ARGUMENT;
  if (n_walks == 0) return FW2V_OK;
  fw2v::walks_kernel<<<148 * 16, 256, 0, (cudaStream_t)stream>>>(offs, dst, nodes, starts, n_walks, walk_len,
                                                                   fw2v::mix64(seed), out);
  return cudaGetLastError() == cudaSuccess ? FW2V_OK : FW2V_ERR_CUDA;
}

extern "C" fw2v_status fw2v_relabel_stream(int32_t* stream, int64_t n, const int32_t* vocab_of, int64_t nodes,
                                           void* cuda_stream) {
  if (!stream || !vocab_of || n < 0 || nodes < 1) return FW2V_ERR_ARGUMENT;
  if (n == 0) return FW2V_OK;
  fw2v::relabel_kernel<<<148 * 8, 256, 0, (cudaStream_t)cuda_stream>>>(stream, n, vocab_of, nodes);
  return cudaGetLastError() == cudaSuccess ? FW2V_OK : FW2V_ERR_CUDA;
}
