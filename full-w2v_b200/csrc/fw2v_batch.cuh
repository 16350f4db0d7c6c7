// Persistent training kernel for a batch of independent SGNS jobs.
//
// One launch drains a device work queue of (job, sentence) items: the entries
// of a round's sampling streams, numbered in round order through the round's
// entry prefix.  Each warp claims items with an atomic counter (or, in the
// deterministic mode, warp 0 takes them all in order), finds the item's
// stream, job and entry, keeps the job's parameter block in shared memory
// while consecutive items belong to the same job, and trains the sentence
// with train_sentence (fw2v_train.cuh) on the job's own tables.
//
// Jobs differ in layer size, window and tables; the kernel holds the compiled
// bodies for every (lane vector width, pipeline stages) pair a job may use and
// dispatches on the job's own pair per sentence.  A job's pair is a per-job
// parameter (set by the caller or chosen by the autotuner), so one launch can
// train jobs of d <= 64 on 2-float lane vectors, jobs of d <= 128 on 4-float
// ones, each with the stage count that suits its window.
#pragma once
#include "fw2v_train.cuh"

namespace fw2v {

struct BatchTrainArgs {
  const TrainParams* jobs;      // per job; ids / negs point into the round's buffers
  BatchRound round;
  const int64_t* entry_prefix;  // round streams + 1
  const int64_t* uid_base;      // per round stream: the job-epoch number of its first entry
  const int64_t* ent_start;
  const int32_t* ent_len;
  const float* ent_alpha;
  unsigned long long* work_counter;
  int deterministic;
  int epoch;                    // stochastic-rounding seeds: launch number of each job
  void* orig_scratch;           // per warp: scratch_elems table elements
  int64_t scratch_elems;
  int64_t scratch_warps;
  int64_t smem_floats;          // per warp: shared-memory floats (warp_smem_bytes / 4)
  const float* exp_table;
};

// Stage counts compiled into the batched kernels (a job with 1 + K targets
// per centre sweeps them in ceil((1 + K) / stages) groups).
constexpr int kBatchStages[] = {2, 3, 4, 6};

// Kernel families, each compiled for its own register budget (the largest of
// its bodies sets it for all):
//   0  rows of one vector per lane (d <= 128: 2-float lanes for d <= 64,
//      4-float for d <= 128), up to 8 warps per block, 128 registers
//   1  wide rows: 2 four-float vectors per lane with 2 or 3 stages, 3 vectors
//      with 2; up to 6 warps per block, 168 registers (12 warps per SM: 2
//      blocks of 6, or 3 of 4)
//   2  other wide rows (2 vectors: 4 or 6 stages; 3 vectors: 3 or 4); 4 warps
//      per block, 255 registers
constexpr int kBatchMaxWarps = 8;
constexpr int kBatchFamilies = 3;
template <int FAMILY>
struct BatchFamily;
template <>
struct BatchFamily<0> {
  static constexpr int kMaxWarps = 8, kMinBlocks = 2;
};
template <>
struct BatchFamily<1> {
  static constexpr int kMaxWarps = 6, kMinBlocks = 2;
};
template <>
struct BatchFamily<2> {
  static constexpr int kMaxWarps = 4, kMinBlocks = 2;
};

__host__ __device__ constexpr int batch_max_warps(int family) {
  return family == 0 ? BatchFamily<0>::kMaxWarps : family == 1 ? BatchFamily<1>::kMaxWarps : BatchFamily<2>::kMaxWarps;
}

// The family of a (lane vector width, vectors per lane, stages) shape.
__host__ __device__ constexpr int batch_family(int nv, int stages) {
  return nv == 1 ? 0 : (stages == 2 || (nv == 2 && stages == 3)) ? 1 : 2;
}

// Rows of three vectors per lane stop at 4 stages: their 6-stage body does not
// fit the register file.
template <typename T, int VEC, int NV>
__device__ __forceinline__ bool batch_stages(const TrainParams& p, const Sentence& sn, float* ring, T* orig,
                                             const float* table, int lane, uint32_t bar, uint32_t& phase) {
  switch (p.stages) {
    case 2: return train_sentence<T, VEC, NV, 2, 0>(p, sn, ring, orig, table, lane, bar, phase);
    case 3: return train_sentence<T, VEC, NV, 3, 0>(p, sn, ring, orig, table, lane, bar, phase);
    case 4: return train_sentence<T, VEC, NV, 4, 0>(p, sn, ring, orig, table, lane, bar, phase);
    default:
      if constexpr (NV < 3) return train_sentence<T, VEC, NV, 6, 0>(p, sn, ring, orig, table, lane, bar, phase);
      return true;
  }
}

// False if the sentence stopped on a bulk copy that did not complete.
template <typename T, int FAMILY>
__device__ __forceinline__ bool batch_dispatch(const TrainParams& p, const Sentence& sn, float* ring, T* orig,
                                               const float* table, int lane, uint32_t bar, uint32_t& phase) {
  if constexpr (FAMILY == 0) {
    if (p.lane_vec == 2) return batch_stages<T, 2, 1>(p, sn, ring, orig, table, lane, bar, phase);
    return batch_stages<T, 4, 1>(p, sn, ring, orig, table, lane, bar, phase);
  } else if constexpr (FAMILY == 1) {
    if (p.lane_nv == 3) return train_sentence<T, 4, 3, 2, 0>(p, sn, ring, orig, table, lane, bar, phase);
    if (p.stages == 2) return train_sentence<T, 4, 2, 2, 0>(p, sn, ring, orig, table, lane, bar, phase);
    return train_sentence<T, 4, 2, 3, 0>(p, sn, ring, orig, table, lane, bar, phase);
  } else {
    if (p.lane_nv == 3) {
      if (p.stages == 3) return train_sentence<T, 4, 3, 3, 0>(p, sn, ring, orig, table, lane, bar, phase);
      return train_sentence<T, 4, 3, 4, 0>(p, sn, ring, orig, table, lane, bar, phase);
    }
    if (p.stages == 4) return train_sentence<T, 4, 2, 4, 0>(p, sn, ring, orig, table, lane, bar, phase);
    return train_sentence<T, 4, 2, 6, 0>(p, sn, ring, orig, table, lane, bar, phase);
  }
}

template <typename T, int FAMILY>
__global__ void __launch_bounds__(BatchFamily<FAMILY>::kMaxWarps * 32, BatchFamily<FAMILY>::kMinBlocks)
    sgns_batch_kernel(BatchTrainArgs a) {
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) TrainParams tp[BatchFamily<FAMILY>::kMaxWarps];
  __shared__ float table[kExpTableSize];  // the sigmoid table, read once per pipeline step
  for (int i = threadIdx.x; i < kExpTableSize; i += blockDim.x) table[i] = a.exp_table[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* ring = smem + (int64_t)warp * a.smem_floats;
  const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  T* orig = reinterpret_cast<T*>(a.orig_scratch) + gwarp * a.scratch_elems;
  const int64_t total = a.entry_prefix[a.round.n];
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  if (a.deterministic && gwarp != 0) return;
  if (gwarp >= a.scratch_warps) return;
  // the mbarrier at the end of the warp's region (every job's layout fits before it)
  const uint32_t bar = warp_bulk_init(ring, (uint32_t)(a.smem_floats * 4), lane);
  uint32_t phase = 0;
  int cur = -1;
  int64_t next = gwarp;
  for (;;) {
    int64_t w;
    if (a.deterministic) {
      w = next++;
    } else if (a.work_counter) {
      unsigned long long c = 0;
      if (lane == 0) c = atomicAdd(a.work_counter, 1ULL);
      w = (int64_t)__shfl_sync(kFull, c, 0);
    } else {
      w = next;
      next += nwarps;
    }
    if (w >= total) break;
    int lo = 0, hi = a.round.n - 1;  // last round stream with prefix <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.entry_prefix[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int j = a.round.job[lo];
    if (j != cur) {
      __syncwarp();
      copy_params(&tp[warp], &a.jobs[j], lane, 32);
      __syncwarp();
      if (lane == 0) tp[warp].sr_seed = mix64(0x5EEDF00DULL + (uint64_t)a.epoch + tp[warp].sr_seed);
      __syncwarp();
      cur = j;
    }
    const int64_t e = w - a.entry_prefix[lo];
    const int64_t slot = a.round.kbase[lo] + 2 * (int64_t)lo + e;
    Sentence sn;
    sn.start = a.ent_start[slot];
    sn.len = a.ent_len[slot];
    sn.alpha = a.ent_alpha[slot];
    sn.uid = a.uid_base[lo] + e;
    if (!batch_dispatch<T, FAMILY>(tp[warp], sn, ring, orig, table, lane, bar, phase)) break;
  }
}

// Grid of a batched launch: `warps` warps per block (sentences trained side
// by side in a block), as many blocks per SM as registers and shared memory
// allow, at most `per_sm_cap` if that is positive, and no more warps than the
// scratch covers.  Called before any stream capture.
template <typename T, int FAMILY>
cudaError_t batch_grid(int64_t smem_floats, int warps, int per_sm_cap, int num_sms, int64_t scratch_warps,
                       int deterministic, int* blocks, int* threads, size_t* smem) {
  auto kern = sgns_batch_kernel<T, FAMILY>;
  if (deterministic) warps = 1;
  if (warps < 1 || warps > BatchFamily<FAMILY>::kMaxWarps) return cudaErrorInvalidValue;
  *smem = (size_t)warps * (size_t)smem_floats * sizeof(float);
  *threads = warps * 32;
  // A block that does not fit is refused here, before any CUDA call can fail
  // and leave its error to be read back after a later launch.
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  if (*smem + fa.sharedSizeBytes > (size_t)optin) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  if (e != cudaSuccess) return e;
  if (deterministic) {
    *blocks = 1;
    return cudaSuccess;
  }
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, *threads, *smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm_cap > 0 && per_sm > per_sm_cap) per_sm = per_sm_cap;
  int64_t b = (int64_t)per_sm * num_sms;
  if (b * warps > scratch_warps) b = scratch_warps / warps;
  if (b < 1) return cudaErrorInvalidConfiguration;
  *blocks = (int)b;
  return cudaSuccess;
}

template <typename T, int FAMILY>
cudaError_t batch_launch(const BatchTrainArgs& a, int blocks, int threads, size_t smem, cudaStream_t st) {
  sgns_batch_kernel<T, FAMILY><<<blocks, threads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace fw2v
