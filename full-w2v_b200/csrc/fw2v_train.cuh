// SGNS training kernel: the method of FULL-W2V-kernels.cu:106-250 re-laid out
// for one warp per sentence.
//
// Layout.  A warp trains one sentence at a time.  Every table row is split over
// the 32 lanes in VEC-float vectors: lane l holds elements ((i*32+l)*VEC + j)
// for i < NV, j < VEC, so a row is read with 128-bit loads and a dot product is
// VEC*NV FMAs per lane plus a 5-step xor-shuffle reduction (16,8,4,2,1) — no
// block barrier per (context, target) pair as in the reference's blockReduceM2.
//
// Lifetime reuse of context words.  Each warp owns a ring of 2W+1 row slots in
// shared memory (current value + value at load).  Position p of the sentence
// lives in slot p mod (2W+1) from the moment it enters the window until it
// leaves, when its accumulated change (current - loaded) is added to syn0 once.
// Each lane only ever touches its own elements of a slot, so the ring needs no
// synchronisation beyond program order.
//
// Independence of negative samples.  The 1+K target rows of a centre are read
// fresh from syn1neg, kept in registers through the whole window sweep and their
// change is added back once.  Because a target's sweep only depends on the
// previous target through the context rows, the 1+K sweeps run as a software
// pipeline skewed by one context: at step t target k works on context t-k,
// receiving the context row from target k-1 in registers.  The R independent
// dot products of a step overlap their shuffle latency, and the ring is read
// and written once per context per centre instead of once per pair.  The
// arithmetic of every value is the same, in the same order, as the serial
// method.  If two targets of a centre are the same word the centre falls back
// to serial sweeps, so the second one sees the first one's write.
//
// Context order: ascending ring slot (the reference's steady-state order,
// FULL-W2V-kernels.cu:170-182), over the textbook window [w-W, w+W] clipped to
// the sentence.  The reference's warm-up/cool-down deviations at sentence edges
// are not reproduced.
#pragma once
#include <cstdio>

#include "fw2v_common.cuh"

namespace fw2v {

template <int VEC, int NV>
struct Row {
  float x[NV][VEC];
};

template <int VEC, int NV>
__device__ __forceinline__ void row_zero(Row<VEC, NV>& r) {
#pragma unroll
  for (int i = 0; i < NV; i++)
#pragma unroll
    for (int j = 0; j < VEC; j++) r.x[i][j] = 0.0f;
}

// Row helpers.  Elements at or past the layer size d are never read from or
// written to global memory and are zero in registers; a vector that straddles d
// is accessed element by element.  Shared-memory rows have room for whole
// vectors (their stride is at least d rounded up to VEC).
template <int VEC, int NV>
__device__ __forceinline__ void row_load_global(Row<VEC, NV>& r, const float* row, int lane, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (e + VEC <= d) {
      if constexpr (VEC == 4) {
        const float4 t = __ldcg(reinterpret_cast<const float4*>(row + e));
        r.x[i][0] = t.x; r.x[i][1] = t.y; r.x[i][2] = t.z; r.x[i][3] = t.w;
      } else {
        const float2 t = __ldcg(reinterpret_cast<const float2*>(row + e));
        r.x[i][0] = t.x; r.x[i][1] = t.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++) r.x[i][j] = e + j < d ? __ldcg(row + e + j) : 0.0f;
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ void row_load_smem(Row<VEC, NV>& r, const float* row, int lane, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (e < d) {
      if constexpr (VEC == 4) {
        const float4 t = *reinterpret_cast<const float4*>(row + e);
        r.x[i][0] = t.x; r.x[i][1] = t.y; r.x[i][2] = t.z; r.x[i][3] = t.w;
      } else {
        const float2 t = *reinterpret_cast<const float2*>(row + e);
        r.x[i][0] = t.x; r.x[i][1] = t.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++) r.x[i][j] = 0.0f;
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ void row_store_smem(const Row<VEC, NV>& r, float* row, int lane, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (e < d) {
      if constexpr (VEC == 4) {
        *reinterpret_cast<float4*>(row + e) = make_float4(r.x[i][0], r.x[i][1], r.x[i][2], r.x[i][3]);
      } else {
        *reinterpret_cast<float2*>(row + e) = make_float2(r.x[i][0], r.x[i][1]);
      }
    }
  }
}

// row[e] += a[e] - b[e]: one vector atomic per lane and vector (sm_90+ float4 /
// float2 atomicAdd), element atomics for a vector that straddles d.
template <int VEC, int NV>
__device__ __forceinline__ void row_add_delta(float* row, const Row<VEC, NV>& a, const Row<VEC, NV>& b,
                                              int lane, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (e + VEC <= d) {
      if constexpr (VEC == 4) {
        const float4 dlt = make_float4(__fsub_rn(a.x[i][0], b.x[i][0]), __fsub_rn(a.x[i][1], b.x[i][1]),
                                       __fsub_rn(a.x[i][2], b.x[i][2]), __fsub_rn(a.x[i][3], b.x[i][3]));
        atomicAdd(reinterpret_cast<float4*>(row + e), dlt);
      } else {
        const float2 dlt = make_float2(__fsub_rn(a.x[i][0], b.x[i][0]), __fsub_rn(a.x[i][1], b.x[i][1]));
        atomicAdd(reinterpret_cast<float2*>(row + e), dlt);
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++)
        if (e + j < d) atomicAdd(row + e + j, __fsub_rn(a.x[i][j], b.x[i][j]));
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ float row_dot(const Row<VEC, NV>& a, const Row<VEC, NV>& b) {
  float p = __fmul_rn(a.x[0][0], b.x[0][0]);
#pragma unroll
  for (int i = 0; i < NV; i++)
#pragma unroll
    for (int j = 0; j < VEC; j++)
      if (i != 0 || j != 0) p = __fmaf_rn(a.x[i][j], b.x[i][j], p);
  return p;
}

__device__ __forceinline__ float warp_sum(float p) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) p = __fadd_rn(p, __shfl_xor_sync(kFull, p, m));
  return p;
}

// v += g*o and o += g*v_old, elementwise with single-rounding FMAs.
template <int VEC, int NV>
__device__ __forceinline__ void row_update(Row<VEC, NV>& v, Row<VEC, NV>& o, float g) {
#pragma unroll
  for (int i = 0; i < NV; i++)
#pragma unroll
    for (int j = 0; j < VEC; j++) {
      const float vo = v.x[i][j];
      v.x[i][j] = __fmaf_rn(g, o.x[i][j], vo);
      o.x[i][j] = __fmaf_rn(g, vo, o.x[i][j]);
    }
}

// alpha * (label - sigma(x)).  Table mode reproduces FULL-W2V-kernels.cu:92-99:
// index = (int)(saturate((x + 6) / 12) * 999); the positive target reads the
// reversed table (nexpTable[i] == expTable[999 - i]).
__device__ __forceinline__ float gradient(float x, bool positive, float alpha, int sigmoid,
                                          const float* table) {
  if (sigmoid == 0) {
    const float s = __saturatef(__fmul_rn(__fadd_rn(x, 6.0f), 1.0f / 12.0f));
    const int idx = __float2int_rz(__fmul_rn(s, 999.0f));
    return positive ? __fmul_rn(alpha, table[kExpTableSize - 1 - idx]) : __fmul_rn(-alpha, table[idx]);
  }
  return positive ? __fdiv_rn(alpha, __fadd_rn(1.0f, expf(x)))
                  : __fdiv_rn(-alpha, __fadd_rn(1.0f, expf(-x)));
}

struct Sentence {
  int64_t start;
  int32_t len;
  float alpha;
};

__device__ __forceinline__ int64_t total_sentences(const TrainParams& p) {
  if (p.source == kSourceEpoch) return p.entry_prefix[p.threads];
  return p.n_sentences;
}

__device__ __forceinline__ Sentence fetch_sentence(const TrainParams& p, int64_t w) {
  Sentence s;
  if (p.source == kSourceEpoch) {
    int lo = 0, hi = p.threads - 1;  // last stream with prefix <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.entry_prefix[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int64_t slot = entry_base(p.chunk_off, p.n_chunks, p.threads, lo) + (w - p.entry_prefix[lo]);
    s.start = p.ent_start[slot];
    s.len = p.ent_len[slot];
    s.alpha = p.ent_alpha[slot];
  } else if (p.source == kSourceExplicit) {
    s.start = p.starts[w];
    s.len = p.lens[w];
    s.alpha = p.alphas[w];
  } else {
    s.start = w * (int64_t)p.msl;
    s.len = p.lens[w];
    s.alpha = p.alphas[w];
    if (s.len > p.msl) s.len = -1;  // flagged below
  }
  return s;
}

// Reduce N per-lane partial sums at once (N a power of two <= 8).  The first
// log2(N) xor levels (masks 16, 8, 4) exchange half of the values each, so a
// level costs N/2 shuffles instead of N; afterwards lane l holds the complete
// sum of value stage_of_lane<N>(l), and the remaining levels are a plain
// butterfly.  Every partial is combined with the same partner in the same
// mask order (16, 8, 4, 2, 1) as a per-value butterfly, so the sums are
// bit-identical to reducing each value separately.
template <int N>
__device__ __forceinline__ float transpose_reduce(float (&a)[N], int lane) {
  static_assert(N == 1 || N == 2 || N == 4 || N == 8, "N must be 1, 2, 4 or 8");
  if constexpr (N >= 2) {
    const bool hi = lane & 16;
#pragma unroll
    for (int j = 0; j < N / 2; j++) {
      const float send = hi ? a[j] : a[j + N / 2];
      const float keep = hi ? a[j + N / 2] : a[j];
      a[j] = __fadd_rn(keep, __shfl_xor_sync(kFull, send, 16));
    }
  }
  if constexpr (N >= 4) {
    const bool hi = lane & 8;
#pragma unroll
    for (int j = 0; j < N / 4; j++) {
      const float send = hi ? a[j] : a[j + N / 4];
      const float keep = hi ? a[j + N / 4] : a[j];
      a[j] = __fadd_rn(keep, __shfl_xor_sync(kFull, send, 8));
    }
  }
  if constexpr (N >= 8) {
    const bool hi = lane & 4;
    const float send = hi ? a[0] : a[1];
    const float keep = hi ? a[1] : a[0];
    a[0] = __fadd_rn(keep, __shfl_xor_sync(kFull, send, 4));
  }
  float r = a[0];
  constexpr int first_plain = N == 8 ? 2 : N == 4 ? 4 : N == 2 ? 8 : 16;
#pragma unroll
  for (int m = first_plain; m >= 1; m >>= 1) r = __fadd_rn(r, __shfl_xor_sync(kFull, r, m));
  return r;
}

template <int N>
__device__ __forceinline__ int stage_of_lane(int lane) {
  if constexpr (N == 8) return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
  if constexpr (N == 4) return ((lane >> 4) & 1) * 2 + ((lane >> 3) & 1);
  if constexpr (N == 2) return (lane >> 4) & 1;
  return 0;
}

template <int N>
__device__ __forceinline__ constexpr int lane_of_stage(int k) {
  if constexpr (N == 8) return ((k >> 2) & 1) * 16 + ((k >> 1) & 1) * 8 + (k & 1) * 4;
  if constexpr (N == 4) return ((k >> 1) & 1) * 16 + (k & 1) * 8;
  if constexpr (N == 2) return k * 16;
  return 0;
}

template <int R>
struct PadPow2 {
  static constexpr int value = R <= 1 ? 1 : R <= 2 ? 2 : R <= 4 ? 4 : 8;
};

// Ids of the targets of centre w, lane k < nt holding target k0 + k (positive
// word first, then the K negatives).
__device__ __forceinline__ int target_id(const int32_t* ids, const int32_t* negs, int K, int w, int k0,
                                         int nt, int lane) {
  if (lane >= nt) return 0;
  const int k = k0 + lane;
  return k == 0 ? __ldg(ids + w) : __ldg(negs + (int64_t)w * K + (k - 1));
}

template <int VEC, int NV, int R>
__device__ void train_sentence(const TrainParams& p, const Sentence& sn, float* ring_cur, float* ring_orig,
                               const float* table, int lane) {
  constexpr int RP = PadPow2<R>::value;
  const int W = p.window, K = p.negative, D = 2 * W + 1;
  const int P = (int)p.pitch;  // row stride, global and shared
  const int d = p.d;
  const int L = sn.len;
  const int32_t* ids = p.ids + sn.start;
  const int32_t* negs = p.negs + sn.start * (int64_t)K;
  const float alpha = sn.alpha;
  const bool one_group = K + 1 <= R;

  // Every id is checked before any table access.
  bool bad = L < 0;
  for (int i = lane; i < L; i += 32) {
    const int32_t t = __ldg(ids + i);
    bad |= (t < 0) | ((int64_t)t >= p.vocab);
  }
  for (int64_t i = lane; i < (int64_t)L * K; i += 32) {
    const int32_t t = __ldg(negs + i);
    bad |= (t < 0) | ((int64_t)t >= p.vocab);
  }
  if (__any_sync(kFull, bad)) {
    if (lane == 0) atomicExch(p.error_flag, 1);
    return;
  }
  if (L <= 0) return;

  Row<VEC, NV> tmp;
  const int n_enter = W + 1 < L ? W + 1 : L;
  for (int q = 0; q < n_enter; q++) {
    row_load_global(tmp, p.syn0 + (int64_t)__ldg(ids + q) * P, lane, d);
    row_store_smem(tmp, ring_cur + q * P, lane, d);
    row_store_smem(tmp, ring_orig + q * P, lane, d);
  }

  // v[r] holds the context row whose index j in the centre's list has
  // j % R == r: stage k works on context t-k at step t, i.e. on register slot
  // (t - k) % R, so a row moves from stage to stage without being copied.
  Row<VEC, NV> v[R], o[R], o0[R];
  int vslot[R];
#pragma unroll
  for (int k = 0; k < R; k++) {
    row_zero(v[k]);
    vslot[k] = 0;
  }

  int t_next = one_group ? target_id(ids, negs, K, 0, 0, K + 1, lane) : 0;
  for (int w = 0; w < L; w++) {
    // Ids needed later in this centre, loaded ahead of use.
    const int q_out = w - W, q_in = w + W + 1;
    const int id_out = q_out >= 0 ? __ldg(ids + q_out) : -1;
    const int id_in = q_in < L ? __ldg(ids + q_in) : -1;
    const int t_here = t_next;
    if (one_group && w + 1 < L) t_next = target_id(ids, negs, K, w + 1, 0, K + 1, lane);
    // The entering row can be fetched now unless the leaving position holds
    // the same word (its write-back must land first).
    const bool enter_early = id_in >= 0 && id_in != id_out;
    Row<VEC, NV> enter_row;
    if (enter_early) row_load_global(enter_row, p.syn0 + (int64_t)id_in * P, lane, d);

    // Lane r < D decides whether ring slot r holds a context of centre w.
    const int base = w - W;
    bool valid = false;
    if (lane < D) {
      const int off = ((lane - base) % D + D) % D;
      const int pos = base + off;
      valid = pos != w && pos >= 0 && pos < L;
    }
    const unsigned mask = __ballot_sync(kFull, valid);
    const int nctx = __popc(mask);

    if (nctx > 0) {
      for (int k0 = 0; k0 <= K; k0 += R) {
        const int nt = (K + 1 - k0) < R ? (K + 1 - k0) : R;
        const int my_t = one_group ? t_here : target_id(ids, negs, K, w, k0, nt, lane);
        bool dup = false;
        for (int j = 0; j + 1 < nt; j++) {
          const int tj = __shfl_sync(kFull, my_t, j);
          dup |= lane > j && lane < nt && tj == my_t;
        }
        if (!__any_sync(kFull, dup)) {
          // ---- pipelined sweeps of nt targets ----
          int t[R];
#pragma unroll
          for (int k = 0; k < R; k++) {
            t[k] = __shfl_sync(kFull, my_t, k);
            if (k < nt) {
              row_load_global(o[k], p.syn1neg + (int64_t)t[k] * P, lane, d);
              o0[k] = o[k];
            } else {
              row_zero(o[k]);
            }
          }
          const int my_stage = stage_of_lane<RP>(lane);
          const bool my_positive = k0 + my_stage == 0;
          unsigned rem = mask;
          const int steps = nctx + R - 1;
          for (int t0 = 0; t0 < steps; t0 += R) {
#pragma unroll
            for (int u = 0; u < R; u++) {
              const int ts = t0 + u;
              if (ts < steps) {
                if (ts < nctx) {
                  const int s0 = __ffs(rem) - 1;
                  rem &= rem - 1;
                  vslot[u] = s0;
                  row_load_smem(v[u], ring_cur + s0 * P, lane, d);
                } else {
                  row_zero(v[u]);
                }
                float x[RP];
#pragma unroll
                for (int k = 0; k < RP; k++) x[k] = k < R ? row_dot(v[(u - k + R) % R], o[k < R ? k : 0]) : 0.0f;
                const float xs = transpose_reduce<RP>(x, lane);
                const int j = ts - my_stage;
                const bool act = my_stage < nt && j >= 0 && j < nctx;
                const float g = act ? gradient(xs, my_positive, alpha, p.sigmoid, table) : 0.0f;
#pragma unroll
                for (int k = 0; k < R; k++) {
                  const float gk = __shfl_sync(kFull, g, lane_of_stage<RP>(k));
                  row_update(v[(u - k + R) % R], o[k], gk);
                }
                const int jo = ts - (R - 1);
                if (jo >= 0 && jo < nctx) row_store_smem(v[(u + 1) % R], ring_cur + vslot[(u + 1) % R] * P, lane, d);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < R; k++)
            if (k < nt) row_add_delta(p.syn1neg + (int64_t)t[k] * P, o[k], o0[k], lane, d);
        } else {
          // ---- serial sweeps: a repeated target must see the earlier write ----
          for (int k = 0; k < nt; k++) {
            const int tk = __shfl_sync(kFull, my_t, k);
            Row<VEC, NV> so, so0, sv;
            row_load_global(so, p.syn1neg + (int64_t)tk * P, lane, d);
            so0 = so;
            unsigned rem = mask;
            for (int j = 0; j < nctx; j++) {
              const int s0 = __ffs(rem) - 1;
              rem &= rem - 1;
              row_load_smem(sv, ring_cur + s0 * P, lane, d);
              const float x = warp_sum(row_dot(sv, so));
              const float g = gradient(x, k0 + k == 0, alpha, p.sigmoid, table);
              row_update(sv, so, g);
              row_store_smem(sv, ring_cur + s0 * P, lane, d);
            }
            row_add_delta(p.syn1neg + (int64_t)tk * P, so, so0, lane, d);
          }
        }
      }
    }

    // Slide the window: position w-W leaves, position w+W+1 takes its slot.
    if (q_out >= 0) {
      const int s = q_out % D;
      Row<VEC, NV> cur, org;
      row_load_smem(cur, ring_cur + s * P, lane, d);
      row_load_smem(org, ring_orig + s * P, lane, d);
      row_add_delta(p.syn0 + (int64_t)id_out * P, cur, org, lane, d);
    }
    if (id_in >= 0) {
      const int s = q_in % D;
      if (!enter_early) row_load_global(enter_row, p.syn0 + (int64_t)id_in * P, lane, d);
      row_store_smem(enter_row, ring_cur + s * P, lane, d);
      row_store_smem(enter_row, ring_orig + s * P, lane, d);
    }
  }
  // Positions still in the window leave in increasing order.
  for (int q = L - W > 0 ? L - W : 0; q < L; q++) {
    const int s = q % D;
    Row<VEC, NV> cur, org;
    row_load_smem(cur, ring_cur + s * P, lane, d);
    row_load_smem(org, ring_orig + s * P, lane, d);
    row_add_delta(p.syn0 + (int64_t)__ldg(ids + q) * P, cur, org, lane, d);
  }
}

template <int VEC, int NV, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) sgns_train_kernel(TrainParams p) {
  extern __shared__ __align__(16) float smem[];
  float* table = smem;
  for (int i = threadIdx.x; i < kExpTableSize; i += blockDim.x) table[i] = p.exp_table[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int D = 2 * p.window + 1;
  const int64_t ring = (int64_t)D * p.pitch;
  float* ring_cur = smem + 1024 + (int64_t)warp * 2 * ring;
  float* ring_orig = ring_cur + ring;
  const int64_t total = total_sentences(p);
  if (p.deterministic) {
    if (blockIdx.x != 0 || warp != 0) return;
    for (int64_t w = 0; w < total; w++) {
      const Sentence sn = fetch_sentence(p, w);
      train_sentence<VEC, NV, R>(p, sn, ring_cur, ring_orig, table, lane);
    }
    return;
  }
  if (p.work_counter == nullptr) {
    // Static assignment (the kernel seam, whose launches may run concurrently).
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; w < total; w += warps) {
      const Sentence sn = fetch_sentence(p, w);
      train_sentence<VEC, NV, R>(p, sn, ring_cur, ring_orig, table, lane);
    }
    return;
  }
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(p.work_counter, 1ULL);
    w = __shfl_sync(kFull, w, 0);
    if ((int64_t)w >= total) break;
    const Sentence sn = fetch_sentence(p, (int64_t)w);
    train_sentence<VEC, NV, R>(p, sn, ring_cur, ring_orig, table, lane);
  }
}

// ---------------------------------------------------------------------------
// Held-out SGNS loss: one warp per sentence, FP64 accumulation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double log_sigmoid(double x) {
  return x >= 0 ? -log1p(exp(-x)) : x - log1p(exp(x));
}

template <int VEC, int NV>
__global__ void __launch_bounds__(128) heldout_loss_kernel(TrainParams p, double* loss, unsigned long long* pairs) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int P = (int)p.pitch, W = p.window, K = p.negative, D = 2 * W + 1, d = p.d;
  double acc = 0.0;
  unsigned long long np = 0;
  for (int64_t s = gw; s < p.n_sentences; s += nw) {
    const int64_t start = p.starts[s];
    const int L = p.lens[s];
    const int32_t* ids = p.ids + start;
    const int32_t* negs = p.negs + start * (int64_t)K;
    bool bad = false;
    for (int i = lane; i < L; i += 32) bad |= ids[i] < 0 || (int64_t)ids[i] >= p.vocab;
    for (int64_t i = lane; i < (int64_t)L * K; i += 32) bad |= negs[i] < 0 || (int64_t)negs[i] >= p.vocab;
    if (__any_sync(kFull, bad)) {
      if (lane == 0) atomicExch(p.error_flag, 1);
      continue;
    }
    for (int w = 0; w < L; w++) {
      const int base = w - W;
      for (int r = 0; r < D; r++) {
        const int pos = base + ((r - base) % D + D) % D;
        if (pos == w || pos < 0 || pos >= L) continue;
        Row<VEC, NV> v, o;
        row_load_global(v, p.syn0 + (int64_t)ids[pos] * P, lane, d);
        for (int k = 0; k <= K; k++) {
          const int32_t t = k == 0 ? ids[w] : negs[(int64_t)w * K + k - 1];
          row_load_global(o, p.syn1neg + (int64_t)t * P, lane, d);
          // FP64 dot: per-lane partial in double, then the xor tree
          double part = 0.0;
#pragma unroll
          for (int i = 0; i < NV; i++)
#pragma unroll
            for (int j = 0; j < VEC; j++) part += (double)v.x[i][j] * (double)o.x[i][j];
#pragma unroll
          for (int m = 16; m >= 1; m >>= 1) part += __shfl_xor_sync(kFull, part, m);
          acc -= k == 0 ? log_sigmoid(part) : log_sigmoid(-part);
        }
        np++;
      }
    }
  }
  if (lane == 0) {
    atomicAdd(loss, acc);
    atomicAdd(pairs, np);
  }
}

// Launch of one (VEC, NV) shape for any stage count R (instantiated per shape
// in fw2v_train_<shape>.cu so the shapes compile in parallel).
template <int VEC, int NV, int R>
cudaError_t launch_t(const TrainParams& p, int num_sms, size_t smem, cudaStream_t st) {
  auto kern = sgns_train_kernel<VEC, NV, R>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int blocks = 1;
  int threads = kWarpsPerBlock * 32;
  if (p.deterministic) {
    threads = 32;
  } else {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    blocks = per_sm * num_sms;
  }
  kern<<<blocks, threads, smem, st>>>(p);
  return cudaGetLastError();
}

template <int VEC, int NV>
cudaError_t launch_r(const TrainParams& p, int r, int num_sms, size_t smem, cudaStream_t st) {
  switch (r) {
    case 1: return launch_t<VEC, NV, 1>(p, num_sms, smem, st);
    case 2: return launch_t<VEC, NV, 2>(p, num_sms, smem, st);
    case 4: return launch_t<VEC, NV, 4>(p, num_sms, smem, st);
    case 6: return launch_t<VEC, NV, 6>(p, num_sms, smem, st);
    default: return launch_t<VEC, NV, 8>(p, num_sms, smem, st);
  }
}

}  // namespace fw2v
