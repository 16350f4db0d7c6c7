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
#include <cuda_bf16.h>

#include <cstdio>
#include <type_traits>
#include <utility>

#include "fw2v_common.cuh"

namespace fw2v {

// Compile-time loop: f(std::integral_constant<int, I>) for I = 0..N-1, so that
// register arrays indexed by I are never indexed at run time.
template <class F, int... Is>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <int VEC, int NV>
struct Row {
  float x[NV][VEC];
};

// Shared-memory rows addressed by 32-bit shared-window byte offsets.  Lane l
// accesses vector i of a row at byte offset lane_off(i) when lane_ok(i).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Lane layouts of up to 4 vectors per lane use ceil(d / (32 VEC)) of them,
// so every vector but the last lies wholly inside the row on every lane: its
// accesses need no test.  (Layouts of 6 or 8 vectors may end in vectors past
// d; all their vectors are tested.)
template <int VEC, int NV>
__host__ __device__ constexpr bool head_vector(int i) {
  return NV <= 4 && i < NV - 1;
}
// Vector i of a lane starting at element e: wholly inside a row of d elements.
template <int VEC, int NV>
__device__ __forceinline__ bool vec_whole(int i, int e, int d) {
  return head_vector<VEC, NV>(i) || e + VEC <= d;
}
// ... starting inside it.
template <int VEC, int NV>
__device__ __forceinline__ bool vec_inside(int i, int e, int d) {
  return head_vector<VEC, NV>(i) || e < d;
}
// The tail vectors of rows of several vectors per lane lie wholly inside the
// row on some lanes and wholly past it on the others (unless d is not a
// multiple of VEC, when one lane straddles it).  A lane accesses such a vector
// whole or not at all under a predicate instead of a branch that would split
// the warp; only a straddling lane takes the element path.
template <int VEC, int NV>
__device__ __forceinline__ bool vec_predicated(int i, int e, int d) {
  return NV > 1 && !head_vector<VEC, NV>(i) && (e >= d || e + VEC <= d);
}

// Predicated stores and reductions: `on` selects whether the access happens.
__device__ __forceinline__ void st_shared_u32x2_if(uint32_t a, uint32_t x, uint32_t y, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q st.shared.v2.b32 [%0], {%1,%2};\n\t}" ::"r"(a),
               "r"(x), "r"(y), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void st_shared_u32_if(uint32_t a, uint32_t x, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.shared.b32 [%0], %1;\n\t}" ::"r"(a), "r"(x),
               "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void st_global_cg_f32x4_if(float* p, float x, float y, float z, float w, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t@q st.global.cg.v4.f32 [%0], {%1,%2,%3,%4};\n\t}" ::"l"(p),
               "f"(x), "f"(y), "f"(z), "f"(w), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void st_global_cg_f32x2_if(float* p, float x, float y, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q st.global.cg.v2.f32 [%0], {%1,%2};\n\t}" ::"l"(p),
               "f"(x), "f"(y), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void st_global_cg_u32x2_if(void* p, uint32_t x, uint32_t y, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q st.global.cg.v2.b32 [%0], {%1,%2};\n\t}" ::"l"(p),
               "r"(x), "r"(y), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void st_global_cg_u32_if(void* p, uint32_t x, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.cg.b32 [%0], %1;\n\t}" ::"l"(p), "r"(x),
               "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void red_add_f32x4_if(float* p, float x, float y, float z, float w, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t@q red.global.add.v4.f32 [%0], {%1,%2,%3,%4};\n\t}" ::"l"(p),
               "f"(x), "f"(y), "f"(z), "f"(w), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void red_add_f32x2_if(float* p, float x, float y, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q red.global.add.v2.f32 [%0], {%1,%2};\n\t}" ::"l"(p),
               "f"(x), "f"(y), "r"((int)on)
               : "memory");
}
__device__ __forceinline__ void red_add_bf16x2x2_if(void* p, uint32_t x, uint32_t y, bool on) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q red.global.add.noftz.v2.bf16x2 [%0], {%1,%2};\n\t}" ::"l"(p),
      "r"(x), "r"(y), "r"((int)on)
      : "memory");
}
__device__ __forceinline__ void red_add_bf16x2_if(void* p, uint32_t x, bool on) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q red.global.add.noftz.bf16x2 [%0], %1;\n\t}" ::"l"(p),
               "r"(x), "r"((int)on)
               : "memory");
}

template <int VEC, int NV>
struct LaneMap {
  uint32_t off[NV];  // byte offset of this lane's vector i within a row
  bool ok[NV];       // vector i starts inside the row (e < d)
  uint32_t zero;     // a 16-byte zero vector in shared memory, read in place of vectors past d
  __device__ __forceinline__ LaneMap(int lane, int d, uint32_t zero_b) : zero(zero_b) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      const int e = (i * 32 + lane) * VEC;
      off[i] = (uint32_t)e * 4u;
      ok[i] = head_vector<VEC, NV>(i) || e < d;
    }
  }
  // shared-memory address of vector i of a row for a load: the zero vector
  // past d
  __device__ __forceinline__ uint32_t ld_addr(uint32_t row, int i) const {
    if (head_vector<VEC, NV>(i)) return row + off[i];
    return ok[i] ? row + off[i] : zero;
  }
};

// A row staged by a bulk copy holds the table row's padding past d; the one
// lane whose vector straddles d (d not a multiple of VEC) clears it.
template <int VEC, int NV>
__device__ __forceinline__ void clear_past_d(Row<VEC, NV>& r, const LaneMap<VEC, NV>& m, int d) {
  if ((d & (VEC - 1)) == 0) return;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (int)(m.off[i] / 4);
    if (e < d && e + VEC > d) {
#pragma unroll
      for (int j = 0; j < VEC; j++)
        if (e + j >= d) r.x[i][j] = 0.0f;
    }
  }
}

// Rows of one vector per lane (d <= 128) test the lane with a branch, which
// is the same on every lane when d fills the warp.  The last vector of wider
// rows, which ends inside the row on some lanes only, is loaded from the zero
// vector and stored under a predicate instead: a branch that splits the warp
// costs more than the select.
template <int VEC, int NV>
__device__ __forceinline__ void lds_row(Row<VEC, NV>& r, uint32_t row, const LaneMap<VEC, NV>& m) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    if constexpr (VEC == 4) {
      if (NV == 1 && !m.ok[i]) {
        r.x[i][0] = r.x[i][1] = r.x[i][2] = r.x[i][3] = 0.0f;
        continue;
      }
      asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                   : "=f"(r.x[i][0]), "=f"(r.x[i][1]), "=f"(r.x[i][2]), "=f"(r.x[i][3])
                   : "r"(m.ld_addr(row, i)));
    } else {
      if (NV == 1 && !m.ok[i]) {
        r.x[i][0] = r.x[i][1] = 0.0f;
        continue;
      }
      asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(r.x[i][0]), "=f"(r.x[i][1]) : "r"(m.ld_addr(row, i)));
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ void sts_row(const Row<VEC, NV>& r, uint32_t row, const LaneMap<VEC, NV>& m) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const uint32_t a = row + m.off[i];
    if (head_vector<VEC, NV>(i) || NV == 1) {
      if (NV == 1 && !m.ok[i]) continue;
      if constexpr (VEC == 4)
        asm volatile("st.shared.v4.f32 [%0], {%1,%2,%3,%4};" ::"r"(a), "f"(r.x[i][0]), "f"(r.x[i][1]),
                     "f"(r.x[i][2]), "f"(r.x[i][3])
                     : "memory");
      else
        asm volatile("st.shared.v2.f32 [%0], {%1,%2};" ::"r"(a), "f"(r.x[i][0]), "f"(r.x[i][1]) : "memory");
    } else {
      const int on = m.ok[i];
      if constexpr (VEC == 4)
        asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t@q st.shared.v4.f32 [%0], {%1,%2,%3,%4};\n\t}"
                     ::"r"(a), "f"(r.x[i][0]), "f"(r.x[i][1]), "f"(r.x[i][2]), "f"(r.x[i][3]), "r"(on)
                     : "memory");
      else
        asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q st.shared.v2.f32 [%0], {%1,%2};\n\t}"
                     ::"r"(a), "f"(r.x[i][0]), "f"(r.x[i][1]), "r"(on)
                     : "memory");
    }
  }
}

// Global -> shared copy of this lane's part of a row without a register
// round trip (cp.async, 16 or 8 bytes per vector); complete with cp_async_wait.
template <int VEC, int NV>
__device__ __forceinline__ void cp_row(uint32_t dst, const float* src, const LaneMap<VEC, NV>& m, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e0 = (int)(m.off[i] / 4);
    if (vec_predicated<VEC, NV>(i, e0, d)) {
      // whole, or nothing on lanes past d (their loads read the zero vector)
      const uint32_t da = dst + m.off[i];
      const float* g = src + e0;
      if constexpr (VEC == 4)
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %2, 0; @p cp.async.cg.shared.global [%0], [%1], 16; }"
                     ::"r"(da), "l"(g), "r"((int)(e0 < d)) : "memory");
      else
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %2, 0; @p cp.async.ca.shared.global [%0], [%1], 8; }"
                     ::"r"(da), "l"(g), "r"((int)(e0 < d)) : "memory");
    } else if (m.ok[i]) {
      const float* g = src + m.off[i] / 4;
      if (vec_whole<VEC, NV>(i, (int)(m.off[i] / 4), d)) {
        if constexpr (VEC == 4)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + m.off[i]), "l"(g) : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst + m.off[i]), "l"(g) : "memory");
      } else {
        // a vector that straddles d: element copies, zeros past d
#pragma unroll
        for (int j = 0; j < VEC; j++) {
          const int e = (int)(m.off[i] / 4) + j;
          if (e < d)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst + m.off[i] + 4 * j), "l"(g + j)
                         : "memory");
          else
            asm volatile("st.shared.f32 [%0], %1;" ::"r"(dst + m.off[i] + 4 * j), "f"(0.0f) : "memory");
        }
      }
    }
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// All but the most recently committed group complete.
__device__ __forceinline__ void cp_async_wait_but_last() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Bulk copies (cp.async.bulk, the async proxy; non-multicast, this GPU's own
// memory only) of whole staged rows, issued by one lane.  Loads complete on
// a per-warp mbarrier (transaction bytes); stores are bulk groups.
__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of the barrier, at most kBulkWaitTries tries
// (each try suspends the thread for a bounded time): false if it gave up.
constexpr int kBulkWaitTries = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < kBulkWaitTries; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// The bulk stores' reads of shared memory are done / all but the latest
// group's stores are complete / all are complete.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_but_last() { asm volatile("cp.async.bulk.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic-proxy accesses (shared and global) with
// async-proxy accesses on either side of it.
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async;" ::: "memory"); }

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
    if (vec_predicated<VEC, NV>(i, e, d)) {
      const bool on = e < d;
      const float* g = row + (on ? e : 0);
      if constexpr (VEC == 4) {
        const float4 t = __ldcg(reinterpret_cast<const float4*>(g));
        r.x[i][0] = on ? t.x : 0.0f; r.x[i][1] = on ? t.y : 0.0f;
        r.x[i][2] = on ? t.z : 0.0f; r.x[i][3] = on ? t.w : 0.0f;
      } else {
        const float2 t = __ldcg(reinterpret_cast<const float2*>(g));
        r.x[i][0] = on ? t.x : 0.0f; r.x[i][1] = on ? t.y : 0.0f;
      }
    } else if (vec_whole<VEC, NV>(i, e, d)) {
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
    if (vec_inside<VEC, NV>(i, e, d)) {
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
    if (vec_inside<VEC, NV>(i, e, d)) {
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
    if (vec_predicated<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4)
        red_add_f32x4_if(row + e, __fsub_rn(a.x[i][0], b.x[i][0]), __fsub_rn(a.x[i][1], b.x[i][1]),
                         __fsub_rn(a.x[i][2], b.x[i][2]), __fsub_rn(a.x[i][3], b.x[i][3]), e < d);
      else
        red_add_f32x2_if(row + e, __fsub_rn(a.x[i][0], b.x[i][0]), __fsub_rn(a.x[i][1], b.x[i][1]), e < d);
    } else if (vec_whole<VEC, NV>(i, e, d)) {
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

// ---- bfloat16 tables: FP32 math, rows converted on load, stochastic-rounded
// write-back.  The table type only changes these helpers; everything between
// a row's load and its write-back is FP32. ----
using bf16_t = __nv_bfloat16;

template <int VEC, int NV>
__device__ __forceinline__ void row_load_global(Row<VEC, NV>& r, const bf16_t* row, int lane, int d) {
  const uint16_t* h = reinterpret_cast<const uint16_t*>(row);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (vec_predicated<VEC, NV>(i, e, d)) {
      const bool on = e < d;
      const uint16_t* g = h + (on ? e : 0);
      if constexpr (VEC == 4) {
        uint2 t = __ldcg(reinterpret_cast<const uint2*>(g));
        t.x = on ? t.x : 0u;
        t.y = on ? t.y : 0u;
        r.x[i][0] = bf16_value((uint16_t)t.x); r.x[i][1] = bf16_value((uint16_t)(t.x >> 16));
        r.x[i][2] = bf16_value((uint16_t)t.y); r.x[i][3] = bf16_value((uint16_t)(t.y >> 16));
      } else {
        unsigned t = __ldcg(reinterpret_cast<const unsigned*>(g));
        t = on ? t : 0u;
        r.x[i][0] = bf16_value((uint16_t)t); r.x[i][1] = bf16_value((uint16_t)(t >> 16));
      }
    } else if (vec_whole<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4) {
        const uint2 t = __ldcg(reinterpret_cast<const uint2*>(h + e));
        r.x[i][0] = bf16_value((uint16_t)t.x); r.x[i][1] = bf16_value((uint16_t)(t.x >> 16));
        r.x[i][2] = bf16_value((uint16_t)t.y); r.x[i][3] = bf16_value((uint16_t)(t.y >> 16));
      } else {
        const unsigned t = __ldcg(reinterpret_cast<const unsigned*>(h + e));
        r.x[i][0] = bf16_value((uint16_t)t); r.x[i][1] = bf16_value((uint16_t)(t >> 16));
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++) r.x[i][j] = e + j < d ? bf16_value(__ldcg(h + e + j)) : 0.0f;
    }
  }
}

// bfloat16 write-back of a row that moved from b (its value when loaded) to a
// (FP32): s = the stochastic rounding of a (bf16_stochastic, 16 random bits
// per element from the event key), and the increment s - b, rounded to
// bfloat16, is added to the stored row with the hardware's fire-and-forget
// bfloat16 reduction (red.add.noftz: exact sum rounded to nearest even,
// subnormals kept).  s - b is a multiple of the finer of the two values' ulps,
// so it is exact in bfloat16 unless the change exceeds 255 of them; then, when
// no other writer touched the row since the load, the stored value becomes s
// exactly.  Concurrent writers never lose each other's updates.
__device__ __forceinline__ uint32_t sr_increment2(float a0, float b0, float a1, float b1, uint32_t r32) {
  // s - b for both elements with one packed FP32x2 add (s + (-b), exact as s - b)
  const float2 x = __fadd2_rn(make_float2(bf16_stochastic_value(a0, r32 & 0xFFFFu), bf16_stochastic_value(a1, r32 >> 16)),
                              make_float2(-b0, -b1));
  const __nv_bfloat162 v = __floats2bfloat162_rn(x.x, x.y);  // element 0 in the low half (lower address)
  return *reinterpret_cast<const uint32_t*>(&v);
}

template <int VEC, int NV>
__device__ __forceinline__ void row_add_delta(bf16_t* row, const Row<VEC, NV>& a, const Row<VEC, NV>& b, int lane,
                                              int d, uint64_t key, uint64_t row_id) {
  uint16_t* h = reinterpret_cast<uint16_t*>(row);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (vec_predicated<VEC, NV>(i, e, d)) {
      const uint64_t bits = sr_vector_bits(key, row_id, (uint64_t)(e / VEC));
      const uint32_t p0 = sr_increment2(a.x[i][0], b.x[i][0], a.x[i][1], b.x[i][1], (uint32_t)bits);
      if constexpr (VEC == 4) {
        const uint32_t p1 = sr_increment2(a.x[i][2], b.x[i][2], a.x[i][3], b.x[i][3], (uint32_t)(bits >> 32));
        red_add_bf16x2x2_if(h + e, p0, p1, e < d);
      } else {
        red_add_bf16x2_if(h + e, p0, e < d);
      }
      continue;
    }
    if (!vec_inside<VEC, NV>(i, e, d)) continue;
    const uint64_t bits = sr_vector_bits(key, row_id, (uint64_t)(e / VEC));
    if (vec_whole<VEC, NV>(i, e, d)) {
      const uint32_t p0 = sr_increment2(a.x[i][0], b.x[i][0], a.x[i][1], b.x[i][1], (uint32_t)bits);
      if constexpr (VEC == 4) {
        const uint32_t p1 = sr_increment2(a.x[i][2], b.x[i][2], a.x[i][3], b.x[i][3], (uint32_t)(bits >> 32));
        asm volatile("red.global.add.noftz.v2.bf16x2 [%0], {%1, %2};" ::"l"(h + e), "r"(p0), "r"(p1) : "memory");
      } else {
        asm volatile("red.global.add.noftz.bf16x2 [%0], %1;" ::"l"(h + e), "r"(p0) : "memory");
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        if (e + j >= d) continue;
        const uint32_t r16 = (uint32_t)(bits >> (16 * j)) & 0xFFFFu;
        const float x = __fsub_rn(bf16_stochastic_value(a.x[i][j], r16), b.x[i][j]);
        const __nv_bfloat16 v = __float2bfloat16_rn(x);
        const unsigned short u = *reinterpret_cast<const unsigned short*>(&v);
        asm volatile("red.global.add.noftz.bf16 [%0], %1;" ::"l"(h + e + j), "h"(u) : "memory");
      }
    }
  }
}

// The FP32 table takes exact atomic adds; the key is unused.
template <int VEC, int NV>
__device__ __forceinline__ void row_add_delta(float* row, const Row<VEC, NV>& a, const Row<VEC, NV>& b, int lane,
                                              int d, uint64_t, uint64_t) {
  row_add_delta(row, a, b, lane, d);
}

// Lane partial of a dot product as two independent running sums, "even" and
// "odd" (elements j and j+1 of every vector, j even), each a product then
// FMAs in vector order, in sm_100's packed FP32x2 FMA (two IEEE
// single-rounding FMAs per instruction); the lane's partial is even + odd.
// Two chains halve the dependent latency of the dot, which sits on the
// critical path of every pipeline step.
template <int VEC, int NV>
__device__ __forceinline__ float row_dot(const Row<VEC, NV>& a, const Row<VEC, NV>& b) {
  float2 p = __fmul2_rn(make_float2(a.x[0][0], a.x[0][1]), make_float2(b.x[0][0], b.x[0][1]));
#pragma unroll
  for (int i = 0; i < NV; i++)
#pragma unroll
    for (int j = 0; j < VEC; j += 2)
      if (i != 0 || j != 0)
        p = __ffma2_rn(make_float2(a.x[i][j], a.x[i][j + 1]), make_float2(b.x[i][j], b.x[i][j + 1]), p);
  return __fadd_rn(p.x, p.y);
}

__device__ __forceinline__ float warp_sum(float p) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) p = __fadd_rn(p, __shfl_xor_sync(kFull, p, m));
  return p;
}

// v += g*o and o += g*v_old, elementwise with single-rounding FMAs.  (Scalar
// FMAs issue to both FP32 pipes; the packed FP32x2 form, which runs on one,
// measured 4% slower here.)
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
// reversed table (nexpTable[i] == expTable[999 - i]).  `table` is the block's
// shared-memory copy.
template <int SIG>
__device__ __forceinline__ float gradient(float x, bool positive, float alpha, const float* table) {
  if constexpr (SIG == 0) {
    const float s = __saturatef(__fmul_rn(__fadd_rn(x, 6.0f), 1.0f / 12.0f));
    const int idx = __float2int_rz(__fmul_rn(s, 999.0f));
    return positive ? __fmul_rn(alpha, table[kExpTableSize - 1 - idx]) : __fmul_rn(-alpha, table[idx]);
  }
  return positive ? __fdiv_rn(alpha, __fadd_rn(1.0f, expf(x)))
                  : __fdiv_rn(-alpha, __fadd_rn(1.0f, expf(-x)));
}

// The table-mode gradient of a pipeline stage with its constant parts folded
// in ahead of the step, so that the dependent chain from the dot product to g
// is FADD, FMUL (saturating), FMUL, FADD, IMAD, shared-memory load, FMUL:
//   * the truncation (int)y of y = s * 999 in [0, 999] is read from the bits
//     of y + 2^23 added toward zero: 0x4B000000 + (int)y;
//   * the entry address is a + b * bits (32-bit wrap-around), with b = 4 and
//     a = table - 4 * 0x4B000000 for a negative target, b = -4 and
//     a = table + 4 * 999 + 4 * 0x4B000000 for the positive one (which reads
//     the table reversed);
//   * alpha_k is alpha (positive), -alpha (negative) or 0 (an idle stage:
//     g = +0 exactly as a skipped step).
// The result is bit-identical to gradient<0>.
struct TableStage {
  uint32_t a, b;
};
__device__ __forceinline__ TableStage table_stage(uint32_t table_b, bool positive) {
  TableStage t;
  t.b = positive ? (uint32_t)-4 : 4u;
  t.a = positive ? table_b + 4u * (uint32_t)(kExpTableSize - 1) + 4u * 0x4B000000u : table_b - 4u * 0x4B000000u;
  return t;
}
__device__ __forceinline__ float table_gradient(float x, const TableStage& t, float alpha_k) {
  const float s = __saturatef(__fmul_rn(__fadd_rn(x, 6.0f), 1.0f / 12.0f));
  const float y = __fadd_rz(__fmul_rn(s, 999.0f), 8388608.0f);
  float e;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(e) : "r"(t.a + t.b * __float_as_uint(y)));
  return __fmul_rn(alpha_k, e);
}

struct Sentence {
  int64_t start;
  int32_t len;
  float alpha;
  int64_t uid;  // the sentence's number in its launch (stochastic-rounding key)
};

__device__ __forceinline__ int64_t total_sentences(const TrainParams& p) {
  if (p.source == kSourceEpoch) return p.entry_prefix[p.threads];
  return p.n_sentences;
}

__device__ __forceinline__ Sentence fetch_sentence(const TrainParams& p, int64_t w) {
  Sentence s;
  s.uid = w;
  if (p.source == kSourceEpoch) {
    int lo = 0, hi = p.threads - 1;  // last stream with prefix <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.entry_prefix[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const int64_t slot = entry_base(p.stream_base, lo) + (w - p.entry_prefix[lo]);
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

template <int VEC, int NV>
__device__ __forceinline__ void row_store_global(const Row<VEC, NV>& r, float* row, int lane, int d) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (vec_predicated<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4)
        st_global_cg_f32x4_if(row + e, r.x[i][0], r.x[i][1], r.x[i][2], r.x[i][3], e < d);
      else
        st_global_cg_f32x2_if(row + e, r.x[i][0], r.x[i][1], e < d);
    } else if (vec_inside<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4) {
        __stcg(reinterpret_cast<float4*>(row + e), make_float4(r.x[i][0], r.x[i][1], r.x[i][2], r.x[i][3]));
      } else {
        __stcg(reinterpret_cast<float2*>(row + e), make_float2(r.x[i][0], r.x[i][1]));
      }
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ void row_store_global(const Row<VEC, NV>& r, bf16_t* row, int lane, int d) {
  uint16_t* h = reinterpret_cast<uint16_t*>(row);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e = (i * 32 + lane) * VEC;
    if (vec_predicated<VEC, NV>(i, e, d)) {
      const uint32_t x = (unsigned)bf16_nearest(r.x[i][0]) | ((unsigned)bf16_nearest(r.x[i][1]) << 16);
      if constexpr (VEC == 4) {
        const uint32_t y = (unsigned)bf16_nearest(r.x[i][2]) | ((unsigned)bf16_nearest(r.x[i][3]) << 16);
        st_global_cg_u32x2_if(h + e, x, y, e < d);
      } else {
        st_global_cg_u32_if(h + e, x, e < d);
      }
    } else if (vec_whole<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4) {
        uint2 t;
        t.x = (unsigned)bf16_nearest(r.x[i][0]) | ((unsigned)bf16_nearest(r.x[i][1]) << 16);
        t.y = (unsigned)bf16_nearest(r.x[i][2]) | ((unsigned)bf16_nearest(r.x[i][3]) << 16);
        __stcg(reinterpret_cast<uint2*>(h + e), t);
      } else {
        __stcg(reinterpret_cast<unsigned*>(h + e),
               (unsigned)bf16_nearest(r.x[i][0]) | ((unsigned)bf16_nearest(r.x[i][1]) << 16));
      }
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++)
        if (e + j < d) h[e + j] = bf16_nearest(r.x[i][j]);
    }
  }
}

// Staging copies of a bfloat16 row keep its 2-byte elements (byte offset e*2).
template <int VEC, int NV>
__device__ __forceinline__ void cp_row(uint32_t dst, const bf16_t* src, const LaneMap<VEC, NV>& m, int d) {
  const uint16_t* h = reinterpret_cast<const uint16_t*>(src);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    const int e0 = (int)(m.off[i] / 4);
    if (vec_predicated<VEC, NV>(i, e0, d)) {
      // whole, or nothing on lanes past d (their loads read the zero vector)
      const uint32_t da = dst + (uint32_t)e0 * 2u;
      const uint16_t* g = h + e0;
      if constexpr (VEC == 4)
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %2, 0; @p cp.async.ca.shared.global [%0], [%1], 8; }"
                     ::"r"(da), "l"(g), "r"((int)(e0 < d)) : "memory");
      else
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %2, 0; @p cp.async.ca.shared.global [%0], [%1], 4; }"
                     ::"r"(da), "l"(g), "r"((int)(e0 < d)) : "memory");
      continue;
    }
    if (!m.ok[i]) continue;
    const int e = e0;
    const uint32_t da = dst + (uint32_t)e * 2u;
    if (vec_whole<VEC, NV>(i, e, d)) {
      if constexpr (VEC == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(da), "l"(h + e) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(da), "l"(h + e) : "memory");
    } else {
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        const unsigned short v = e + j < d ? __ldcg(h + e + j) : (unsigned short)0;
        asm volatile("st.shared.u16 [%0], %1;" ::"r"(da + 2u * j), "h"(v) : "memory");
      }
    }
  }
}

template <int VEC, int NV>
__device__ __forceinline__ void lds_row_bf16(Row<VEC, NV>& r, uint32_t row, const LaneMap<VEC, NV>& m) {
#pragma unroll
  for (int i = 0; i < NV; i++) {
    unsigned a = 0, b = 0;
    if (NV > 1 || m.ok[i]) {
      const uint32_t at = head_vector<VEC, NV>(i) || m.ok[i] ? row + (m.off[i] / 4) * 2u : m.zero;
      if constexpr (VEC == 4) asm volatile("ld.shared.v2.u32 {%0,%1}, [%2];" : "=r"(a), "=r"(b) : "r"(at));
      else asm volatile("ld.shared.u32 %0, [%1];" : "=r"(a) : "r"(at));
    }
    r.x[i][0] = bf16_value((uint16_t)a);
    r.x[i][1] = bf16_value((uint16_t)(a >> 16));
    if constexpr (VEC == 4) {
      r.x[i][2] = bf16_value((uint16_t)b);
      r.x[i][3] = bf16_value((uint16_t)(b >> 16));
    }
  }
}

// A staging row written by cp_row, in the table's element type.
template <typename T, int VEC, int NV>
__device__ __forceinline__ void lds_staged(Row<VEC, NV>& r, uint32_t row, const LaneMap<VEC, NV>& m) {
  if constexpr (std::is_same_v<T, float>) lds_row(r, row, m);
  else lds_row_bf16(r, row, m);
}

// A row into a staging row of the table's element type; with bfloat16 tables
// the values must be bfloat16 already (rows as loaded from a table), so
// keeping their top 16 bits is exact.
template <typename T, int VEC, int NV>
__device__ __forceinline__ void sts_staged(const Row<VEC, NV>& r, uint32_t row, const LaneMap<VEC, NV>& m) {
  if constexpr (std::is_same_v<T, float>) {
    sts_row(r, row, m);
  } else {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      const bool pred = NV > 1 && !head_vector<VEC, NV>(i);  // stored under a predicate, no branch
      if (!pred && !m.ok[i]) continue;
      const uint32_t at = row + (m.off[i] / 4) * 2u;
      const uint32_t a = __byte_perm(__float_as_uint(r.x[i][0]), __float_as_uint(r.x[i][1]), 0x7632);
      if constexpr (VEC == 4) {
        const uint32_t b = __byte_perm(__float_as_uint(r.x[i][2]), __float_as_uint(r.x[i][3]), 0x7632);
        if (pred) st_shared_u32x2_if(at, a, b, m.ok[i]);
        else asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(at), "r"(a), "r"(b) : "memory");
      } else {
        if (pred) st_shared_u32_if(at, a, m.ok[i]);
        else asm volatile("st.shared.u32 [%0], %1;" ::"r"(at), "r"(a) : "memory");
      }
    }
  }
}

// Shared memory of one warp, rows of `pitch` elements: the FP32 ring of
// D = 2W+1 rows and a sink row, then staged rows of the table's element type
// (R target originals, 2 x R with the target prefetch, and 2 staging rows),
// then a 16-byte zero vector and the 16-byte slot of the warp's mbarrier.
__host__ __device__ constexpr int64_t warp_smem_bytes(int D, int R, bool prefetch, int64_t pitch, int elem) {
  return (int64_t)(D + 1) * pitch * 4 + (int64_t)((prefetch ? 2 : 1) * R + 2) * pitch * elem + 32;
}

// The warp's mbarrier in the last 16 bytes of its shared-memory region of
// region_bytes, initialised once per kernel (an mbarrier is not
// re-initialised while the warp uses it): returns its address.
__device__ __forceinline__ uint32_t warp_bulk_init(const float* region, uint32_t region_bytes, int lane) {
  const uint32_t bar = smem_addr(region) + region_bytes - 16u;
  if (lane == 0) {
    mbar_init(bar);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncwarp();
  return bar;
}

// One sentence on one warp.
//   ring     shared memory (warp_smem_bytes): slot p % D holds the current
//            value of sentence position p while it is in the window; slot D
//            is a sink that the pipeline reads and writes on its idle steps;
//            then the R target rows as loaded (for their write-back), two
//            staging rows filled by bulk copies (the entering row and the
//            leaving row's original value), the zero vector that lanes read in
//            place of vectors past d.
//   orig     this warp's global scratch, D rows: the value each slot's row had
//            when it entered the window (needed for its single write-back).
// Returns false if a bulk copy did not complete in time (the error word is
// set to 2): the warp then stops.
//   bar_b    the warp's mbarrier (initialised once per kernel by warp_bulk_init)
//            and bar_phase its phase parity, carried from sentence to sentence.
template <typename T, int VEC, int NV, int R, int SIG>
__device__ bool train_sentence(const TrainParams& p, const Sentence& sn, float* ring, T* orig,
                               const float* table, int lane, uint32_t bar_b, uint32_t& bar_phase) {
  constexpr int RP = PadPow2<R>::value;
  const int W = p.window, K = p.negative, D = 2 * W + 1;
  const int P = (int)p.pitch;  // row stride, global and shared
  const int d = p.d;
  const int L = sn.len;
  const int32_t* ids = p.ids + sn.start;
  const int32_t* negs = p.negs + sn.start * (int64_t)K;
  T* const syn0 = reinterpret_cast<T*>(p.syn0);
  T* const syn1neg = reinterpret_cast<T*>(p.syn1neg);
  const float alpha = sn.alpha;
  const bool one_group = K + 1 <= R;
  const bool pre = p.prefetch != 0;  // target rows copied one group of targets ahead
  // context rows staged by bulk copies (lane 0, mbarrier) instead of per-lane cp.async
  const bool bulk = p.bulk != 0;
  const uint64_t skey = sr_sentence_key(p.sr_seed, (uint64_t)sn.uid);  // bfloat16 tables only

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
    return true;
  }
  if (L <= 0) return true;

  Row<VEC, NV> tmp;
  const int n_enter = W + 1 < L ? W + 1 : L;
  for (int q = 0; q < n_enter; q++) {
    row_load_global(tmp, syn0 + (int64_t)__ldg(ids + q) * P, lane, d);
    row_store_smem(tmp, ring + q * P, lane, d);
    row_store_global(tmp, orig + q * P, lane, d);
  }
  const uint32_t ring_b = smem_addr(ring);
  const uint32_t table_b = smem_addr(table);  // the block's shared copy of the sigmoid table
  const uint32_t row_bytes = (uint32_t)P * 4u;
  // staged rows (target originals, entering and leaving copies) hold the
  // table's element type: half size with bfloat16 tables
  const uint32_t srow_bytes = (uint32_t)P * (uint32_t)sizeof(T);
  const uint32_t sink_b = ring_b + (uint32_t)D * row_bytes;
  // Target rows, in the table's element type.  With the prefetch, two sets of
  // R rows: the rows of each group of targets (R of a centre's 1 + K, in
  // centre order) are copied (cp.async, each lane its own elements) into one
  // set while the previous group trains, and stay there as the originals for
  // the write-back.  Otherwise one set holds the originals of the current
  // group, loaded when it starts.
  const uint32_t o0_b = sink_b + row_bytes;
  const uint32_t o1_b = o0_b + (uint32_t)R * srow_bytes;
  const uint32_t in_b = pre ? o1_b + (uint32_t)R * srow_bytes : o1_b;
  const uint32_t out_b = in_b + srow_bytes;
  const uint32_t zero_b = out_b + srow_bytes;
  // The entering row and the leaving row's original arrive by bulk copies
  // (lane 0) that complete on the warp's mbarrier, one phase per centre that
  // has any; the entering row goes on to the originals scratch by a bulk store.
  int last_store_slot = -1;  // the slot whose original the latest bulk store wrote
  if (lane < 4) asm volatile("st.shared.f32 [%0], %1;" ::"r"(zero_b + 4u * lane), "f"(0.0f) : "memory");
  __syncwarp();
  const LaneMap<VEC, NV> lm(lane, d, zero_b);
  auto prefetch_targets = [&](uint32_t set, int my_target, int n) {
    for (int k = 0; k < n; k++) {
      const int tk = __shfl_sync(kFull, my_target, k);
      cp_row(set + (uint32_t)k * srow_bytes, syn1neg + (int64_t)tk * P, lm, d);
    }
  };

  // v[r] holds the context row whose index j in the centre's list has
  // j % R == r: stage k works on context t-k at step t, i.e. on register slot
  // (t - k) % R, so a row moves from stage to stage without being copied.
  Row<VEC, NV> v[R], o[R];
  uint32_t voff[R];
#pragma unroll
  for (int k = 0; k < R; k++) {
    row_zero(v[k]);
    voff[k] = sink_b;
  }

  int t_next = one_group ? target_id(ids, negs, K, 0, 0, K + 1, lane) : 0;
  // cp.async commit groups with the prefetch: the first group's rows before
  // the loop, then at every centre its staging copies (Enter) and at every
  // group of targets the next group's rows.
  const int nt0 = K + 1 < R ? K + 1 : R;
  uint32_t cur_b = o0_b;  // the set holding the rows of the group about to train
  if (pre) {
    if (L >= 2) prefetch_targets(o0_b, target_id(ids, negs, K, 0, 0, nt0, lane), nt0);
    cp_async_commit();
  }
  int t_prev = -1;  // lane k < R: target k of the previous group of targets (written back), else -1
  // The ring slot of position w - W, which leaves at centre w and whose slot
  // position w + W + 1 takes ((w - W) mod D), and on lane r < D the offset of
  // slot r from it ((r - (w - W)) mod D): both move by one slot per centre.
  int slot_out = W + 1 < D ? W + 1 : 0;
  int lane_off = lane + W < D ? lane + W : lane + W - D;
  for (int w = 0; w < L; w++) {
    // Ids and rows needed later in this centre, loaded ahead of use.
    const int q_out = w - W, q_in = w + W + 1;
    const int id_out = q_out >= 0 ? __ldg(ids + q_out) : -1;
    const int id_in = q_in < L ? __ldg(ids + q_in) : -1;
    const int t_here = t_next;
    if (one_group && w + 1 < L) t_next = target_id(ids, negs, K, w + 1, 0, K + 1, lane);
    // The entering row can be fetched now unless the leaving position holds
    // the same word (its write-back must land first).  Both staging copies run
    // in the background while the centre trains.
    const bool enter_early = id_in >= 0 && id_in != id_out;
    const uint32_t stage_bytes = bulk ? (enter_early ? srow_bytes : 0u) + (q_out >= 0 ? srow_bytes : 0u) : 0u;
    if (!bulk) {
      if (enter_early) cp_row(in_b, syn0 + (int64_t)id_in * P, lm, d);
      if (q_out >= 0) cp_row(out_b, orig + slot_out * P, lm, d);
      cp_async_commit();
    } else if (stage_bytes) {
      // every lane's generic accesses so far (its reads of the staging rows,
      // its stores and write-backs to the tables and the originals scratch)
      // before the async-proxy copies
      proxy_fence();
      __syncwarp();
      if (lane == 0) {
        // the last bulk store has read the entering row's staging row, and
        // the leaving row's original is written: every store but the latest
        // is complete, and the latest too if it was this slot's
        if (q_out >= 0 && slot_out == last_store_slot) bulk_wait_all();
        else bulk_wait_but_last();
        bulk_wait_read();
        mbar_expect_tx(bar_b, stage_bytes);
        if (enter_early) bulk_load(in_b, syn0 + (int64_t)id_in * P, srow_bytes, bar_b);
        if (q_out >= 0) bulk_load(out_b, orig + slot_out * P, srow_bytes, bar_b);
      }
    }

    // Lane r < D decides whether ring slot r holds a context of centre w.
    const int base = w - W;
    bool valid = false;
    if (lane < D) {
      const int pos = base + lane_off;
      valid = pos != w && pos >= 0 && pos < L;
    }
    const unsigned mask = __ballot_sync(kFull, valid);
    const int nctx = __popc(mask);

    int prefetches = 0;  // groups committed after this centre's staging copies
    if (nctx > 0) {
      for (int k0 = 0; k0 <= K; k0 += R) {
        const int nt = (K + 1 - k0) < R ? (K + 1 - k0) : R;
        const int my_t = one_group ? t_here : target_id(ids, negs, K, w, k0, nt, lane);
        if (pre) {
          // This group's rows: committed before this centre's staging copies
          // (per-lane staging) for its first group, else the latest group.
          if (k0 == 0 && !bulk) cp_async_wait_but_last();
          else cp_async_wait();
          // A row copied before the previous group's write-back of the same
          // target is fetched again (after this lane's own reduction, in
          // program order).
          // Lane k < nt compares its target with the previous group's.
          bool stale = false;
#pragma unroll
          for (int j = 0; j < R; j++) stale |= __shfl_sync(kFull, t_prev, j) == my_t;
          unsigned stale_mask = __ballot_sync(kFull, stale && lane < nt);
          if (stale_mask) {
            while (stale_mask) {
              const int k = __ffs(stale_mask) - 1;
              stale_mask &= stale_mask - 1;
              const int tk = __shfl_sync(kFull, my_t, k);
              cp_row(cur_b + (uint32_t)k * srow_bytes, syn1neg + (int64_t)tk * P, lm, d);
            }
            cp_async_commit();
            cp_async_wait();
          }
          // the next group's rows, into the other set
          const uint32_t nxt_b = cur_b == o0_b ? o1_b : o0_b;
          if (k0 + R <= K) {
            const int nt1 = (K + 1 - k0 - R) < R ? (K + 1 - k0 - R) : R;
            prefetch_targets(nxt_b, target_id(ids, negs, K, w, k0 + R, nt1, lane), nt1);
          } else if (w + 1 < L) {
            prefetch_targets(nxt_b, target_id(ids, negs, K, w + 1, 0, nt0, lane), nt0);
          }
          cp_async_commit();
          prefetches++;
        }
        bool dup = false;
        for (int j = 0; j + 1 < nt; j++) {
          const int tj = __shfl_sync(kFull, my_t, j);
          dup |= lane > j && lane < nt && tj == my_t;
        }
        if (!__any_sync(kFull, dup)) {
          // ---- pipelined sweeps of nt targets ----
          int tks[R];  // the group's target ids, on every lane
#pragma unroll
          for (int k = 0; k < R; k++) tks[k] = __shfl_sync(kFull, my_t, k);
#pragma unroll
          for (int k = 0; k < R; k++) {
            const int tk = tks[k];
            if (k < nt) {
              if (pre) {
                lds_staged<T>(o[k], cur_b + (uint32_t)k * srow_bytes, lm);
              } else {
                row_load_global(o[k], syn1neg + (int64_t)tk * P, lane, d);
                sts_staged<T>(o[k], o0_b + (uint32_t)k * srow_bytes, lm);
              }
            } else {
              row_zero(o[k]);
            }
          }
          const int my_stage = stage_of_lane<RP>(lane);
          const bool my_positive = k0 + my_stage == 0;
          const TableStage my_tab = table_stage(table_b, my_positive);
          const float my_alpha = my_positive ? alpha : -alpha;
          // the lane's stage is active at steps [my_stage, my_stage + nctx)
          const unsigned my_span = my_stage < nt ? (unsigned)nctx : 0u;
          unsigned rem = mask;
          const int steps = nctx + R - 1;
          for (int t0 = 0; t0 < steps; t0 += R) {
            static_for<R>([&](auto uc) {
              constexpr int u = decltype(uc)::value;
              const int ts = t0 + u;
              if (ts < steps) {
                // stage 0 takes the next context (the sink once they run out);
                // stage R-1 hands its row back (to the sink while ramping up)
                const int s0 = __ffs(rem) - 1;
                rem &= rem - 1;
                voff[u] = s0 >= 0 ? ring_b + (uint32_t)s0 * row_bytes : sink_b;
                lds_row(v[u], voff[u], lm);
                float x[RP];
                static_for<RP>([&](auto kc) {
                  constexpr int k = decltype(kc)::value;
                  if constexpr (k < R) x[k] = row_dot(v[(u - k + R) % R], o[k]);
                  else x[k] = 0.0f;
                });
                const float xs = transpose_reduce<RP>(x, lane);
                const bool act = (unsigned)(ts - my_stage) < my_span;
                float g;
                if constexpr (SIG == 0) g = table_gradient(xs, my_tab, act ? my_alpha : 0.0f);
                else g = act ? gradient<SIG>(xs, my_positive, alpha, table) : 0.0f;
                // every lane needs every stage's g; with two stages the other
                // half-warp holds the other one
                float g_other = 0.0f;
                if constexpr (RP == 2) g_other = __shfl_xor_sync(kFull, g, 16);
                static_for<R>([&](auto kc) {
                  constexpr int k = decltype(kc)::value;
                  float gk;
                  if constexpr (RP == 2) gk = (my_stage == k) ? g : g_other;
                  else gk = __shfl_sync(kFull, g, lane_of_stage<RP>(k));
                  row_update(v[(u - k + R) % R], o[k], gk);
                });
                constexpr int out = (u + 1) % R;
                sts_row(v[out], voff[out], lm);
                voff[out] = sink_b;
              }
            });
          }
#pragma unroll
          for (int k = 0; k < R; k++) {
            const int tk = tks[k];
            if (k < nt) {
              Row<VEC, NV> o0;
              lds_staged<T>(o0, (pre ? cur_b : o0_b) + (uint32_t)k * srow_bytes, lm);
              row_add_delta(syn1neg + (int64_t)tk * P, o[k], o0, lane, d,
                            sr_event_key(skey, (uint64_t)w * (K + 1) + (k0 + k)),
                            (uint64_t)tk);
            }
          }
        } else {
          // ---- serial sweeps: a repeated target must see the earlier write ----
          for (int k = 0; k < nt; k++) {
            const int tk = __shfl_sync(kFull, my_t, k);
            Row<VEC, NV> so, so0, sv;
            row_load_global(so, syn1neg + (int64_t)tk * P, lane, d);
            so0 = so;
            unsigned rem = mask;
            for (int j = 0; j < nctx; j++) {
              const int s0 = __ffs(rem) - 1;
              rem &= rem - 1;
              const uint32_t a = ring_b + (uint32_t)s0 * row_bytes;
              lds_row(sv, a, lm);
              const float x = warp_sum(row_dot(sv, so));
              const float g = gradient<SIG>(x, k0 + k == 0, alpha, table);
              row_update(sv, so, g);
              sts_row(sv, a, lm);
            }
            row_add_delta(syn1neg + (int64_t)tk * P, so, so0, lane, d,
                          sr_event_key(skey, (uint64_t)w * (K + 1) + (k0 + k)),
                          (uint64_t)tk);
          }
        }
        t_prev = lane < nt ? my_t : -1;
        if (pre) cur_b = cur_b == o0_b ? o1_b : o0_b;
      }
    }

    // Slide the window: position w-W leaves, position w+W+1 takes its slot.
    // The staging copies must be complete; the next group's prefetch may run on.
    if (!bulk) {
      if (prefetches > 0) cp_async_wait_but_last();
      else cp_async_wait();
    } else if (stage_bytes) {
      if (!mbar_wait(bar_b, bar_phase)) {
        // give the copies a second bounded wait before the warp stops
        if (lane == 0) atomicExch(p.error_flag, 2);
        mbar_wait(bar_b, bar_phase);
        if (lane == 0) bulk_wait_all();
        __syncwarp();
        return false;
      }
      bar_phase ^= 1u;
    }
    if (q_out >= 0) {
      Row<VEC, NV> cur, org;
      lds_row(cur, ring_b + (uint32_t)slot_out * row_bytes, lm);
      lds_staged<T>(org, out_b, lm);
      if (bulk) clear_past_d(org, lm, d);
      row_add_delta(syn0 + (int64_t)id_out * P, cur, org, lane, d,
                    sr_event_key(skey, (uint64_t)L * (K + 1) + q_out), (uint64_t)id_out);
    }
    if (id_in >= 0) {
      const int s = slot_out;
      Row<VEC, NV> enter_row;
      if (enter_early) {
        lds_staged<T>(enter_row, in_b, lm);
        if (bulk) {
          clear_past_d(enter_row, lm, d);
          if (lane == 0) bulk_store(orig + s * P, in_b, srow_bytes);
          last_store_slot = s;
        } else {
          row_store_global(enter_row, orig + s * P, lane, d);
        }
      } else {
        row_load_global(enter_row, syn0 + (int64_t)id_in * P, lane, d);
        row_store_global(enter_row, orig + s * P, lane, d);
      }
      sts_row(enter_row, ring_b + (uint32_t)s * row_bytes, lm);
    }
    slot_out = slot_out + 1 < D ? slot_out + 1 : 0;
    lane_off = lane_off > 0 ? lane_off - 1 : D - 1;
  }
  // Positions still in the window leave in increasing order; their originals
  // are read back with generic loads once the bulk stores are complete.
  if (lane == 0) bulk_wait_all();
  __syncwarp();
  proxy_fence();
  for (int q = L - W > 0 ? L - W : 0; q < L; q++) {
    const int s = q % D;
    Row<VEC, NV> cur, org;
    lds_row(cur, ring_b + (uint32_t)s * row_bytes, lm);
    row_load_global(org, orig + s * P, lane, d);
    const int id_q = __ldg(ids + q);
    row_add_delta(syn0 + (int64_t)id_q * P, cur, org, lane, d,
                  sr_event_key(skey, (uint64_t)L * (K + 1) + q), (uint64_t)id_q);
  }
  return true;
}

// Blocks per SM the register budget is sized for: the one-vector shapes fit
// 4 blocks (<= 128 registers); wider rows keep their stage registers with 2.
template <int NV>
struct MinBlocks {
  static constexpr int value = NV == 1 ? 4 : 2;
};

template <typename T, int VEC, int NV, int R, int SIG>
// Sentences are taken one per warp: all by warp 0 in order (deterministic),
// by static assignment (work_counter null: the kernel seam, whose launches
// may run concurrently), or from an atomic work counter.  One call site of
// train_sentence keeps the code (and the instruction cache footprint) to one
// copy of the body; its parameters are read from a shared-memory copy.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, MinBlocks<NV>::value) sgns_train_kernel(TrainParams p) {
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) TrainParams sp;
  __shared__ float table[kExpTableSize];  // the sigmoid table, read once per pipeline step
  copy_params(&sp, &p, threadIdx.x, blockDim.x);
  if constexpr (SIG == 0)
    for (int i = threadIdx.x; i < kExpTableSize; i += blockDim.x) table[i] = p.exp_table[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int D = 2 * p.window + 1;
  float* ring = smem + (int64_t)warp * warp_smem_bytes(D, R, p.prefetch != 0, p.pitch, (int)sizeof(T)) / 4;
  const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  T* orig = reinterpret_cast<T*>(p.orig_scratch) + gwarp * D * p.pitch;
  const int64_t total = total_sentences(p);
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  if (p.deterministic && gwarp != 0) return;
  const uint32_t bar_b =
      warp_bulk_init(ring, (uint32_t)warp_smem_bytes(D, R, p.prefetch != 0, p.pitch, (int)sizeof(T)), lane);
  uint32_t bar_phase = 0;
  int64_t next = gwarp;
  for (;;) {
    int64_t w;
    if (p.deterministic) {
      w = next++;
    } else if (p.work_counter == nullptr) {
      w = next;
      next += nwarps;
    } else {
      unsigned long long c = 0;
      if (lane == 0) c = atomicAdd(p.work_counter, 1ULL);
      w = (int64_t)__shfl_sync(kFull, c, 0);
    }
    if (w >= total) break;
    const Sentence sn = fetch_sentence(p, w);
    if (!train_sentence<T, VEC, NV, R, SIG>(sp, sn, ring, orig, table, lane, bar_b, bar_phase)) break;
  }
}

// ---------------------------------------------------------------------------
// Held-out SGNS loss: one warp per sentence, FP64 accumulation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double log_sigmoid(double x) {
  return x >= 0 ? -log1p(exp(-x)) : x - log1p(exp(x));
}

template <typename T, int VEC, int NV>
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
        row_load_global(v, reinterpret_cast<const T*>(p.syn0) + (int64_t)ids[pos] * P, lane, d);
        for (int k = 0; k <= K; k++) {
          const int32_t t = k == 0 ? ids[w] : negs[(int64_t)w * K + k - 1];
          row_load_global(o, reinterpret_cast<const T*>(p.syn1neg) + (int64_t)t * P, lane, d);
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
// Warps per block of a launch whose warps need warp_smem bytes of dynamic
// shared memory each, beside `static_smem` bytes of the kernel's own: 4, or 2
// or 1 where 4 do not fit a block (wide rows with long windows); 0 if not
// even one does.  The kernel takes its warp count from blockDim.
inline int train_block_warps(size_t warp_smem, size_t static_smem, int deterministic) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  int warps = deterministic ? 1 : kWarpsPerBlock;
  while (warps > 1 && (size_t)warps * warp_smem + static_smem > (size_t)optin) warps /= 2;
  return warp_smem + static_smem <= (size_t)optin ? warps : 0;
}

template <typename T, int VEC, int NV, int R, int SIG>
cudaError_t launch_t(const TrainParams& p, int num_sms, size_t warp_smem, cudaStream_t st) {
  auto kern = sgns_train_kernel<T, VEC, NV, R, SIG>;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  const int warps = train_block_warps(warp_smem, fa.sharedSizeBytes, p.deterministic);
  if (warps < 1) return cudaErrorInvalidValue;
  const size_t smem = (size_t)warps * warp_smem;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int blocks = 1;
  const int threads = warps * 32;
  if (!p.deterministic) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    blocks = per_sm * num_sms;
    const int64_t cap = p.scratch_warps / warps;
    if (blocks > cap) blocks = (int)cap;
    if (blocks < 1) return cudaErrorInvalidConfiguration;
  }
  kern<<<blocks, threads, smem, st>>>(p);
  return cudaGetLastError();
}

// Stage counts compiled per shape: rows of up to 3 vectors per lane pipeline
// up to 8 targets; wider rows (d > 384) sweep targets one at a time.
template <typename T, int VEC, int NV, int SIG>
cudaError_t launch_r(const TrainParams& p, int r, int num_sms, size_t warp_smem, cudaStream_t st) {
  if constexpr (NV >= 4) {
    return launch_t<T, VEC, NV, 1, SIG>(p, num_sms, warp_smem, st);
  } else {
    switch (r) {
      case 1: return launch_t<T, VEC, NV, 1, SIG>(p, num_sms, warp_smem, st);
      case 2: return launch_t<T, VEC, NV, 2, SIG>(p, num_sms, warp_smem, st);
      case 4: return launch_t<T, VEC, NV, 4, SIG>(p, num_sms, warp_smem, st);
      case 6: return launch_t<T, VEC, NV, 6, SIG>(p, num_sms, warp_smem, st);
      default: return launch_t<T, VEC, NV, 8, SIG>(p, num_sms, warp_smem, st);
    }
  }
}

}  // namespace fw2v
