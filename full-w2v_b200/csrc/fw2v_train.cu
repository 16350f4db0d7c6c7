// Dispatch of the SGNS training and held-out loss kernels (fw2v_train.cuh).
#include "fw2v_train.cuh"

namespace fw2v {

extern template cudaError_t launch_r<float, 2, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 2, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 2, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 2, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 3, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 3, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 4, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 4, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 6, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 6, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 8, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<float, 4, 8, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 2, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 2, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 2, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 2, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 3, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<bf16_t, 4, 3, 1>(const TrainParams&, int, int, size_t, cudaStream_t);



struct LaunchShape {
  int vec, nv, r;
};

// Lane layout from the layer size (the same rule as fw2v_lane_layout).
LaunchShape choose_shape(int d, int negative) {
  LaunchShape s;
  const int pitch = (d + 7) / 8 * 8;
  if (pitch <= 64) {
    s.vec = 2;
    s.nv = 1;
  } else {
    s.vec = 4;
    const int nv = (pitch + 127) / 128;
    s.nv = nv <= 4 ? nv : (nv <= 6 ? 6 : 8);
  }
  const int want = negative + 1;
  s.r = want <= 1 ? 1 : want <= 2 ? 2 : want <= 4 ? 4 : want <= 6 ? 6 : 8;
  if (s.nv == 3 && s.r > 4) s.r = 4;  // three vectors per lane: more stages spill registers
  if (s.nv >= 4) s.r = 1;
  return s;
}

// Shared memory of one block: warp_smem_bytes per warp.
size_t train_smem_bytes(int window, int64_t pitch, int warps, int r, bool prefetch, int elem) {
  return (size_t)warps * (size_t)warp_smem_bytes(2 * window + 1, r, prefetch, pitch, elem);
}

// Warps the scratch of a handle must cover: every warp the persistent grid can
// hold (64 per SM at most).
int64_t train_scratch_warps(int num_sms) { return (int64_t)num_sms * 64; }

// Table type and sigmoid mode of a launch; bfloat16 tables cover rows of up to
// 384 elements (three 4-float vectors per lane).
template <int VEC, int NV>
static cudaError_t launch_rt(const TrainParams& p, int r, int num_sms, size_t smem, cudaStream_t st) {
  // smem: shared memory of one warp
  if (p.bf16) {
    if constexpr (NV <= 3) {
      return p.sigmoid == 0 ? launch_r<bf16_t, VEC, NV, 0>(p, r, num_sms, smem, st)
                            : launch_r<bf16_t, VEC, NV, 1>(p, r, num_sms, smem, st);
    } else {
      return cudaErrorInvalidValue;
    }
  }
  return p.sigmoid == 0 ? launch_r<float, VEC, NV, 0>(p, r, num_sms, smem, st)
                        : launch_r<float, VEC, NV, 1>(p, r, num_sms, smem, st);
}

// Shared memory of one warp of a launch of the training kernel.
size_t launch_warp_smem(const TrainParams& p) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  return train_smem_bytes(p.window, p.pitch, 1, s.r, p.prefetch != 0, p.bf16 ? 2 : 4);
}

// Static shared memory of the training kernel, with a margin: its parameter
// block and the sigmoid table.
size_t train_static_smem() { return sizeof(TrainParams) + kExpTableSize * sizeof(float) + 64; }

// Whether one warp of a launch of p fits a block's shared memory (launch_t
// takes 4, 2 or 1 warps per block, as many as fit).
bool launch_fits(const TrainParams& p) {
  return train_block_warps(launch_warp_smem(p), train_static_smem(), 1) == 1;
}

cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  const size_t smem = launch_warp_smem(p);
  if (s.vec == 2) return launch_rt<2, 1>(p, s.r, num_sms, smem, st);
  switch (s.nv) {
    case 1: return launch_rt<4, 1>(p, s.r, num_sms, smem, st);
    case 2: return launch_rt<4, 2>(p, s.r, num_sms, smem, st);
    case 3: return launch_rt<4, 3>(p, s.r, num_sms, smem, st);
    case 4: return launch_rt<4, 4>(p, s.r, num_sms, smem, st);
    case 6: return launch_rt<4, 6>(p, s.r, num_sms, smem, st);
    default: return launch_rt<4, 8>(p, s.r, num_sms, smem, st);
  }
}

template <int VEC, int NV>
static void heldout_t(const TrainParams& p, double* loss, unsigned long long* pairs, int blocks, cudaStream_t st) {
  if (p.bf16) heldout_loss_kernel<bf16_t, VEC, NV><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else heldout_loss_kernel<float, VEC, NV><<<blocks, 128, 0, st>>>(p, loss, pairs);
}

cudaError_t launch_heldout(const TrainParams& p, double* loss, unsigned long long* pairs, cudaStream_t st) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  const int blocks = 148 * 8;
  if (s.vec == 2) heldout_t<2, 1>(p, loss, pairs, blocks, st);
  else if (s.nv == 1) heldout_t<4, 1>(p, loss, pairs, blocks, st);
  else if (s.nv == 2) heldout_t<4, 2>(p, loss, pairs, blocks, st);
  else if (s.nv == 3) heldout_t<4, 3>(p, loss, pairs, blocks, st);
  else if (s.nv == 4) heldout_t<4, 4>(p, loss, pairs, blocks, st);
  else if (s.nv == 6) heldout_t<4, 6>(p, loss, pairs, blocks, st);
  else heldout_t<4, 8>(p, loss, pairs, blocks, st);
  return cudaGetLastError();
}

}  // namespace fw2v
