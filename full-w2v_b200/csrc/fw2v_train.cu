// Dispatch of the SGNS training and held-out loss kernels (fw2v_train.cuh).
#include "fw2v_train.cuh"

namespace fw2v {

extern template cudaError_t launch_r<2, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<2, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 1, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 1, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 2, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 2, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 3, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 3, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 4, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 4, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 6, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 6, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 8, 0>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 8, 1>(const TrainParams&, int, int, size_t, cudaStream_t);


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
  if (s.nv >= 4) s.r = 1;
  return s;
}

// Shared memory of one block: per warp, the ring of 2W+1 rows, a sink row, R
// target originals and two staging rows (WarpRows).
size_t train_smem_bytes(int window, int64_t pitch, int warps, int r) {
  return (size_t)warps * (2 * window + 1 + 3 + r) * pitch * sizeof(float);
}

// Warps the scratch of a handle must cover: every warp the persistent grid can
// hold (64 per SM at most).
int64_t train_scratch_warps(int num_sms) { return (int64_t)num_sms * 64; }

cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  const size_t smem = train_smem_bytes(p.window, p.pitch, p.deterministic ? 1 : kWarpsPerBlock, s.r);
  if (s.vec == 2) return p.sigmoid == 0 ? launch_r<2, 1, 0>(p, s.r, num_sms, smem, st) : launch_r<2, 1, 1>(p, s.r, num_sms, smem, st);
  switch (s.nv) {
    case 1: return p.sigmoid == 0 ? launch_r<4, 1, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 1, 1>(p, s.r, num_sms, smem, st);
    case 2: return p.sigmoid == 0 ? launch_r<4, 2, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 2, 1>(p, s.r, num_sms, smem, st);
    case 3: return p.sigmoid == 0 ? launch_r<4, 3, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 3, 1>(p, s.r, num_sms, smem, st);
    case 4: return p.sigmoid == 0 ? launch_r<4, 4, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 4, 1>(p, s.r, num_sms, smem, st);
    case 6: return p.sigmoid == 0 ? launch_r<4, 6, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 6, 1>(p, s.r, num_sms, smem, st);
    default: return p.sigmoid == 0 ? launch_r<4, 8, 0>(p, s.r, num_sms, smem, st) : launch_r<4, 8, 1>(p, s.r, num_sms, smem, st);
  }
}

cudaError_t launch_heldout(const TrainParams& p, double* loss, unsigned long long* pairs, cudaStream_t st) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  const int blocks = 148 * 8;
  if (s.vec == 2) heldout_loss_kernel<2, 1><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else if (s.nv == 1) heldout_loss_kernel<4, 1><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else if (s.nv == 2) heldout_loss_kernel<4, 2><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else if (s.nv == 3) heldout_loss_kernel<4, 3><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else if (s.nv == 4) heldout_loss_kernel<4, 4><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else if (s.nv == 6) heldout_loss_kernel<4, 6><<<blocks, 128, 0, st>>>(p, loss, pairs);
  else heldout_loss_kernel<4, 8><<<blocks, 128, 0, st>>>(p, loss, pairs);
  return cudaGetLastError();
}

}  // namespace fw2v
