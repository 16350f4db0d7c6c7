// Dispatch of the SGNS training and held-out loss kernels (fw2v_train.cuh).
#include "fw2v_train.cuh"

namespace fw2v {

extern template cudaError_t launch_r<2, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 1>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 2>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 3>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 4>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 6>(const TrainParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_r<4, 8>(const TrainParams&, int, int, size_t, cudaStream_t);

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
  return s;
}

size_t train_smem_bytes(int window, int64_t pitch, int warps) {
  return (size_t)(1024 + (size_t)warps * 2 * (2 * window + 1) * pitch) * sizeof(float);
}

cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st) {
  const LaunchShape s = choose_shape(p.d, p.negative);
  const size_t smem = train_smem_bytes(p.window, p.pitch, p.deterministic ? 1 : kWarpsPerBlock);
  if (s.vec == 2) return launch_r<2, 1>(p, s.r, num_sms, smem, st);
  switch (s.nv) {
    case 1: return launch_r<4, 1>(p, s.r, num_sms, smem, st);
    case 2: return launch_r<4, 2>(p, s.r, num_sms, smem, st);
    case 3: return launch_r<4, 3>(p, s.r, num_sms, smem, st);
    case 4: return launch_r<4, 4>(p, s.r, num_sms, smem, st);
    case 6: return launch_r<4, 6>(p, s.r, num_sms, smem, st);
    default: return launch_r<4, 8>(p, s.r, num_sms, smem, st);
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
