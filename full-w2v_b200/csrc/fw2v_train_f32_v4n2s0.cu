// Instantiation of the training kernel: f32 tables, lanes of 4-float vectors x 2, table sigmoid.
#include "fw2v_train.cuh"

namespace fw2v {
template cudaError_t launch_r<float, 4, 2, 0>(const TrainParams& p, int r, int num_sms, size_t smem, cudaStream_t st);
}  // namespace fw2v
