// Instantiation of the training kernel: f32 tables, lanes of 2-float vectors x 1, exact sigmoid.
#include "fw2v_train.cuh"

namespace fw2v {
template cudaError_t launch_r<float, 2, 1, 1>(const TrainParams& p, int r, int num_sms, size_t smem, cudaStream_t st);
}  // namespace fw2v
