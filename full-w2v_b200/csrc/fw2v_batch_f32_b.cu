// Instantiation of the batched training kernel: FP32 tables, wide rows, light pipelines.
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<float, 1>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<float, 1>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
