// Instantiation of the batched training kernel: FP32 tables, wide rows, deep pipelines.
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<float, 2>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<float, 2>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
