// Instantiation of the batched training kernel: bfloat16 tables, wide rows, light pipelines.
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<bf16_t, 1>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<bf16_t, 1>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
