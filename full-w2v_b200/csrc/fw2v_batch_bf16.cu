// Instantiation of the batched training kernel for bfloat16 tables.
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<bf16_t>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<bf16_t>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
