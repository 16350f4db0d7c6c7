// Instantiation of the batched training kernel for FP32 tables.
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<float>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<float>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
