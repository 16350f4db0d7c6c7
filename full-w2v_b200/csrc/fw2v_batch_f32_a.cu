// Instantiation of the batched training kernel: FP32 tables, rows of one vector per lane (d <= 128).
#include "fw2v_batch.cuh"

namespace fw2v {
template cudaError_t batch_grid<float, 0>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*);
template cudaError_t batch_launch<float, 0>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
}  // namespace fw2v
