// fw2v_kernel_batch: the reference's `cuda_kernel` seam (FULL-W2V-kernels.cu:11-12,
// launched at FULL-W2V-driver.cu:293 and :317) on the B200 training kernel.
// Block b of a batch trains sen[b*msl .. +len[b]] with negatives at
// neg[b*msl*K ...] and learning rate alpha[b]; tables have `pitch` floats per
// row.  Launches may run concurrently on several streams (the reference drives
// this seam from T host threads x S streams), so sentences are assigned to
// warps statically and the only shared state is a sticky error word and the
// sigmoid table, both per device.
#include <mutex>

#include "../../include/fw2v.h"
#include "fw2v_common.cuh"

extern "C" void fw2v_exp_table(float* t);

namespace fw2v {
cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st);
bool launch_fits(const TrainParams& p);
size_t train_smem_bytes(int window, int64_t pitch, int warps, int r, bool prefetch, int elem);
int64_t train_scratch_warps(int num_sms);
}  // namespace fw2v

namespace {

__device__ float g_seam_exp_table[fw2v::kExpTableSize];
__device__ int g_seam_error;

constexpr int kMaxDevices = 64;
std::mutex g_seam_mu;
bool g_seam_ready[kMaxDevices];
int g_seam_sms[kMaxDevices];

fw2v_status seam_setup(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return FW2V_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_seam_mu);
  if (g_seam_ready[dev]) return FW2V_OK;
  float table[fw2v::kExpTableSize];
  fw2v_exp_table(table);
  int zero = 0;
  int sms = 0;
  if (cudaMemcpyToSymbol(g_seam_exp_table, table, sizeof(table)) != cudaSuccess ||
      cudaMemcpyToSymbol(g_seam_error, &zero, sizeof(int)) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return FW2V_ERR_CUDA;
  g_seam_sms[dev] = sms;
  g_seam_ready[dev] = true;
  return FW2V_OK;
}

}  // namespace

extern "C" fw2v_status fw2v_kernel_batch(float* syn0, float* syn1neg, const int32_t* sen, const int32_t* neg,
                                         const int32_t* len, const float* alpha, int32_t n_blocks,
                                         int32_t layer_size, int32_t window, int32_t negative, int32_t msl,
                                         uint32_t pitch, int64_t vocab_size, void* stream) {
  if (!syn0 || !syn1neg || !sen || !len || !alpha || (negative > 0 && !neg) || n_blocks < 0 ||
      layer_size < 1 || layer_size > 1024 || window < 1 || window > fw2v::kMaxWindow || negative < 0 ||
      negative > fw2v::kMaxNegative || msl < 1 || (int64_t)pitch < layer_size || pitch % 4 != 0 ||
      vocab_size < 1)
    return FW2V_ERR_ARGUMENT;
  if (((uintptr_t)syn0 | (uintptr_t)syn1neg) % 16 != 0) return FW2V_ERR_ARGUMENT;
  if (n_blocks == 0) return FW2V_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FW2V_ERR_NO_DEVICE;
  fw2v_status s = seam_setup(dev);
  if (s != FW2V_OK) return s;
  fw2v::TrainParams p{};
  p.syn0 = syn0;
  p.syn1neg = syn1neg;
  p.pitch = pitch;
  p.vocab = vocab_size;
  p.d = layer_size;
  p.window = window;
  p.negative = negative;
  p.sigmoid = 0;
  p.ids = sen;
  p.negs = neg;
  p.source = fw2v::kSourceBlocks;
  p.lens = len;
  p.alphas = alpha;
  p.n_sentences = n_blocks;
  p.msl = msl;
  p.work_counter = nullptr;
  p.deterministic = 0;
  p.bf16 = 0;
  if (!fw2v::launch_fits(p)) return FW2V_ERR_ARGUMENT;
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_seam_error) != cudaSuccess) return FW2V_ERR_CUDA;
  p.error_flag = (int*)addr;
  if (cudaGetSymbolAddress(&addr, g_seam_exp_table) != cudaSuccess) return FW2V_ERR_CUDA;
  p.exp_table = (const float*)addr;
  // Per-launch scratch from the stream-ordered allocator, so concurrent
  // launches on different streams never share it.
  cudaStream_t st = (cudaStream_t)stream;
  p.scratch_warps = fw2v::train_scratch_warps(g_seam_sms[dev]);
  const size_t bytes = (size_t)p.scratch_warps * (2 * window + 1) * pitch * sizeof(float);
  if (cudaMallocAsync((void**)&p.orig_scratch, bytes, st) != cudaSuccess) return FW2V_ERR_NOMEM;
  const cudaError_t e = fw2v::launch_train(p, g_seam_sms[dev], st);
  cudaFreeAsync(p.orig_scratch, st);
  return e == cudaSuccess ? FW2V_OK : FW2V_ERR_CUDA;
}

namespace fw2v {

// The seam's per-device state (sigmoid table, sticky error word, SM count),
// set up on first use; shared with the allocation-free variant of the seam.
fw2v_status seam_state(int dev, int** error_word, const float** exp_table, int* sms) {
  fw2v_status s = seam_setup(dev);
  if (s != FW2V_OK) return s;
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_seam_error) != cudaSuccess) return FW2V_ERR_CUDA;
  *error_word = (int*)addr;
  if (cudaGetSymbolAddress(&addr, g_seam_exp_table) != cudaSuccess) return FW2V_ERR_CUDA;
  *exp_table = (const float*)addr;
  *sms = g_seam_sms[dev];
  return FW2V_OK;
}

}  // namespace fw2v

extern "C" fw2v_status fw2v_kernel_batch_error(void* stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FW2V_ERR_NO_DEVICE;
  fw2v_status s = seam_setup(dev);
  if (s != FW2V_OK) return s;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return FW2V_ERR_CUDA;
  int flag = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&flag, g_seam_error, sizeof(int)) != cudaSuccess) return FW2V_ERR_CUDA;
  if (!flag) return FW2V_OK;
  if (cudaMemcpyToSymbol(g_seam_error, &zero, sizeof(int)) != cudaSuccess) return FW2V_ERR_CUDA;
  return flag == 2 ? FW2V_ERR_CUDA : FW2V_ERR_BOUNDS;  // 2: a bulk row copy did not complete in time
}
