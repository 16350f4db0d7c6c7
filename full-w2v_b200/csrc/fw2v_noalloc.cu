// fw2v_kernel_batch_noalloc: the kernel seam (fw2v_kernel_batch) for callers
// that cannot allocate device memory — programs whose device memory belongs to
// a framework's pool allocator (a direct cudaMalloc bypasses its accounting
// and can fail once the pool holds the device), plugin hosts with a fixed
// memory budget, and loops in which an allocator call would stall or
// synchronise the device.  It runs the same training kernel; the only
// difference is where the per-warp scratch comes from: a fixed array in this
// file instead of a per-launch allocation.
#include <mutex>

#include "../../include/fw2v.h"
#include "fw2v_common.cuh"

namespace fw2v {
cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st);
bool launch_fits(const TrainParams& p);
fw2v_status seam_state(int dev, int** error_word, const float** exp_table, int* sms);
}  // namespace fw2v

namespace {

// The scratch: (2W+1) * pitch floats per warp, as many warps as fit.  Host code
// must not use the symbol as an address; the device address comes from
// cudaGetSymbolAddress, once per device.
__device__ __align__(256) float g_noalloc_scratch[FW2V_NOALLOC_SCRATCH_BYTES / sizeof(float)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch[kMaxDevices];  // device address of g_noalloc_scratch per device

fw2v_status scratch_address(int dev, float** out) {
  if (dev < 0 || dev >= kMaxDevices) return FW2V_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return FW2V_ERR_CUDA;
    g_scratch[dev] = (float*)addr;
  }
  *out = g_scratch[dev];
  return FW2V_OK;
}

}  // namespace

extern "C" fw2v_status fw2v_kernel_batch_noalloc(float* syn0, float* syn1neg, const int32_t* sen,
                                                 const int32_t* neg, const int32_t* len, const float* alpha,
                                                 int32_t n_blocks, int32_t layer_size, int32_t window,
                                                 int32_t negative, int32_t msl, uint32_t pitch, int64_t vocab_size,
                                                 void* stream) {
  if (!syn0 || !syn1neg || !sen || !len || !alpha || (negative > 0 && !neg) || n_blocks < 0 ||
      layer_size < 1 || layer_size > 1024 || window < 1 || window > fw2v::kMaxWindow || negative < 0 ||
      negative > fw2v::kMaxNegative || msl < 1 || (int64_t)pitch < layer_size || pitch % 4 != 0 ||
      vocab_size < 1)
    return FW2V_ERR_ARGUMENT;
  if (((uintptr_t)syn0 | (uintptr_t)syn1neg) % 16 != 0) return FW2V_ERR_ARGUMENT;
  // Scratch per warp; one block of kWarpsPerBlock warps must fit.
  const uint64_t warp_floats = (uint64_t)(2 * window + 1) * pitch;
  const uint64_t cap_warps = (FW2V_NOALLOC_SCRATCH_BYTES / sizeof(float)) / warp_floats;
  if (cap_warps < (uint64_t)fw2v::kWarpsPerBlock) return FW2V_ERR_TOO_LARGE;
  fw2v::TrainParams p{};
  p.pitch = pitch;
  p.d = layer_size;
  p.window = window;
  p.negative = negative;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FW2V_ERR_NO_DEVICE;
  // one warp's ring and staged rows must fit a block's shared memory
  if (!fw2v::launch_fits(p)) return FW2V_ERR_ARGUMENT;
  if (n_blocks == 0) return FW2V_OK;
  float* scratch = nullptr;
  fw2v_status s = scratch_address(dev, &scratch);
  if (s != FW2V_OK) return s;
  int* error_word = nullptr;
  const float* table = nullptr;
  int sms = 0;
  s = fw2v::seam_state(dev, &error_word, &table, &sms);
  if (s != FW2V_OK) return s;

  p.syn0 = syn0;
  p.syn1neg = syn1neg;
  p.vocab = vocab_size;
  p.sigmoid = 0;
  p.ids = sen;
  p.negs = neg;
  p.source = fw2v::kSourceBlocks;
  p.lens = len;
  p.alphas = alpha;
  p.n_sentences = n_blocks;
  p.msl = msl;
  p.work_counter = nullptr;  // static sentence-to-warp assignment
  p.deterministic = 0;
  p.bf16 = 0;
  p.error_flag = error_word;
  p.exp_table = table;
  p.orig_scratch = scratch;
  p.scratch_warps = (int64_t)cap_warps;  // the launch caps its grid to this
  return fw2v::launch_train(p, sms, (cudaStream_t)stream) == cudaSuccess ? FW2V_OK : FW2V_ERR_CUDA;
}
