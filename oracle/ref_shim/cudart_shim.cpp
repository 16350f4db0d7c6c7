// TEST INFRASTRUCTURE ONLY — never linked into the product library or the CLI.
//
// A host-memory stand-in for the few CUDA runtime / driver entry points that the
// reference program (FULL-W2V-driver.cu and the .cpp files it includes) calls.
// oracle/Makefile compiles the UNMODIFIED reference driver with nvcc and links it
// against this file instead of libcudart, so the reference's own host code (vocab,
// unigram table, subsampling, LCG negatives, batch builder, alpha schedule,
// InitNet, saveModel) runs on a machine without a GPU.  "Device" buffers are host
// allocations, copies are memcpy, and every kernel launch is a no-op except for the
// training kernel, whose batch arguments are written to a dump file.  Those dumps
// are the golden integer vectors the oracle and the CUDA sampler are checked
// against (tests/golden/make_golden.py).
//
// Dump format (little-endian, one file per calling host thread, opened lazily in
// $FW2V_REF_DUMP_DIR as thread_<n>.bin where n is the order of first launch):
//   per launch of matrix_matrix_w2v_kernel_small:
//     int32 magic 0x57325644, int32 fresh_blocks, int32 K, int32 MSL
//     per fresh block b: int32 len, float alpha, int32 sen[len], int32 neg[len*K]
// "fresh_blocks" is the element count of the most recent host->device copy into
// the launch's sentence-length buffer (FULL-W2V-driver.cu:289,313); blocks past it
// are stale replays of earlier batches (FULL-W2V-driver.cu:305-318) and are skipped.

#include <cuda.h>
#include <cuda_runtime_api.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace {

// Function-local statics: the reference's registration code runs from a static
// constructor in another translation unit, before this file's globals would be.
std::mutex& mu() { static std::mutex m; return m; }
std::map<const void*, std::string>& kernel_names() {   // host stub -> device symbol
  static std::map<const void*, std::string> m; return m;
}
std::map<const void*, size_t>& last_copy_bytes() {     // "device" dst -> bytes of last H2D copy
  static std::map<const void*, size_t> m; return m;
}
std::atomic<int> g_thread_counter{0};

struct LaunchConfig {
  dim3 grid, block;
  size_t smem;
  void* stream;
};
thread_local LaunchConfig t_cfg;
thread_local FILE* t_dump = nullptr;

FILE* thread_dump() {
  if (t_dump) return t_dump;
  const char* dir = std::getenv("FW2V_REF_DUMP_DIR");
  if (!dir || !*dir) return nullptr;
  int n = g_thread_counter.fetch_add(1);
  std::string path = std::string(dir) + "/thread_" + std::to_string(n) + ".bin";
  t_dump = std::fopen(path.c_str(), "wb");
  return t_dump;
}

void record_copy(const void* dst, size_t bytes) {
  std::lock_guard<std::mutex> lk(mu());
  last_copy_bytes()[dst] = bytes;
}

}  // namespace

extern "C" {

void** __cudaRegisterFatBinary(void* fatCubin) {
  static void* handle_storage = nullptr;
  (void)fatCubin;
  return &handle_storage;
}
void __cudaRegisterFatBinaryEnd(void** h) { (void)h; }
void __cudaUnregisterFatBinary(void** h) { (void)h; }
void __cudaRegisterVar(void** h, char* hostVar, char* devAddr, const char* name, int ext,
                       size_t size, int constant, int global) {
  (void)h; (void)hostVar; (void)devAddr; (void)name; (void)ext; (void)size; (void)constant;
  (void)global;
}
void __cudaRegisterFunction(void** h, const char* hostFun, char* deviceFun, const char* deviceName,
                            int thread_limit, uint3* tid, uint3* bid, dim3* bDim, dim3* gDim,
                            int* wSize) {
  (void)h; (void)deviceFun; (void)thread_limit; (void)tid; (void)bid; (void)bDim; (void)gDim;
  (void)wSize;
  std::lock_guard<std::mutex> lk(mu());
  kernel_names()[hostFun] = deviceName ? deviceName : "";
}

unsigned __cudaPushCallConfiguration(dim3 grid, dim3 block, size_t smem, struct CUstream_st* stream) {
  t_cfg.grid = grid;
  t_cfg.block = block;
  t_cfg.smem = smem;
  t_cfg.stream = stream;
  return 0;
}
cudaError_t __cudaPopCallConfiguration(dim3* grid, dim3* block, size_t* smem, void* stream) {
  *grid = t_cfg.grid;
  *block = t_cfg.block;
  *smem = t_cfg.smem;
  *(void**)stream = t_cfg.stream;
  return cudaSuccess;
}

cudaError_t cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem,
                             cudaStream_t stream) {
  (void)block; (void)smem; (void)stream;
  std::string name;
  {
    std::lock_guard<std::mutex> lk(mu());
    auto it = kernel_names().find(func);
    if (it != kernel_names().end()) name = it->second;
  }
  if (name.find("matrix_matrix_w2v_kernel_small") == std::string::npos) return cudaSuccess;
  FILE* f = thread_dump();
  if (!f) return cudaSuccess;
  // Argument order of matrix_matrix_w2v_kernel_small (FULL-W2V-kernels.cu:106).
  const int* sen = *(const int* const*)args[2];
  const int* neg = *(const int* const*)args[3];
  const int* len = *(const int* const*)args[4];
  const float* alpha = *(const float* const*)args[5];
  int K = *(const int*)args[8];
  int msl = *(const int*)args[9];
  size_t fresh_bytes;
  {
    std::lock_guard<std::mutex> lk(mu());
    fresh_bytes = last_copy_bytes()[len];
  }
  int32_t fresh = (int32_t)(fresh_bytes / sizeof(int));
  if (fresh > (int32_t)grid.x) fresh = (int32_t)grid.x;
  int32_t hdr[4] = {0x57325644, fresh, K, msl};
  std::fwrite(hdr, sizeof(int32_t), 4, f);
  for (int32_t b = 0; b < fresh; ++b) {
    int32_t L = len[b];
    std::fwrite(&L, sizeof(int32_t), 1, f);
    std::fwrite(&alpha[b], sizeof(float), 1, f);
    if (L > 0) {
      std::fwrite(sen + (size_t)b * msl, sizeof(int32_t), (size_t)L, f);
      if (K > 0) std::fwrite(neg + (size_t)b * msl * K, sizeof(int32_t), (size_t)L * K, f);
    }
  }
  std::fflush(f);
  return cudaSuccess;
}

cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaStreamCreate(cudaStream_t* s) {
  *s = (cudaStream_t)std::malloc(16);
  return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t s) {
  std::free((void*)s);
  return cudaSuccess;
}
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t) { return "host shim"; }

cudaError_t cudaMalloc(void** p, size_t bytes) {
  *p = std::calloc(bytes ? bytes : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaHostAlloc(void** p, size_t bytes, unsigned int) { return cudaMalloc(p, bytes); }
cudaError_t cudaMallocPitch(void** p, size_t* pitch, size_t width, size_t height) {
  size_t w = (width + 127) / 128 * 128;
  *pitch = w;
  return cudaMalloc(p, w * height);
}
cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaFreeHost(void* p) { return cudaFree(p); }

cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                            cudaStream_t) {
  std::memcpy(dst, src, bytes);
  if (kind == cudaMemcpyHostToDevice) record_copy(dst, bytes);
  return cudaSuccess;
}
cudaError_t cudaMemcpy2D(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                         size_t height, cudaMemcpyKind) {
  for (size_t r = 0; r < height; ++r)
    std::memcpy((char*)dst + r * dpitch, (const char*)src + r * spitch, width);
  return cudaSuccess;
}
cudaError_t cudaMemcpy2DAsync(void* dst, size_t dpitch, const void* src, size_t spitch,
                              size_t width, size_t height, cudaMemcpyKind kind, cudaStream_t) {
  return cudaMemcpy2D(dst, dpitch, src, spitch, width, height, kind);
}

CUresult cuDeviceGet(CUdevice* d, int ordinal) {
  *d = ordinal;
  return CUDA_SUCCESS;
}
CUresult cuDevicePrimaryCtxRetain(CUcontext* c, CUdevice) {
  *c = nullptr;
  return CUDA_SUCCESS;
}

}  // extern "C"
