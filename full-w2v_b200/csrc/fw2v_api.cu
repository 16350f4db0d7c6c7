// C ABI of libfw2v (include/fw2v.h): handle lifetime, device memory, and the
// epoch loop of Train_SGNS (FULL-W2V-driver.cu:80-354) as two kernel launches
// per epoch (sampler, trainer) with no host work in between.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fw2v.h"
#include "fw2v_common.cuh"

extern "C" void fw2v_exp_table(float* t);
extern "C" int fw2v_unigram_firsts(const uint32_t* counts, int64_t V, int64_t size, int64_t* firsts);

namespace fw2v {
cudaError_t launch_sampler(const SamplerParams& p, int64_t max_region, int64_t* entry_prefix, cudaStream_t st);
cudaError_t launch_train(const TrainParams& p, int num_sms, cudaStream_t st);
cudaError_t launch_heldout(const TrainParams& p, double* loss, unsigned long long* pairs, cudaStream_t st);
cudaError_t launch_init_tables(void* syn0, bool bf16, int64_t V, int d, int64_t pitch, const uint32_t* d_counts,
                               float sample, uint64_t train_words, int32_t* keep_thr, const int64_t* d_firsts,
                               int n_firsts, int32_t* unigram, int64_t table_size, uint64_t start,
                               cudaStream_t st);
size_t train_smem_bytes(int window, int64_t pitch, int warps, int r, bool prefetch, int elem);
size_t train_static_smem();
int64_t train_scratch_warps(int num_sms);
cudaError_t launch_validate_ids(const int32_t* ids, int64_t n, int64_t vocab, int* flag, cudaStream_t st);
cudaError_t launch_check_corpus(const int32_t* stream, int64_t len, const int64_t* chunk_off, int64_t n, int* flag,
                                cudaStream_t st);
cudaError_t launch_fisher_yates(int64_t* a, int64_t n, uint64_t key, cudaStream_t st);
cudaError_t launch_corpus_layout(const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                                 int64_t n_chunks, int msl, int threads, int64_t* chunk_base,
                                 int64_t* stream_base, cudaStream_t st);
}  // namespace fw2v

using namespace fw2v;

struct SampleBuf {
  int64_t* ent_start = nullptr;
  int32_t* ent_len = nullptr;
  float* ent_alpha = nullptr;
  int32_t* kept_ids = nullptr;
  uint64_t* kept_state = nullptr;
  int32_t* kept_negs = nullptr;
  int64_t* n_entries = nullptr;
  int64_t* n_kept = nullptr;
  uint64_t* words = nullptr;
  int64_t* entry_prefix = nullptr;
  cudaEvent_t start = nullptr;  // sampler launched
  cudaEvent_t ready = nullptr;  // sampler outputs complete
  cudaEvent_t freed = nullptr;  // trainer done reading them
  bool used = false;            // `freed` has been recorded at least once
};

struct fw2v_handle {
  fw2v_config cfg{};
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  std::string err;

  int64_t V = 0;
  uint64_t train_words = 0;
  int64_t pitch = 0;
  void* syn0 = nullptr;  // float, or uint16 bfloat16 bits with FW2V_BF16
  void* syn1neg = nullptr;
  size_t elem = 4;        // bytes per table element
  uint64_t launches = 0;  // training launches so far (stochastic-rounding seeds)
  int32_t* keep_thr = nullptr;
  int32_t* unigram = nullptr;
  uint64_t* jump_a = nullptr;
  uint64_t* jump_c = nullptr;
  float* exp_table = nullptr;

  int32_t* stream_ids = nullptr;
  int64_t stream_len = 0;
  int64_t* chunk_off = nullptr;
  int64_t n_chunks = 0;
  int64_t* chunk_base = nullptr;   // n_chunks + 1: prefix of readable chunk lengths
  int64_t* stream_base = nullptr;  // threads + 1: kept-id base of each stream
  std::vector<int64_t> h_stream_base;
  int64_t sample_cap = 0;          // kept-id capacity of a sampler output set
  int64_t max_region = 0;

  uint64_t* lcg = nullptr;
  uint64_t* wca = nullptr;
  float* alpha = nullptr;
  // Two sets of sampler outputs: epoch e is sampled into buf[e % 2] on the
  // sampler stream while epoch e-1 trains from the other set.
  SampleBuf buf[2];
  cudaStream_t sstream = nullptr;
  int64_t n_sampled = 0;  // epochs sampled since load_corpus
  int64_t n_trained = 0;  // epochs trained since load_corpus

  int* error_flag = nullptr;
  unsigned long long* work_counter = nullptr;
  void* orig_scratch = nullptr;
  int64_t scratch_warps = 0;

  int epochs_done = 0;
  uint64_t words_total = 0;
};

namespace {

fw2v_status fail(fw2v_handle* h, fw2v_status s, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return s;
}

#define CK(h, call)                                                                         \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      return fail((h), e_ == cudaErrorMemoryAllocation ? FW2V_ERR_NOMEM : FW2V_ERR_CUDA,    \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);    \
    }                                                                                       \
  } while (0)

void dfree_v(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <typename T>
cudaError_t dalloc(T*& p, size_t n) {
  dfree(p);
  return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
}

int64_t pitch_for(int d) { return ((int64_t)d + 7) / 8 * 8; }

fw2v_status check_flag(fw2v_handle* h, const char* what) {
  int flag = 0;
  CK(h, cudaMemcpyAsync(&flag, h->error_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  if (flag) {
    CK(h, cudaMemsetAsync(h->error_flag, 0, sizeof(int), h->stream));
    if (flag == 2) return fail(h, FW2V_ERR_CUDA, "%s: a bulk row copy did not complete in time", what);
    return fail(h, FW2V_ERR_BOUNDS, "%s: an id outside [0, V) or a read past the token stream", what);
  }
  return FW2V_OK;
}

TrainParams base_train_params(fw2v_handle* h) {
  TrainParams p{};
  p.syn0 = h->syn0;
  p.syn1neg = h->syn1neg;
  p.pitch = h->pitch;
  p.vocab = h->V;
  p.d = h->cfg.layer_size;
  p.window = h->cfg.window;
  p.negative = h->cfg.negative;
  p.sigmoid = h->cfg.sigmoid;
  p.deterministic = h->cfg.deterministic;
  p.error_flag = h->error_flag;
  p.work_counter = h->work_counter;
  p.exp_table = h->exp_table;
  p.orig_scratch = h->orig_scratch;
  p.scratch_warps = h->scratch_warps;
  p.bf16 = h->cfg.precision == FW2V_BF16;
  p.sr_seed = mix64(0x5EEDF00DULL + h->launches + seed_offset(h->cfg.seed));
  return p;
}

}  // namespace

extern "C" {

void fw2v_config_default(fw2v_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->layer_size = 100;
  c->window = 5;
  c->negative = 5;
  c->epochs = 5;
  c->threads = 12;
  c->msl = 1000;
  c->alpha = 0.025f;
  c->sample = 1e-3f;
  c->sigmoid = FW2V_SIGMOID_TABLE;
  c->precision = FW2V_FP32;
  c->deterministic = 0;
  c->device = 0;
}

void fw2v_lane_layout(int32_t layer_size, int32_t precision, int32_t* vec, int32_t* nv, int64_t* pitch) {
  (void)precision;
  const int64_t P = pitch_for(layer_size);
  if (P <= 64) {
    *vec = 2;
    *nv = 1;
  } else {
    *vec = 4;
    const int n = (int)((P + 127) / 128);
    *nv = n <= 4 ? n : (n <= 6 ? 6 : 8);
  }
  *pitch = P;
}

const char* fw2v_status_string(fw2v_status s) {
  switch (s) {
    case FW2V_OK: return "ok";
    case FW2V_ERR_ARGUMENT: return "invalid argument";
    case FW2V_ERR_CUDA: return "CUDA error";
    case FW2V_ERR_NOMEM: return "out of memory";
    case FW2V_ERR_STATE: return "call out of order";
    case FW2V_ERR_BOUNDS: return "id out of range";
    case FW2V_ERR_NO_DEVICE: return "no usable CUDA device";
    case FW2V_ERR_TOO_LARGE: return "request exceeds a fixed-size library buffer";
  }
  return "unknown status";
}

const char* fw2v_last_error(fw2v_handle* h) { return h ? h->err.c_str() : ""; }

const char* fw2v_version(void) { return "fw2v 1.0 sm_100a"; }

void* fw2v_stream(fw2v_handle* h) { return h ? (void*)h->stream : nullptr; }

fw2v_status fw2v_create(const fw2v_config* cfg, fw2v_handle** out) {
  if (!cfg || !out) return FW2V_ERR_ARGUMENT;
  *out = nullptr;
  const fw2v_config& c = *cfg;
  if (c.layer_size < 1 || c.layer_size > 1024 || c.window < 1 || c.window > kMaxWindow ||
      c.negative < 0 || c.negative > kMaxNegative || c.epochs < 0 || c.threads < 1 || c.msl < 1 ||
      !(c.alpha > 0) || !(c.sample >= 0) || (c.sigmoid != 0 && c.sigmoid != 1) ||
      (c.precision != FW2V_FP32 && c.precision != FW2V_BF16))
    return FW2V_ERR_ARGUMENT;
  if (c.precision == FW2V_BF16 && c.layer_size > 384) return FW2V_ERR_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= c.device || c.device < 0) return FW2V_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c.device) != cudaSuccess || prop.major != 10) return FW2V_ERR_NO_DEVICE;
  if (cudaSetDevice(c.device) != cudaSuccess) return FW2V_ERR_NO_DEVICE;
  const int64_t P = pitch_for(c.layer_size);
  if (train_smem_bytes(c.window, P, 1, 8, false, 4) + train_static_smem() > (size_t)prop.sharedMemPerBlockOptin)
    return FW2V_ERR_ARGUMENT;
  fw2v_handle* h = new fw2v_handle();
  h->cfg = c;
  h->elem = c.precision == FW2V_BF16 ? 2 : 4;
  h->num_sms = prop.multiProcessorCount;
  h->pitch = P;
  auto cleanup = [&](fw2v_status s) {
    fw2v_destroy(h);
    return s;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(FW2V_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&h->sstream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(FW2V_ERR_CUDA);
  for (auto& e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return cleanup(FW2V_ERR_CUDA);
  for (SampleBuf& b : h->buf)
    for (cudaEvent_t* e : {&b.start, &b.ready, &b.freed})
      if (cudaEventCreate(e) != cudaSuccess) return cleanup(FW2V_ERR_CUDA);
  if (dalloc(h->error_flag, 1) != cudaSuccess || dalloc(h->work_counter, 1) != cudaSuccess ||
      dalloc(h->exp_table, kExpTableSize) != cudaSuccess)
    return cleanup(FW2V_ERR_NOMEM);
  h->scratch_warps = train_scratch_warps(h->num_sms);
  if (cudaMalloc(&h->orig_scratch, (size_t)h->scratch_warps * (2 * c.window + 1) * P * h->elem) != cudaSuccess)
    return cleanup(FW2V_ERR_NOMEM);
  // LCG jump-ahead table for up to 32 tokens of 1+K steps each.
  const int n_jump = 32 * (1 + c.negative) + 1;
  std::vector<uint64_t> ja(n_jump), jc(n_jump);
  for (int m = 0; m < n_jump; m++) {
    const Affine j = lcg_jump((uint64_t)m);
    ja[m] = j.a;
    jc[m] = j.c;
  }
  if (dalloc(h->jump_a, n_jump) != cudaSuccess || dalloc(h->jump_c, n_jump) != cudaSuccess)
    return cleanup(FW2V_ERR_NOMEM);
  if (cudaMemcpy(h->jump_a, ja.data(), n_jump * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->jump_c, jc.data(), n_jump * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(FW2V_ERR_CUDA);
  float table[kExpTableSize];
  fw2v_exp_table(table);
  if (cudaMemcpy(h->exp_table, table, sizeof(table), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(h->error_flag, 0, sizeof(int)) != cudaSuccess)
    return cleanup(FW2V_ERR_CUDA);
  *out = h;
  return FW2V_OK;
}

void fw2v_destroy(fw2v_handle* h) {
  if (!h) return;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  dfree_v(h->syn0); dfree_v(h->syn1neg); dfree(h->keep_thr); dfree(h->unigram); dfree(h->exp_table);
  dfree(h->jump_a); dfree(h->jump_c);
  dfree(h->stream_ids); dfree(h->chunk_off); dfree(h->chunk_base); dfree(h->stream_base);
  if (h->sstream) cudaStreamSynchronize(h->sstream);
  dfree(h->lcg); dfree(h->wca); dfree(h->alpha);
  for (SampleBuf& b : h->buf) {
    dfree(b.ent_start); dfree(b.ent_len); dfree(b.ent_alpha);
    dfree(b.kept_ids); dfree(b.kept_state); dfree(b.kept_negs);
    dfree(b.n_entries); dfree(b.n_kept); dfree(b.words); dfree(b.entry_prefix);
    for (cudaEvent_t* e : {&b.start, &b.ready, &b.freed})
      if (*e) cudaEventDestroy(*e);
  }
  if (h->sstream) cudaStreamDestroy(h->sstream);
  dfree(h->error_flag); dfree(h->work_counter); dfree_v(h->orig_scratch);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

fw2v_status fw2v_set_vocab(fw2v_handle* h, const uint32_t* counts, int64_t V, uint64_t train_words) {
  if (!h || !counts || V < 2 || V > (int64_t)INT32_MAX) return fail(h, FW2V_ERR_ARGUMENT, "set_vocab: V >= 2 required");
  CK(h, cudaSetDevice(h->cfg.device));
  const int d = h->cfg.layer_size;
  const int64_t P = h->pitch;
  h->V = V;
  h->train_words = train_words;
  dfree_v(h->syn0);
  dfree_v(h->syn1neg);
  CK(h, cudaMalloc(&h->syn0, (size_t)V * P * h->elem));
  CK(h, cudaMalloc(&h->syn1neg, (size_t)V * P * h->elem));
  CK(h, dalloc(h->keep_thr, V));
  CK(h, dalloc(h->unigram, kUnigramTableSize));
  CK(h, cudaMemsetAsync(h->syn0, 0, (size_t)V * P * h->elem, h->stream));
  CK(h, cudaMemsetAsync(h->syn1neg, 0, (size_t)V * P * h->elem, h->stream));
  std::vector<int64_t> firsts((size_t)V - 1);
  fw2v_unigram_firsts(counts, V, kUnigramTableSize, firsts.data());
  uint32_t* d_counts = nullptr;
  int64_t* d_firsts = nullptr;
  CK(h, dalloc(d_counts, V));
  CK(h, dalloc(d_firsts, V - 1));
  CK(h, cudaMemcpyAsync(d_counts, counts, V * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(d_firsts, firsts.data(), (V - 1) * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
  CK(h, launch_init_tables(h->syn0, h->elem == 2, V, d, P, d_counts, h->cfg.sample, train_words, h->keep_thr, d_firsts,
                           (int)(V - 1), h->unigram, kUnigramTableSize, 1ULL + seed_offset(h->cfg.seed), h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  dfree(d_counts);
  dfree(d_firsts);
  h->n_sampled = h->n_trained = 0;
  return FW2V_OK;
}

// Readable length of each chunk, the kept-id base of each stream, and sampler
// output sets large enough for them (grown when needed).
static fw2v_status layout_streams(fw2v_handle* h) {
  const int T = h->cfg.threads;
  const int K = h->cfg.negative;
  CK(h, launch_corpus_layout(h->stream_ids, h->stream_len, h->chunk_off, h->n_chunks, h->cfg.msl, T,
                             h->chunk_base, h->stream_base, h->stream));
  h->h_stream_base.assign(T + 1, 0);
  CK(h, cudaMemcpyAsync(h->h_stream_base.data(), h->stream_base, (T + 1) * sizeof(int64_t),
                        cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->max_region = 0;
  for (int s = 0; s < T; s++)
    h->max_region = std::max(h->max_region, h->h_stream_base[s + 1] - h->h_stream_base[s]);
  const int64_t cap = std::max<int64_t>(h->h_stream_base[T], 1);
  if (cap > h->sample_cap) {
    for (SampleBuf& b : h->buf) {
      CK(h, dalloc(b.kept_ids, cap));
      CK(h, dalloc(b.kept_state, cap));
      CK(h, dalloc(b.kept_negs, (size_t)cap * std::max(K, 1)));
      CK(h, dalloc(b.ent_start, cap + 2 * (int64_t)T));
      CK(h, dalloc(b.ent_len, cap + 2 * (int64_t)T));
      CK(h, dalloc(b.ent_alpha, cap + 2 * (int64_t)T));
      b.used = false;
    }
    h->sample_cap = cap;
  }
  return FW2V_OK;
}

static fw2v_status check_chunks(fw2v_handle* h, const int64_t* chunk_off, int64_t n_chunks, int64_t stream_len) {
  if (h->cfg.threads > n_chunks || h->cfg.threads > 65535)
    return fail(h, FW2V_ERR_ARGUMENT, "threads (%d) > sentence chunks (%lld)", h->cfg.threads,
                (long long)n_chunks);
  for (int64_t i = 0; i < n_chunks; i++) {
    if (chunk_off[i] < 0 || chunk_off[i] >= stream_len)
      return fail(h, FW2V_ERR_ARGUMENT, "chunk %lld starts outside the stream", (long long)i);
  }
  return FW2V_OK;
}

// The corpus from host memory (on_device false: checked here, copied host to
// device) or from device memory (checked by a kernel, copied on the device).
static fw2v_status load_corpus(fw2v_handle* h, const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                               int64_t n_chunks, bool on_device) {
  if (!h || !stream || !chunk_off || stream_len < 1 || n_chunks < 1)
    return fail(h, FW2V_ERR_ARGUMENT, "load_corpus: empty corpus");
  if (h->V == 0) return fail(h, FW2V_ERR_STATE, "load_corpus before set_vocab");
  fw2v_status s = FW2V_OK;
  if (!on_device) {
    if (stream[stream_len - 1] != 0) return fail(h, FW2V_ERR_ARGUMENT, "load_corpus: stream must end with 0");
    s = check_chunks(h, chunk_off, n_chunks, stream_len);
    if (s != FW2V_OK) return s;
  } else if (h->cfg.threads > n_chunks || h->cfg.threads > 65535) {
    return fail(h, FW2V_ERR_ARGUMENT, "threads (%d) > sentence chunks (%lld)", h->cfg.threads, (long long)n_chunks);
  }
  CK(h, cudaSetDevice(h->cfg.device));
  if (on_device) {
    CK(h, launch_check_corpus(stream, stream_len, chunk_off, n_chunks, h->error_flag, h->stream));
    int flag = 0;
    CK(h, cudaMemcpyAsync(&flag, h->error_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (flag) {
      CK(h, cudaMemsetAsync(h->error_flag, 0, sizeof(int), h->stream));
      return fail(h, FW2V_ERR_ARGUMENT, "load_corpus_device: the stream must end with 0 and every chunk start in it");
    }
  }
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const int T = h->cfg.threads;
  // Nothing may still read the previous corpus.
  CK(h, cudaStreamSynchronize(h->sstream));
  CK(h, cudaStreamSynchronize(h->stream));
  if (stream_len != h->stream_len || !h->stream_ids) CK(h, dalloc(h->stream_ids, stream_len));
  if (n_chunks != h->n_chunks || !h->chunk_off) {
    CK(h, dalloc(h->chunk_off, n_chunks));
    CK(h, dalloc(h->chunk_base, n_chunks + 1));
  }
  if (!h->stream_base) {
    CK(h, dalloc(h->stream_base, T + 1));
    CK(h, dalloc(h->lcg, T));
    CK(h, dalloc(h->wca, T));
    CK(h, dalloc(h->alpha, T));
    for (SampleBuf& b : h->buf) {
      CK(h, dalloc(b.n_entries, T));
      CK(h, dalloc(b.n_kept, T));
      CK(h, dalloc(b.words, T));
      CK(h, dalloc(b.entry_prefix, T + 1));
    }
  }
  h->stream_len = stream_len;
  h->n_chunks = n_chunks;
  CK(h, cudaMemcpyAsync(h->stream_ids, stream, stream_len * sizeof(int32_t), kind, h->stream));
  CK(h, cudaMemcpyAsync(h->chunk_off, chunk_off, n_chunks * sizeof(int64_t), kind, h->stream));
  CK(h, launch_validate_ids(h->stream_ids, stream_len, h->V, h->error_flag, h->stream));
  s = layout_streams(h);
  if (s != FW2V_OK) return s;
  // Stream state (FULL-W2V-driver.cu:113-114): LCG seeded with the id, alpha0.
  std::vector<uint64_t> lcg(T), zero(T, 0);
  std::vector<float> alpha(T, h->cfg.alpha);
  for (int i = 0; i < T; i++) lcg[i] = (uint64_t)i + seed_offset(h->cfg.seed);
  CK(h, cudaMemcpyAsync(h->lcg, lcg.data(), T * sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->wca, zero.data(), T * sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->alpha, alpha.data(), T * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  s = check_flag(h, "load_corpus");
  if (s != FW2V_OK) return s;
  h->n_sampled = h->n_trained = 0;
  h->epochs_done = 0;
  h->words_total = 0;
  return FW2V_OK;
}

fw2v_status fw2v_load_corpus(fw2v_handle* h, const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                             int64_t n_chunks) {
  return load_corpus(h, stream, stream_len, chunk_off, n_chunks, false);
}

fw2v_status fw2v_load_corpus_device(fw2v_handle* h, const int32_t* stream, int64_t stream_len,
                                    const int64_t* chunk_off, int64_t n_chunks) {
  return load_corpus(h, stream, stream_len, chunk_off, n_chunks, true);
}

fw2v_status fw2v_reorder_chunks(fw2v_handle* h, const int64_t* chunk_off, int64_t n_chunks) {
  if (!h || !chunk_off) return FW2V_ERR_ARGUMENT;
  if (!h->stream_ids) return fail(h, FW2V_ERR_STATE, "reorder_chunks before load_corpus");
  if (n_chunks != h->n_chunks) return fail(h, FW2V_ERR_ARGUMENT, "reorder_chunks: chunk count changed");
  if (h->n_sampled != h->n_trained)
    return fail(h, FW2V_ERR_STATE, "reorder_chunks with a sampled epoch not yet trained");
  fw2v_status s = check_chunks(h, chunk_off, n_chunks, h->stream_len);
  if (s != FW2V_OK) return s;
  CK(h, cudaSetDevice(h->cfg.device));
  CK(h, cudaStreamSynchronize(h->sstream));
  CK(h, cudaStreamSynchronize(h->stream));
  CK(h, cudaMemcpyAsync(h->chunk_off, chunk_off, n_chunks * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
  return layout_streams(h);
}

fw2v_status fw2v_shuffle_chunks(fw2v_handle* h, uint64_t key) {
  if (!h) return FW2V_ERR_ARGUMENT;
  if (!h->stream_ids) return fail(h, FW2V_ERR_STATE, "shuffle_chunks before load_corpus");
  if (h->n_sampled != h->n_trained)
    return fail(h, FW2V_ERR_STATE, "shuffle_chunks with a sampled epoch not yet trained");
  CK(h, cudaSetDevice(h->cfg.device));
  CK(h, cudaStreamSynchronize(h->sstream));
  CK(h, launch_fisher_yates(h->chunk_off, h->n_chunks, key, h->stream));
  return layout_streams(h);
}

fw2v_status fw2v_get_chunks(fw2v_handle* h, int64_t* chunk_off) {
  if (!h || !chunk_off) return FW2V_ERR_ARGUMENT;
  if (!h->stream_ids) return fail(h, FW2V_ERR_STATE, "get_chunks before load_corpus");
  CK(h, cudaSetDevice(h->cfg.device));
  CK(h, cudaMemcpyAsync(chunk_off, h->chunk_off, h->n_chunks * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return FW2V_OK;
}

fw2v_status fw2v_sample_epoch(fw2v_handle* h) {
  if (!h) return FW2V_ERR_ARGUMENT;
  if (!h->stream_ids || h->V == 0) return fail(h, FW2V_ERR_STATE, "sample_epoch before load_corpus");
  if (h->n_sampled - h->n_trained >= 2) return fail(h, FW2V_ERR_STATE, "two sampled epochs are waiting to be trained");
  CK(h, cudaSetDevice(h->cfg.device));
  SampleBuf& b = h->buf[h->n_sampled % 2];
  SamplerParams p{};
  p.stream = h->stream_ids;
  p.stream_len = h->stream_len;
  p.chunk_off = h->chunk_off;
  p.n_chunks = h->n_chunks;
  p.stream_base = h->stream_base;
  p.vocab = h->V;
  p.keep_thr = h->keep_thr;
  p.sample = h->cfg.sample;
  p.unigram = h->unigram;
  p.jump_a = h->jump_a;
  p.jump_c = h->jump_c;
  p.table_size = kUnigramTableSize;
  p.threads = h->cfg.threads;
  p.msl = h->cfg.msl;
  p.negative = h->cfg.negative;
  p.epochs = h->cfg.epochs;
  p.alpha0 = h->cfg.alpha;
  p.train_words = h->train_words;
  p.lcg = h->lcg;
  p.wca_own = h->wca;
  p.alpha = h->alpha;
  p.ent_start = b.ent_start;
  p.ent_len = b.ent_len;
  p.ent_alpha = b.ent_alpha;
  p.kept_ids = b.kept_ids;
  p.kept_state = b.kept_state;
  p.kept_negs = b.kept_negs;
  p.n_entries = b.n_entries;
  p.n_kept = b.n_kept;
  p.words = b.words;
  p.error_flag = h->error_flag;
  // The set is reused two epochs later: wait until that epoch's trainer is done.
  if (b.used) CK(h, cudaStreamWaitEvent(h->sstream, b.freed, 0));
  CK(h, cudaEventRecord(b.start, h->sstream));
  CK(h, launch_sampler(p, h->max_region, b.entry_prefix, h->sstream));
  CK(h, cudaEventRecord(b.ready, h->sstream));
  h->n_sampled++;
  return FW2V_OK;
}

// The most recently sampled epoch's set, complete.
static fw2v_status last_sampled(fw2v_handle* h, SampleBuf** out) {
  if (!h || h->n_sampled == 0) return fail(h, FW2V_ERR_STATE, "no sampled epoch");
  SampleBuf& b = h->buf[(h->n_sampled - 1) % 2];
  CK(h, cudaEventSynchronize(b.ready));
  *out = &b;
  return FW2V_OK;
}

fw2v_status fw2v_epoch_sample_sizes(fw2v_handle* h, int64_t* n_entries, int64_t* n_kept) {
  SampleBuf* b = nullptr;
  fw2v_status st = last_sampled(h, &b);
  if (st != FW2V_OK) return st;
  const int T = h->cfg.threads;
  std::vector<int64_t> ne(T), nk(T);
  CK(h, cudaMemcpyAsync(ne.data(), b->n_entries, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaMemcpyAsync(nk.data(), b->n_kept, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  st = check_flag(h, "sample_epoch");
  if (st != FW2V_OK) return st;
  int64_t a = 0, c = 0;
  for (int i = 0; i < T; i++) {
    a += ne[i];
    c += nk[i];
  }
  if (n_entries) *n_entries = a;
  if (n_kept) *n_kept = c;
  return FW2V_OK;
}

fw2v_status fw2v_epoch_samples(fw2v_handle* h, int32_t* lens, float* alphas, int32_t* ids, int32_t* negs,
                               int64_t* entries_per_stream, int64_t* kept_per_stream, uint64_t* words_per_stream) {
  SampleBuf* b = nullptr;
  fw2v_status st = last_sampled(h, &b);
  if (st != FW2V_OK) return st;
  const int T = h->cfg.threads;
  const int K = h->cfg.negative;
  std::vector<int64_t> ne(T), nk(T);
  std::vector<uint64_t> wr(T);
  CK(h, cudaMemcpyAsync(ne.data(), b->n_entries, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaMemcpyAsync(nk.data(), b->n_kept, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaMemcpyAsync(wr.data(), b->words, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  st = check_flag(h, "sample_epoch");
  if (st != FW2V_OK) return st;
  int64_t eo = 0, ko = 0;
  for (int s = 0; s < T; s++) {
    const int64_t kb = h->h_stream_base[s];
    const int64_t eb = kb + 2 * (int64_t)s;
    if (lens) CK(h, cudaMemcpyAsync(lens + eo, b->ent_len + eb, ne[s] * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    if (alphas) CK(h, cudaMemcpyAsync(alphas + eo, b->ent_alpha + eb, ne[s] * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (ids) CK(h, cudaMemcpyAsync(ids + ko, b->kept_ids + kb, nk[s] * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    if (negs && K > 0)
      CK(h, cudaMemcpyAsync(negs + ko * K, b->kept_negs + kb * K, nk[s] * K * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    if (entries_per_stream) entries_per_stream[s] = ne[s];
    if (kept_per_stream) kept_per_stream[s] = nk[s];
    if (words_per_stream) words_per_stream[s] = wr[s];
    eo += ne[s];
    ko += nk[s];
  }
  CK(h, cudaStreamSynchronize(h->stream));
  return FW2V_OK;
}

// Launch the trainer on the oldest sampled epoch (asynchronous).
static fw2v_status launch_epoch_train(fw2v_handle* h, SampleBuf** used) {
  if (!h || h->n_trained >= h->n_sampled) return fail(h, FW2V_ERR_STATE, "train_sampled without a sampled epoch");
  CK(h, cudaSetDevice(h->cfg.device));
  SampleBuf& b = h->buf[h->n_trained % 2];
  TrainParams p = base_train_params(h);
  p.ids = b.kept_ids;
  p.negs = b.kept_negs;
  p.source = kSourceEpoch;
  p.entry_prefix = b.entry_prefix;
  p.stream_base = h->stream_base;
  p.threads = h->cfg.threads;
  p.ent_start = b.ent_start;
  p.ent_len = b.ent_len;
  p.ent_alpha = b.ent_alpha;
  CK(h, cudaStreamWaitEvent(h->stream, b.ready, 0));
  CK(h, cudaEventRecord(h->ev[1], h->stream));
  CK(h, cudaMemsetAsync(h->work_counter, 0, sizeof(unsigned long long), h->stream));
  CK(h, launch_train(p, h->num_sms, h->stream));
  h->launches++;
  CK(h, cudaEventRecord(h->ev[2], h->stream));
  CK(h, cudaEventRecord(b.freed, h->stream));
  b.used = true;
  h->n_trained++;
  *used = &b;
  return FW2V_OK;
}

// Wait for the trainer, then count the epoch's words and fill the stats.
static fw2v_status finish_epoch_train(fw2v_handle* h, SampleBuf* b, fw2v_epoch_stats* stats) {
  const int T = h->cfg.threads;
  std::vector<uint64_t> wr(T);
  std::vector<int64_t> ne(T), nk(T);
  CK(h, cudaMemcpyAsync(wr.data(), b->words, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  if (stats) {
    CK(h, cudaMemcpyAsync(ne.data(), b->n_entries, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaMemcpyAsync(nk.data(), b->n_kept, T * sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
  }
  fw2v_status s = check_flag(h, "train");
  if (s != FW2V_OK) return s;
  uint64_t words = 0;
  for (int i = 0; i < T; i++) words += wr[i];
  h->words_total += words;
  h->epochs_done++;
  if (stats) {
    stats->words_read = words;
    stats->words_kept = 0;
    stats->sentences = 0;
    for (int i = 0; i < T; i++) {
      stats->words_kept += (uint64_t)nk[i];
      stats->sentences += (uint64_t)ne[i];
    }
    CK(h, cudaEventElapsedTime(&stats->sampler_ms, b->start, b->ready));
    CK(h, cudaEventElapsedTime(&stats->train_ms, h->ev[1], h->ev[2]));
  }
  return FW2V_OK;
}

fw2v_status fw2v_train_sampled(fw2v_handle* h, fw2v_epoch_stats* stats) {
  SampleBuf* b = nullptr;
  fw2v_status s = launch_epoch_train(h, &b);
  if (s != FW2V_OK) return s;
  return finish_epoch_train(h, b, stats);
}

// One epoch: sample it unless that is already done, launch its trainer, and
// while it runs sample the next epoch on the sampler stream (if the configured
// epochs go on) so that sampling overlaps training.
fw2v_status fw2v_train_epoch(fw2v_handle* h, fw2v_epoch_stats* stats) {
  if (!h) return FW2V_ERR_ARGUMENT;
  fw2v_status s = FW2V_OK;
  if (h->n_sampled == h->n_trained) s = fw2v_sample_epoch(h);
  if (s != FW2V_OK) return s;
  SampleBuf* b = nullptr;
  s = launch_epoch_train(h, &b);
  if (s != FW2V_OK) return s;
  if (h->n_sampled < h->cfg.epochs && h->n_sampled == h->n_trained) {
    s = fw2v_sample_epoch(h);
    if (s != FW2V_OK) return s;
  }
  return finish_epoch_train(h, b, stats);
}

fw2v_status fw2v_train(fw2v_handle* h, uint64_t* words_read) {
  if (!h) return FW2V_ERR_ARGUMENT;
  uint64_t before = h->words_total;
  while (h->epochs_done < h->cfg.epochs) {
    fw2v_status s = fw2v_train_epoch(h, nullptr);
    if (s != FW2V_OK) return s;
  }
  if (words_read) *words_read = h->words_total - before;
  return FW2V_OK;
}

fw2v_status fw2v_words_trained(fw2v_handle* h, uint64_t* words) {
  if (!h || !words) return FW2V_ERR_ARGUMENT;
  *words = h->words_total;
  return FW2V_OK;
}

static fw2v_status copy_table(fw2v_handle* h, void* dev, float* host, int64_t stride, bool to_host) {
  if (!h || !host || stride < h->cfg.layer_size) return fail(h, FW2V_ERR_ARGUMENT, "table copy: bad stride");
  if (h->V == 0) return fail(h, FW2V_ERR_STATE, "tables not allocated");
  CK(h, cudaSetDevice(h->cfg.device));
  CK(h, cudaStreamSynchronize(h->sstream));
  const int d = h->cfg.layer_size;
  if (h->elem == 4) {
    const size_t w = (size_t)d * sizeof(float);
    if (to_host)
      CK(h, cudaMemcpy2DAsync(host, stride * sizeof(float), dev, h->pitch * sizeof(float), w, h->V,
                              cudaMemcpyDeviceToHost, h->stream));
    else
      CK(h, cudaMemcpy2DAsync(dev, h->pitch * sizeof(float), host, stride * sizeof(float), w, h->V,
                              cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return FW2V_OK;
  }
  // bfloat16 tables: widen (exact) on the way out, round to nearest on the way in
  std::vector<uint16_t> tmp((size_t)h->V * d);
  const size_t w = (size_t)d * sizeof(uint16_t);
  if (to_host) {
    CK(h, cudaMemcpy2DAsync(tmp.data(), w, dev, h->pitch * sizeof(uint16_t), w, h->V, cudaMemcpyDeviceToHost,
                            h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (int64_t r = 0; r < h->V; r++)
      for (int c = 0; c < d; c++) host[r * stride + c] = bf16_value(tmp[(size_t)r * d + c]);
  } else {
    for (int64_t r = 0; r < h->V; r++)
      for (int c = 0; c < d; c++) tmp[(size_t)r * d + c] = bf16_nearest(host[r * stride + c]);
    CK(h, cudaMemcpy2DAsync(dev, h->pitch * sizeof(uint16_t), tmp.data(), w, w, h->V, cudaMemcpyHostToDevice,
                            h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
  }
  return FW2V_OK;
}

fw2v_status fw2v_get_syn0(fw2v_handle* h, float* out, int64_t row_stride) {
  return copy_table(h, h ? h->syn0 : nullptr, out, row_stride, true);
}
fw2v_status fw2v_get_syn1neg(fw2v_handle* h, float* out, int64_t row_stride) {
  return copy_table(h, h ? h->syn1neg : nullptr, out, row_stride, true);
}
fw2v_status fw2v_set_tables(fw2v_handle* h, const float* syn0, const float* syn1neg, int64_t row_stride) {
  fw2v_status s = FW2V_OK;
  if (syn0) s = copy_table(h, h ? h->syn0 : nullptr, const_cast<float*>(syn0), row_stride, false);
  if (s == FW2V_OK && syn1neg) s = copy_table(h, h ? h->syn1neg : nullptr, const_cast<float*>(syn1neg), row_stride, false);
  return s;
}

// Shared by fw2v_train_sentences and fw2v_heldout_loss: copy host sentences to
// temporary device buffers.
struct DeviceSentences {
  int32_t* ids = nullptr;
  int32_t* negs = nullptr;
  int64_t* starts = nullptr;
  int32_t* lens = nullptr;
  float* alphas = nullptr;
  ~DeviceSentences() {
    dfree(ids); dfree(negs); dfree(starts); dfree(lens); dfree(alphas);
  }
};

static fw2v_status upload_sentences(fw2v_handle* h, DeviceSentences& ds, const int32_t* ids, const int32_t* negs,
                                    const int64_t* starts, const int32_t* lens, const float* alphas, int64_t n) {
  const int K = h->cfg.negative;
  int64_t n_ids = 0;
  for (int64_t s = 0; s < n; s++) {
    if (starts[s] < 0 || lens[s] < 0) return fail(h, FW2V_ERR_ARGUMENT, "sentence %lld: negative start/len", (long long)s);
    n_ids = std::max(n_ids, starts[s] + lens[s]);
  }
  CK(h, dalloc(ds.ids, n_ids));
  CK(h, dalloc(ds.negs, n_ids * std::max(K, 1)));
  CK(h, dalloc(ds.starts, n));
  CK(h, dalloc(ds.lens, n));
  CK(h, dalloc(ds.alphas, n));
  if (n_ids > 0) {
    CK(h, cudaMemcpyAsync(ds.ids, ids, n_ids * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    if (K > 0) CK(h, cudaMemcpyAsync(ds.negs, negs, n_ids * K * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  }
  CK(h, cudaMemcpyAsync(ds.starts, starts, n * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(ds.lens, lens, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  if (alphas) CK(h, cudaMemcpyAsync(ds.alphas, alphas, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  return FW2V_OK;
}

fw2v_status fw2v_train_sentences(fw2v_handle* h, const int32_t* ids, const int32_t* negs, const int64_t* starts,
                                 const int32_t* lens, const float* alphas, int64_t n) {
  if (!h || n < 0 || (n > 0 && (!ids || !starts || !lens || !alphas || (h->cfg.negative > 0 && !negs))))
    return fail(h, FW2V_ERR_ARGUMENT, "train_sentences: null input");
  if (h->V == 0) return fail(h, FW2V_ERR_STATE, "train_sentences before set_vocab");
  if (n == 0) return FW2V_OK;
  CK(h, cudaSetDevice(h->cfg.device));
  DeviceSentences ds;
  fw2v_status s = upload_sentences(h, ds, ids, negs, starts, lens, alphas, n);
  if (s != FW2V_OK) return s;
  TrainParams p = base_train_params(h);
  p.ids = ds.ids;
  p.negs = ds.negs;
  p.source = kSourceExplicit;
  p.starts = ds.starts;
  p.lens = ds.lens;
  p.alphas = ds.alphas;
  p.n_sentences = n;
  CK(h, cudaMemsetAsync(h->work_counter, 0, sizeof(unsigned long long), h->stream));
  CK(h, launch_train(p, h->num_sms, h->stream));
  h->launches++;
  return check_flag(h, "train_sentences");
}

fw2v_status fw2v_heldout_loss(fw2v_handle* h, const int32_t* ids, const int32_t* negs, const int64_t* starts,
                              const int32_t* lens, int64_t n, double* loss_sum, int64_t* pairs) {
  if (!h || !loss_sum || !pairs || n < 0) return fail(h, FW2V_ERR_ARGUMENT, "heldout_loss: null output");
  if (h->V == 0) return fail(h, FW2V_ERR_STATE, "heldout_loss before set_vocab");
  *loss_sum = 0;
  *pairs = 0;
  if (n == 0) return FW2V_OK;
  CK(h, cudaSetDevice(h->cfg.device));
  DeviceSentences ds;
  fw2v_status s = upload_sentences(h, ds, ids, negs, starts, lens, nullptr, n);
  if (s != FW2V_OK) return s;
  double* d_loss = nullptr;
  unsigned long long* d_pairs = nullptr;
  CK(h, dalloc(d_loss, 1));
  CK(h, dalloc(d_pairs, 1));
  CK(h, cudaMemsetAsync(d_loss, 0, sizeof(double), h->stream));
  CK(h, cudaMemsetAsync(d_pairs, 0, sizeof(unsigned long long), h->stream));
  TrainParams p = base_train_params(h);
  p.ids = ds.ids;
  p.negs = ds.negs;
  p.starts = ds.starts;
  p.lens = ds.lens;
  p.n_sentences = n;
  CK(h, launch_heldout(p, d_loss, d_pairs, h->stream));
  unsigned long long np = 0;
  CK(h, cudaMemcpyAsync(loss_sum, d_loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaMemcpyAsync(&np, d_pairs, sizeof(np), cudaMemcpyDeviceToHost, h->stream));
  s = check_flag(h, "heldout_loss");
  dfree(d_loss);
  dfree(d_pairs);
  *pairs = (int64_t)np;
  return s;
}

fw2v_status fw2v_get_unigram(fw2v_handle* h, int64_t first, int64_t n, int32_t* out) {
  if (!h || !out || first < 0 || n < 0 || first + n > kUnigramTableSize)
    return fail(h, FW2V_ERR_ARGUMENT, "get_unigram: range");
  if (!h->unigram) return fail(h, FW2V_ERR_STATE, "get_unigram before set_vocab");
  CK(h, cudaSetDevice(h->cfg.device));
  CK(h, cudaMemcpyAsync(out, h->unigram + first, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return FW2V_OK;
}

}  // extern "C"
