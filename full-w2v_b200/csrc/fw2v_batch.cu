// Batched training of many independent SGNS jobs (include/fw2v.h, "Batched
// training"): job set-up, the round plan of an epoch, the epoch loop as one
// stream of launches (or one captured CUDA graph), and the autotuner.
//
// Layout.  Each job owns its tables, keep thresholds, unigram run boundaries
// (negatives are found by binary search over them: the same ids as the
// reference's 1e8-entry table, without 400 MB per job), token stream and
// chunk table.  Sampling streams of all jobs are numbered globally (job j's
// stream s is gfirst[j] + s) for their carried LCG / word-count / learning-rate
// state.  An epoch is a fixed sequence of rounds; round r is a list of
// (job, stream) pairs in training order (stream_order: groups of jobs whose
// tables fit the group budget, each group's streams s = 0, 1, ... and within
// each s by job), cut where the round's readable tokens would pass
// round_tokens.  Two sets of
// round buffers (kept ids, their LCG states and negatives, entries) alternate:
// round r+1 is sampled on the sampler stream while round r trains.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fw2v.h"
#include "fw2v_batch.cuh"

extern "C" void fw2v_exp_table(float* t);
extern "C" int fw2v_unigram_firsts(const uint32_t* counts, int64_t V, int64_t size, int64_t* firsts);

namespace fw2v {
cudaError_t launch_init_tables(void* syn0, bool bf16, int64_t V, int d, int64_t pitch, const uint32_t* d_counts,
                               float sample, uint64_t train_words, int32_t* keep_thr, const int64_t* d_firsts,
                               int n_firsts, int32_t* unigram, int64_t table_size, uint64_t start,
                               cudaStream_t st);
cudaError_t launch_validate_ids(const int32_t* ids, int64_t n, int64_t vocab, int* flag, cudaStream_t st);
cudaError_t launch_check_corpus(const int32_t* stream, int64_t len, const int64_t* chunk_off, int64_t n, int* flag,
                                cudaStream_t st);
cudaError_t launch_corpus_layout(const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                                 int64_t n_chunks, int msl, int threads, int64_t* chunk_base,
                                 int64_t* stream_base, cudaStream_t st);
cudaError_t launch_sampler_round(const SamplerParams* d_jobs, const BatchRound& r, int epoch, int64_t max_region,
                                 bool any_negatives, const int64_t* n_entries, const int64_t* n_kept,
                                 const uint64_t* words, int n_jobs, int64_t* job_uid, int64_t* uid_base,
                                 unsigned long long* job_words, unsigned long long* job_kept,
                                 int64_t* entry_prefix, cudaStream_t st);
#define FW2V_BATCH_EXTERN(T, F)                                                                     \
  extern template cudaError_t batch_grid<T, F>(int64_t, int, int, int, int64_t, int, int*, int*, size_t*); \
  extern template cudaError_t batch_launch<T, F>(const BatchTrainArgs&, int, int, size_t, cudaStream_t);
FW2V_BATCH_EXTERN(float, 0)
FW2V_BATCH_EXTERN(float, 1)
FW2V_BATCH_EXTERN(float, 2)
FW2V_BATCH_EXTERN(bf16_t, 0)
FW2V_BATCH_EXTERN(bf16_t, 1)
FW2V_BATCH_EXTERN(bf16_t, 2)
#undef FW2V_BATCH_EXTERN
}  // namespace fw2v

using namespace fw2v;

namespace {

struct BatchJob {
  fw2v_config cfg{};
  int64_t V = 0;
  uint64_t train_words = 0;
  int64_t pitch = 0;
  uint64_t soff = 0;
  void* syn0 = nullptr;
  void* syn1neg = nullptr;
  int32_t* keep_thr = nullptr;
  int64_t* firsts = nullptr;
  int32_t* stream = nullptr;
  int64_t stream_len = 0;
  int64_t* chunk_off = nullptr;
  int64_t n_chunks = 0;
  std::vector<int64_t> sbase;  // threads + 1: readable-token prefix of its streams
  int64_t gfirst = 0;          // global number of its stream 0
  int lane_vec = 4, lane_nv = 1, stages = 6;
  // bit 0: target rows of each group copied while the previous group trains;
  // bit 1: context rows staged by bulk copies
  int prefetch = 0;
  int family() const { return batch_family(lane_nv, stages); }
};

struct StreamItem {
  int32_t job, local;
  int64_t gstream, tokens;
};

struct RoundPlan {
  int family = 0;          // kernel family of all its jobs
  int n = 0;
  int64_t kept = 0;        // readable tokens of its streams
  int64_t max_region = 0;  // largest stream
  void* dev = nullptr;     // job[n] | local[n] | gstream[n] | kbase[n+1]
  BatchRound view{};
};

struct RoundBuf {
  int32_t* kept_ids = nullptr;
  uint64_t* kept_state = nullptr;
  int32_t* kept_negs = nullptr;
  int64_t* ent_start = nullptr;
  int32_t* ent_len = nullptr;
  float* ent_alpha = nullptr;
  int64_t* n_entries = nullptr;
  int64_t* n_kept = nullptr;
  uint64_t* words = nullptr;
  int64_t* entry_prefix = nullptr;
  int64_t* uid_base = nullptr;
  SamplerParams* d_sp = nullptr;  // per job
  TrainParams* d_tp = nullptr;    // per job
  cudaEvent_t ready = nullptr, freed = nullptr;
};

// Lane layouts (vector width, vectors per lane) and stage counts a job of
// layer size d may use: the lanes must cover d, no vector may lie wholly past
// it, and wide rows use 4-float vectors.
bool valid_shape(int d, int vec, int nv, int stages) {
  if (vec != 2 && vec != 4) return false;
  if (nv < 1 || nv > 3 || (nv > 1 && vec != 4)) return false;
  if (d > 32 * vec * nv || (nv > 1 && d <= 32 * vec * (nv - 1))) return false;
  if (nv >= 3 && stages > 4) return false;  // no 6-stage body for rows of three vectors
  for (int s : kBatchStages)
    if (s == stages) return true;
  return false;
}

// Layout class of a layer size: d <= 64, <= 128, <= 256, <= 384.
int layout_class(int64_t pitch) { return pitch <= 64 ? 0 : pitch <= 128 ? 1 : pitch <= 256 ? 2 : 3; }

// Default stages: the fewest groups of targets per centre, then the fewest
// idle stages; rows of three vectors per lane stop at 4 (their 6-stage body
// does not fit the register file).
int default_stages(int negative, int nv = 1) {
  const int t = negative + 1;
  int best = 6, best_groups = 1 << 30, best_idle = 1 << 30;
  for (int s : kBatchStages) {
    if (nv >= 3 && s > 4) continue;
    const int g = (t + s - 1) / s, idle = g * s - t;
    if (g < best_groups || (g == best_groups && idle < best_idle)) {
      best = s;
      best_groups = g;
      best_idle = idle;
    }
  }
  return best;
}

}  // namespace

struct fw2v_batch {
  fw2v_batch_config cfg{};
  int num_sms = 0;
  int64_t l2_bytes = 0;
  size_t elem = 4;
  cudaStream_t st = nullptr, sst = nullptr;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr, ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  std::vector<BatchJob> jobs;
  int negative = -1;
  uint64_t* jump_a = nullptr;
  uint64_t* jump_c = nullptr;
  float* exp_table = nullptr;
  int* error_flag = nullptr;
  unsigned long long* counter = nullptr;
  // global stream state
  uint64_t* lcg = nullptr;
  uint64_t* wca = nullptr;
  float* alpha = nullptr;
  int64_t n_gstreams = 0, gstream_cap = 0;
  // per job
  int64_t* job_uid = nullptr;
  unsigned long long* job_words = nullptr;  // this call
  unsigned long long* job_kept = nullptr;
  std::vector<unsigned long long> words_total, kept_total;  // since added
  int64_t job_cap = 0;
  // plan
  bool planned = false;
  std::vector<RoundPlan> rounds;
  RoundBuf buf[2];
  int64_t buf_kept_cap = 0, buf_stream_cap = 0;
  void* orig_scratch = nullptr;
  int64_t scratch_elems = 0, scratch_warps = 0, scratch_bytes = 0;
  // per family; 0 warps: the count that keeps the most warps resident
  int warps_per_block[kBatchFamilies] = {0, 0, 0}, blocks_per_sm[kBatchFamilies] = {0, 0, 0};
  int epochs_run = 0;  // batch epochs trained so far: job j has trained min(epochs_run, its epochs)
  int next_buf = 0;  // the buffer set of the next round
  std::vector<unsigned long long> words_snap, kept_snap;  // counters at the end of the last call
  std::vector<cudaEvent_t> round_ev;  // 2 per training launch of a call: its device time
};

namespace {

fw2v_status bfail(fw2v_batch* b, fw2v_status s, const char* fmt, ...) {
  if (b) {
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof(msg), fmt, ap);
    va_end(ap);
    b->err = msg;
  }
  return s;
}

#define BCK(b, call)                                                                          \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? FW2V_ERR_NOMEM : FW2V_ERR_CUDA,     \
                   "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);     \
    }                                                                                         \
  } while (0)

template <typename T>
void bfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

template <typename T>
cudaError_t balloc(T*& p, size_t n) {
  bfree(p);
  return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
}

// Grow a device array to hold n elements, keeping its first `keep` elements.
template <typename T>
cudaError_t grow(T*& p, int64_t keep, int64_t n) {
  T* q = nullptr;
  cudaError_t e = cudaMalloc((void**)&q, std::max<int64_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  if (p && keep > 0) {
    e = cudaMemcpy(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      cudaFree(q);
      return e;
    }
  }
  bfree(p);
  p = q;
  return cudaSuccess;
}

void free_plan(fw2v_batch* b) {
  for (RoundPlan& r : b->rounds) bfree(r.dev);
  b->rounds.clear();
  for (RoundBuf& rb : b->buf) {
    bfree(rb.kept_ids); bfree(rb.kept_state); bfree(rb.kept_negs);
    bfree(rb.ent_start); bfree(rb.ent_len); bfree(rb.ent_alpha);
    bfree(rb.n_entries); bfree(rb.n_kept); bfree(rb.words); bfree(rb.entry_prefix); bfree(rb.uid_base);
    bfree(rb.d_sp); bfree(rb.d_tp);
  }
  b->buf_kept_cap = b->buf_stream_cap = 0;
  b->planned = false;
}

int64_t shape_smem_floats(const BatchJob& j, int elem) {
  return warp_smem_bytes(2 * j.cfg.window + 1, j.stages, (j.prefetch & 1) != 0, j.pitch, elem) / 4;
}
int64_t shape_scratch_elems(const BatchJob& j) { return (int64_t)(2 * j.cfg.window + 1) * j.pitch; }

SamplerParams sampler_params(const fw2v_batch* b, const BatchJob& j, const RoundBuf& rb) {
  SamplerParams p{};
  p.stream = j.stream;
  p.stream_len = j.stream_len;
  p.chunk_off = j.chunk_off;
  p.n_chunks = j.n_chunks;
  p.vocab = j.V;
  p.keep_thr = j.keep_thr;
  p.sample = j.cfg.sample;
  p.unigram = nullptr;
  p.unigram_firsts = j.firsts;
  p.n_firsts = j.V - 1;
  p.table_size = kUnigramTableSize;
  p.jump_a = b->jump_a;
  p.jump_c = b->jump_c;
  p.threads = j.cfg.threads;
  p.msl = j.cfg.msl;
  p.negative = j.cfg.negative;
  p.epochs = j.cfg.epochs;
  p.alpha0 = j.cfg.alpha;
  p.train_words = j.train_words;
  p.lcg = b->lcg;
  p.wca_own = b->wca;
  p.alpha = b->alpha;
  p.ent_start = rb.ent_start;
  p.ent_len = rb.ent_len;
  p.ent_alpha = rb.ent_alpha;
  p.kept_ids = rb.kept_ids;
  p.kept_state = rb.kept_state;
  p.kept_negs = rb.kept_negs;
  p.n_entries = rb.n_entries;
  p.n_kept = rb.n_kept;
  p.words = rb.words;
  p.error_flag = b->error_flag;
  return p;
}

// sr_seed holds the job's seed offset: the kernel adds the (absolute) epoch
// and mixes, which is the single-job seed of the same launch number.
TrainParams train_params(const fw2v_batch* b, const BatchJob& j, const RoundBuf& rb) {
  TrainParams p{};
  p.syn0 = j.syn0;
  p.syn1neg = j.syn1neg;
  p.pitch = j.pitch;
  p.vocab = j.V;
  p.d = j.cfg.layer_size;
  p.window = j.cfg.window;
  p.negative = j.cfg.negative;
  p.sigmoid = FW2V_SIGMOID_TABLE;
  p.ids = rb.kept_ids;
  p.negs = rb.kept_negs;
  p.source = kSourceEpoch;
  p.deterministic = b->cfg.deterministic;
  p.error_flag = b->error_flag;
  p.exp_table = b->exp_table;
  p.sr_seed = j.soff;
  p.bf16 = b->elem == 2;
  p.lane_vec = j.lane_vec;
  p.lane_nv = j.lane_nv;
  p.stages = j.stages;
  p.prefetch = j.prefetch & 1;
  p.bulk = (j.prefetch >> 1) & 1;
  return p;
}

// Streams of the jobs with in[j] set, in training order.  Jobs, in index
// order, are gathered into groups whose tables together fit the group budget
// (a larger job is a group of its own); a group's streams are taken
// s = 0, 1, ... and within each s by job.  The work queue hands out sentences
// in this order, so the warps in flight at any time train a few streams of
// one group: interleaving its jobs keeps fewer warps at once on any one job's
// rows than training it alone would, and bounding the group keeps the rows in
// use resident in L2 between the sentences that touch them.  Each job's own
// streams keep their order, so deterministic results do not depend on it.
std::vector<StreamItem> stream_order(const fw2v_batch* b, const std::vector<char>& in) {
  const int64_t budget = b->cfg.group_bytes ? b->cfg.group_bytes : b->l2_bytes / 2;
  std::vector<StreamItem> out;
  size_t g0 = 0;
  while (g0 < b->jobs.size()) {
    size_t g1 = g0;
    int64_t bytes = 0;
    int max_t = 0;
    for (; g1 < b->jobs.size(); g1++) {
      const BatchJob& j = b->jobs[g1];
      if (!in[g1]) continue;
      const int64_t tb = 2 * j.V * j.pitch * (int64_t)b->elem;
      if (budget > 0 && max_t > 0 && bytes + tb > budget) break;
      bytes += tb;
      max_t = std::max(max_t, j.cfg.threads);
    }
    for (int s = 0; s < max_t; s++)
      for (size_t ji = g0; ji < g1; ji++) {
        const BatchJob& j = b->jobs[ji];
        if (in[ji] && s < j.cfg.threads)
          out.push_back({(int32_t)ji, s, j.gfirst + s, j.sbase[s + 1] - j.sbase[s]});
      }
    g0 = g1;
  }
  return out;
}

// The round plan of an epoch and buffers for its largest round.
fw2v_status plan(fw2v_batch* b) {
  if (b->planned) return FW2V_OK;
  if (b->jobs.empty()) return bfail(b, FW2V_ERR_STATE, "batch has no jobs");
  free_plan(b);
  const int64_t cap = b->cfg.round_tokens > 0 ? b->cfg.round_tokens : (int64_t)1 << 27;
  for (int fam = 0; fam < kBatchFamilies; fam++) {
  std::vector<char> in(b->jobs.size());
  for (size_t ji = 0; ji < b->jobs.size(); ji++) in[ji] = b->jobs[ji].family() == fam;
  const std::vector<StreamItem> order = stream_order(b, in);
  size_t i = 0;
  while (i < order.size()) {
    size_t e = i;
    int64_t tok = 0;
    while (e < order.size() && (e == i || (tok + order[e].tokens <= cap && e - i < 65535))) tok += order[e++].tokens;
    RoundPlan r;
    r.family = fam;
    r.n = (int)(e - i);
    std::vector<int32_t> job(r.n), local(r.n);
    std::vector<int64_t> gs(r.n), kb(r.n + 1, 0);
    for (int g = 0; g < r.n; g++) {
      const StreamItem& it = order[i + g];
      job[g] = it.job;
      local[g] = it.local;
      gs[g] = it.gstream;
      kb[g + 1] = kb[g] + it.tokens;
      r.max_region = std::max(r.max_region, it.tokens);
    }
    r.kept = kb[r.n];
    const size_t bytes = (size_t)r.n * 8 * 2 + (size_t)r.n * 8 + (size_t)(r.n + 1) * 8;
    BCK(b, cudaMalloc(&r.dev, bytes));
    char* base = (char*)r.dev;
    int64_t* d_gs = (int64_t*)base;
    int64_t* d_kb = d_gs + r.n;
    int32_t* d_job = (int32_t*)(d_kb + r.n + 1);
    int32_t* d_local = d_job + r.n;
    BCK(b, cudaMemcpy(d_gs, gs.data(), r.n * 8, cudaMemcpyHostToDevice));
    BCK(b, cudaMemcpy(d_kb, kb.data(), (r.n + 1) * 8, cudaMemcpyHostToDevice));
    BCK(b, cudaMemcpy(d_job, job.data(), r.n * 4, cudaMemcpyHostToDevice));
    BCK(b, cudaMemcpy(d_local, local.data(), r.n * 4, cudaMemcpyHostToDevice));
    r.view = BatchRound{d_job, d_local, d_gs, d_kb, r.n};
    b->rounds.push_back(r);
    b->buf_kept_cap = std::max(b->buf_kept_cap, r.kept);
    b->buf_stream_cap = std::max<int64_t>(b->buf_stream_cap, r.n);
    i = e;
  }
  }
  const int64_t kc = std::max<int64_t>(b->buf_kept_cap, 1), sc = b->buf_stream_cap;
  const int K = std::max(b->negative, 1);
  for (RoundBuf& rb : b->buf) {
    BCK(b, balloc(rb.kept_ids, kc));
    BCK(b, balloc(rb.kept_state, kc));
    BCK(b, balloc(rb.kept_negs, (size_t)kc * K));
    BCK(b, balloc(rb.ent_start, kc + 2 * sc));
    BCK(b, balloc(rb.ent_len, kc + 2 * sc));
    BCK(b, balloc(rb.ent_alpha, kc + 2 * sc));
    BCK(b, balloc(rb.n_entries, sc));
    BCK(b, balloc(rb.n_kept, sc));
    BCK(b, balloc(rb.words, sc));
    BCK(b, balloc(rb.entry_prefix, sc + 1));
    BCK(b, balloc(rb.uid_base, sc));
    BCK(b, balloc(rb.d_sp, b->jobs.size()));
    BCK(b, balloc(rb.d_tp, b->jobs.size()));
  }
  b->planned = true;
  return FW2V_OK;
}

// Per-job parameter blocks of both buffer sets, and scratch for the current shapes.
fw2v_status upload_params(fw2v_batch* b) {
  const size_t J = b->jobs.size();
  for (RoundBuf& rb : b->buf) {
    std::vector<SamplerParams> sp(J);
    std::vector<TrainParams> tp(J);
    for (size_t j = 0; j < J; j++) {
      sp[j] = sampler_params(b, b->jobs[j], rb);
      tp[j] = train_params(b, b->jobs[j], rb);
    }
    BCK(b, cudaMemcpy(rb.d_sp, sp.data(), J * sizeof(SamplerParams), cudaMemcpyHostToDevice));
    BCK(b, cudaMemcpy(rb.d_tp, tp.data(), J * sizeof(TrainParams), cudaMemcpyHostToDevice));
  }
  int64_t se = 0;
  for (const BatchJob& j : b->jobs) se = std::max(se, shape_scratch_elems(j));
  const int64_t warps = (int64_t)b->num_sms * 64;
  const int64_t bytes = warps * se * (int64_t)b->elem;
  if (bytes > b->scratch_bytes) {
    bfree(b->orig_scratch);
    BCK(b, cudaMalloc(&b->orig_scratch, bytes));
    b->scratch_bytes = bytes;
  }
  b->scratch_elems = se;
  b->scratch_warps = warps;
  return FW2V_OK;
}

struct Grid {
  int blocks = 0, threads = 0;
  size_t smem = 0;
  int64_t smem_floats = 0;
};

// Grid of kernel family `fam` for the jobs `active` of that family.
fw2v_status grid_for(fw2v_batch* b, const std::vector<int>& active, int fam, int wpb, int cap, Grid* g) {
  g->smem_floats = 0;
  for (int j : active)
    if (b->jobs[j].family() == fam)
      g->smem_floats = std::max(g->smem_floats, shape_smem_floats(b->jobs[j], (int)b->elem));
  if (g->smem_floats == 0) return FW2V_OK;
  const int det = b->cfg.deterministic;
  cudaError_t e = cudaErrorInvalidValue;
  auto grid = [&](int w, Grid* out) {
    cudaError_t r = cudaErrorInvalidValue;
#define FW2V_GRID(T, F)                                                                                      \
  if (fam == F)                                                                                             \
    r = batch_grid<T, F>(out->smem_floats, w, cap, b->num_sms, b->scratch_warps, det, &out->blocks, &out->threads, \
                         &out->smem);
    if (b->elem == 2) {
      FW2V_GRID(bf16_t, 0) FW2V_GRID(bf16_t, 1) FW2V_GRID(bf16_t, 2)
    } else {
      FW2V_GRID(float, 0) FW2V_GRID(float, 1) FW2V_GRID(float, 2)
    }
#undef FW2V_GRID
    return r;
  };
  if (wpb > 0) {
    e = grid(wpb, g);
  } else {
    // automatic: the most resident warps (blocks x warps), the larger block on
    // a tie; every try sets the kernel's shared-memory limit, so the chosen
    // count is set up again last
    int64_t most = 0;
    int best = 0;
    for (int w : {8, 6, 4, 2}) {
      if (w > batch_max_warps(fam)) continue;
      Grid t = *g;
      if (grid(w, &t) != cudaSuccess) continue;
      if ((int64_t)t.blocks * (t.threads / 32) > most) {
        most = (int64_t)t.blocks * (t.threads / 32);
        best = w;
      }
    }
    if (best > 0) e = grid(best, g);
  }
  if (e != cudaSuccess)
    return bfail(b, FW2V_ERR_ARGUMENT, "batch grid (%d warps per block, %lld floats per warp): %s", wpb,
                 (long long)g->smem_floats, cudaGetErrorString(e));
  return FW2V_OK;
}

BatchTrainArgs train_args(const fw2v_batch* b, const RoundBuf& rb, const BatchRound& r, int epoch, const Grid& g) {
  BatchTrainArgs a{};
  a.jobs = rb.d_tp;
  a.round = r;
  a.entry_prefix = rb.entry_prefix;
  a.uid_base = rb.uid_base;
  a.ent_start = rb.ent_start;
  a.ent_len = rb.ent_len;
  a.ent_alpha = rb.ent_alpha;
  a.work_counter = b->counter;
  a.deterministic = b->cfg.deterministic;
  a.epoch = epoch;
  a.orig_scratch = b->orig_scratch;
  a.scratch_elems = b->scratch_elems;
  a.scratch_warps = b->scratch_warps;
  a.smem_floats = g.smem_floats;
  a.exp_table = b->exp_table;
  return a;
}

cudaError_t launch_train_round(const fw2v_batch* b, int fam, const BatchTrainArgs& a, const Grid& g,
                               cudaStream_t st) {
  if (b->elem == 2) {
    if (fam == 0) return batch_launch<bf16_t, 0>(a, g.blocks, g.threads, g.smem, st);
    if (fam == 1) return batch_launch<bf16_t, 1>(a, g.blocks, g.threads, g.smem, st);
    return batch_launch<bf16_t, 2>(a, g.blocks, g.threads, g.smem, st);
  }
  if (fam == 0) return batch_launch<float, 0>(a, g.blocks, g.threads, g.smem, st);
  if (fam == 1) return batch_launch<float, 1>(a, g.blocks, g.threads, g.smem, st);
  return batch_launch<float, 2>(a, g.blocks, g.threads, g.smem, st);
}

// Sample one round into buffer set rb on the sampler stream.
cudaError_t enqueue_sample(fw2v_batch* b, RoundBuf& rb, const BatchRound& r, int64_t max_region, int epoch) {
  return launch_sampler_round(rb.d_sp, r, epoch, max_region, b->negative > 0, rb.n_entries, rb.n_kept, rb.words,
                              (int)b->jobs.size(), b->job_uid, rb.uid_base, b->job_words, b->job_kept,
                              rb.entry_prefix, b->sst);
}

// Every round of epochs [e0, e0 + epochs): sampler stream and training stream
// joined by events, ending with the sampler stream joined into the training
// stream.  Jobs past their own epoch count sample nothing in an epoch.
cudaError_t enqueue_epochs(fw2v_batch* b, int e0, int epochs, const Grid* grids, bool graph) {
  cudaError_t e = cudaEventRecord(b->ev_fork, b->st);
  const unsigned ev_flags = graph ? cudaEventRecordExternal : cudaEventRecordDefault;
  if (e == cudaSuccess) e = cudaStreamWaitEvent(b->sst, b->ev_fork, 0);
  int64_t k = 0;
  for (int ep = e0; ep < e0 + epochs && e == cudaSuccess; ep++) {
    e = cudaMemsetAsync(b->job_uid, 0, b->jobs.size() * sizeof(int64_t), b->sst);
    for (size_t ri = 0; ri < b->rounds.size() && e == cudaSuccess; ri++, k++) {
      RoundBuf& rb = b->buf[(b->next_buf + k) % 2];
      const RoundPlan& r = b->rounds[ri];
      if (k >= 2 && e == cudaSuccess) e = cudaStreamWaitEvent(b->sst, rb.freed, 0);
      if (e == cudaSuccess) e = enqueue_sample(b, rb, r.view, r.max_region, ep);
      if (e == cudaSuccess) e = cudaEventRecord(rb.ready, b->sst);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, rb.ready, 0);
      if (e == cudaSuccess) e = cudaMemsetAsync(b->counter, 0, sizeof(unsigned long long), b->st);
      const Grid& g = grids[r.family];
      if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->round_ev[2 * k], b->st, ev_flags);
      if (e == cudaSuccess) e = launch_train_round(b, r.family, train_args(b, rb, r.view, ep, g), g, b->st);
      if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->round_ev[2 * k + 1], b->st, ev_flags);
      if (e == cudaSuccess) e = cudaEventRecord(rb.freed, b->st);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecord(b->ev_join, b->sst);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->ev_join, 0);
  return e;
}

fw2v_status check_error_flag(fw2v_batch* b, const char* what) {
  int flag = 0;
  BCK(b, cudaMemcpy(&flag, b->error_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    BCK(b, cudaMemset(b->error_flag, 0, sizeof(int)));
    if (flag == 2) return bfail(b, FW2V_ERR_CUDA, "%s: a bulk row copy did not complete in time", what);
    return bfail(b, FW2V_ERR_BOUNDS, "%s: an id outside [0, V), a read past a token stream or a full buffer", what);
  }
  return FW2V_OK;
}

fw2v_status copy_table(fw2v_batch* b, int32_t job, bool out_table, float* out, int64_t ld) {
  if (!b || job < 0 || job >= (int32_t)b->jobs.size() || !out) return bfail(b, FW2V_ERR_ARGUMENT, "bad job or buffer");
  const BatchJob& j = b->jobs[job];
  const int d = j.cfg.layer_size;
  if (ld < d) return bfail(b, FW2V_ERR_ARGUMENT, "ld < layer_size");
  BCK(b, cudaSetDevice(b->cfg.device));
  BCK(b, cudaStreamSynchronize(b->st));
  const void* src = out_table ? j.syn1neg : j.syn0;
  std::vector<char> host((size_t)j.V * j.pitch * b->elem);
  BCK(b, cudaMemcpy(host.data(), src, host.size(), cudaMemcpyDeviceToHost));
  for (int64_t r = 0; r < j.V; r++)
    for (int c = 0; c < d; c++) {
      const size_t i = (size_t)r * j.pitch + c;
      out[r * ld + c] = b->elem == 2 ? bf16_value(((const uint16_t*)host.data())[i]) : ((const float*)host.data())[i];
    }
  return FW2V_OK;
}

}  // namespace

extern "C" {

void fw2v_batch_config_default(fw2v_batch_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->precision = FW2V_FP32;
  c->use_graph = 1;
}

const char* fw2v_batch_last_error(fw2v_batch* b) { return b ? b->err.c_str() : ""; }

fw2v_status fw2v_batch_create(const fw2v_batch_config* cfg, fw2v_batch** out) {
  if (!cfg || !out) return FW2V_ERR_ARGUMENT;
  *out = nullptr;
  if ((cfg->precision != FW2V_FP32 && cfg->precision != FW2V_BF16) || cfg->round_tokens < 0)
    return FW2V_ERR_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || cfg->device < 0 || cfg->device >= n) return FW2V_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10) return FW2V_ERR_NO_DEVICE;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return FW2V_ERR_NO_DEVICE;
  fw2v_batch* b = new fw2v_batch();
  b->cfg = *cfg;
  b->elem = cfg->precision == FW2V_BF16 ? 2 : 4;
  b->num_sms = prop.multiProcessorCount;
  b->l2_bytes = prop.l2CacheSize;
  auto bad = [&](fw2v_status s) {
    fw2v_batch_destroy(b);
    return s;
  };
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->sst, cudaStreamNonBlocking) != cudaSuccess)
    return bad(FW2V_ERR_CUDA);
  for (cudaEvent_t* e : {&b->ev_start, &b->ev_end})
    if (cudaEventCreate(e) != cudaSuccess) return bad(FW2V_ERR_CUDA);
  for (cudaEvent_t* e : {&b->ev_fork, &b->ev_join})
    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return bad(FW2V_ERR_CUDA);
  for (RoundBuf& rb : b->buf)
    for (cudaEvent_t* e : {&rb.ready, &rb.freed})
      if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return bad(FW2V_ERR_CUDA);
  if (balloc(b->error_flag, 1) != cudaSuccess || balloc(b->counter, 1) != cudaSuccess ||
      balloc(b->exp_table, kExpTableSize) != cudaSuccess)
    return bad(FW2V_ERR_NOMEM);
  float table[kExpTableSize];
  fw2v_exp_table(table);
  if (cudaMemcpy(b->exp_table, table, sizeof(table), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(b->error_flag, 0, sizeof(int)) != cudaSuccess)
    return bad(FW2V_ERR_CUDA);
  *out = b;
  return FW2V_OK;
}

void fw2v_batch_destroy(fw2v_batch* b) {
  if (!b) return;
  cudaSetDevice(b->cfg.device);
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->sst) cudaStreamSynchronize(b->sst);
  free_plan(b);
  for (BatchJob& j : b->jobs) {
    bfree(j.syn0); bfree(j.syn1neg); bfree(j.keep_thr); bfree(j.firsts); bfree(j.stream); bfree(j.chunk_off);
  }
  bfree(b->jump_a); bfree(b->jump_c); bfree(b->exp_table); bfree(b->error_flag); bfree(b->counter);
  bfree(b->lcg); bfree(b->wca); bfree(b->alpha);
  bfree(b->job_uid); bfree(b->job_words); bfree(b->job_kept); bfree(b->orig_scratch);
  for (RoundBuf& rb : b->buf)
    for (cudaEvent_t e : {rb.ready, rb.freed})
      if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {b->ev_start, b->ev_end, b->ev_fork, b->ev_join})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : b->round_ev) cudaEventDestroy(e);
  if (b->st) cudaStreamDestroy(b->st);
  if (b->sst) cudaStreamDestroy(b->sst);
  delete b;
}

static fw2v_status add_job(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts, int64_t V,
                           uint64_t train_words, const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                           int64_t n_chunks, int32_t* job_out, bool on_device);

fw2v_status fw2v_batch_add_job(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts, int64_t V,
                               uint64_t train_words, const int32_t* stream, int64_t stream_len,
                               const int64_t* chunk_off, int64_t n_chunks, int32_t* job_out) {
  return add_job(b, cfg, counts, V, train_words, stream, stream_len, chunk_off, n_chunks, job_out, false);
}

fw2v_status fw2v_batch_add_job_device(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts, int64_t V,
                                      uint64_t train_words, const int32_t* stream, int64_t stream_len,
                                      const int64_t* chunk_off, int64_t n_chunks, int32_t* job_out) {
  return add_job(b, cfg, counts, V, train_words, stream, stream_len, chunk_off, n_chunks, job_out, true);
}

// A job from host memory (on_device false: the corpus checked here, copied
// host to device) or device memory (checked by a kernel, copied on the device).
static fw2v_status add_job(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts, int64_t V,
                           uint64_t train_words, const int32_t* stream, int64_t stream_len, const int64_t* chunk_off,
                           int64_t n_chunks, int32_t* job_out, bool on_device) {
  if (!b || !cfg || !counts || !stream || !chunk_off) return bfail(b, FW2V_ERR_ARGUMENT, "null argument");
  const fw2v_config& c = *cfg;
  if (c.layer_size < 1 || c.layer_size > 384 || c.window < 1 || c.window > kMaxWindow || c.negative < 0 ||
      c.negative > kMaxNegative || c.epochs < 0 || c.threads < 1 || c.msl < 1 || !(c.alpha > 0) ||
      !(c.sample >= 0) || c.sigmoid != FW2V_SIGMOID_TABLE)
    return bfail(b, FW2V_ERR_ARGUMENT,
                 "batch job: layer_size 1..384, window 1..15, negative 0..31, table sigmoid required");
  if (b->negative >= 0 && c.negative != b->negative)
    return bfail(b, FW2V_ERR_ARGUMENT, "batch job: negative %d differs from the batch's %d", c.negative, b->negative);
  if (V < 2 || V > (int64_t)INT32_MAX) return bfail(b, FW2V_ERR_ARGUMENT, "batch job: V >= 2 required");
  if (stream_len < 1 || (!on_device && stream[stream_len - 1] != 0) || n_chunks < 1 || c.threads > n_chunks ||
      c.threads > 65535)
    return bfail(b, FW2V_ERR_ARGUMENT, "batch job: stream must end with 0, threads <= chunks");
  if (!on_device)
    for (int64_t i = 0; i < n_chunks; i++)
      if (chunk_off[i] < 0 || chunk_off[i] >= stream_len)
        return bfail(b, FW2V_ERR_ARGUMENT, "batch job: chunk %lld starts outside the stream", (long long)i);
  BCK(b, cudaSetDevice(b->cfg.device));
  if (on_device) {
    BCK(b, launch_check_corpus(stream, stream_len, chunk_off, n_chunks, b->error_flag, b->st));
    int flag = 0;
    BCK(b, cudaMemcpyAsync(&flag, b->error_flag, sizeof(int), cudaMemcpyDeviceToHost, b->st));
    BCK(b, cudaStreamSynchronize(b->st));
    if (flag) {
      BCK(b, cudaMemsetAsync(b->error_flag, 0, sizeof(int), b->st));
      return bfail(b, FW2V_ERR_ARGUMENT, "batch job: the stream must end with 0 and every chunk start in it");
    }
  }
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  BCK(b, cudaStreamSynchronize(b->st));
  BCK(b, cudaStreamSynchronize(b->sst));
  BatchJob j;
  j.cfg = c;
  j.cfg.precision = b->cfg.precision;
  j.cfg.deterministic = b->cfg.deterministic;
  j.V = V;
  j.train_words = train_words;
  j.pitch = ((int64_t)c.layer_size + 7) / 8 * 8;
  j.soff = seed_offset(c.seed);
  j.lane_vec = j.pitch <= 64 ? 2 : 4;
  j.lane_nv = j.pitch <= 128 ? 1 : (j.pitch <= 256 ? 2 : 3);
  j.stages = default_stages(c.negative, j.lane_nv);
  j.stream_len = stream_len;
  j.n_chunks = n_chunks;
  auto undo = [&](fw2v_status s) {
    bfree(j.syn0); bfree(j.syn1neg); bfree(j.keep_thr); bfree(j.firsts); bfree(j.stream); bfree(j.chunk_off);
    return s;
  };
  const size_t tbytes = (size_t)V * j.pitch * b->elem;
  uint32_t* d_counts = nullptr;
  int64_t* chunk_base = nullptr;
  int64_t* sbase = nullptr;
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  step(cudaMalloc(&j.syn0, tbytes));
  step(cudaMalloc(&j.syn1neg, tbytes));
  step(balloc(j.keep_thr, V));
  step(balloc(j.firsts, V - 1));
  step(balloc(j.stream, stream_len));
  step(balloc(j.chunk_off, n_chunks));
  step(balloc(d_counts, V));
  step(balloc(chunk_base, n_chunks + 1));
  step(balloc(sbase, c.threads + 1));
  std::vector<int64_t> firsts((size_t)V - 1);
  fw2v_unigram_firsts(counts, V, kUnigramTableSize, firsts.data());
  step(cudaMemsetAsync(j.syn0, 0, tbytes, b->st));
  step(cudaMemsetAsync(j.syn1neg, 0, tbytes, b->st));
  step(cudaMemcpyAsync(d_counts, counts, V * sizeof(uint32_t), cudaMemcpyHostToDevice, b->st));
  step(cudaMemcpyAsync(j.firsts, firsts.data(), (V - 1) * sizeof(int64_t), cudaMemcpyHostToDevice, b->st));
  step(cudaMemcpyAsync(j.stream, stream, stream_len * sizeof(int32_t), kind, b->st));
  step(cudaMemcpyAsync(j.chunk_off, chunk_off, n_chunks * sizeof(int64_t), kind, b->st));
  if (e == cudaSuccess)
    step(launch_init_tables(j.syn0, b->elem == 2, V, c.layer_size, j.pitch, d_counts, c.sample, train_words,
                            j.keep_thr, nullptr, 0, nullptr, kUnigramTableSize, 1ULL + j.soff, b->st));
  if (e == cudaSuccess) step(launch_validate_ids(j.stream, stream_len, V, b->error_flag, b->st));
  if (e == cudaSuccess)
    step(launch_corpus_layout(j.stream, stream_len, j.chunk_off, n_chunks, c.msl, c.threads, chunk_base, sbase, b->st));
  j.sbase.assign(c.threads + 1, 0);
  if (e == cudaSuccess)
    step(cudaMemcpyAsync(j.sbase.data(), sbase, (c.threads + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, b->st));
  step(cudaStreamSynchronize(b->st));
  bfree(d_counts);
  bfree(chunk_base);
  bfree(sbase);
  if (e != cudaSuccess)
    return undo(bfail(b, e == cudaErrorMemoryAllocation ? FW2V_ERR_NOMEM : FW2V_ERR_CUDA, "batch job set-up: %s",
                      cudaGetErrorString(e)));
  fw2v_status s = check_error_flag(b, "batch job corpus");
  if (s != FW2V_OK) return undo(s);
  // global stream state, per-job counters and the jump table (first job sets K)
  j.gfirst = b->n_gstreams;
  const int64_t ng = b->n_gstreams + c.threads;
  if (ng > b->gstream_cap) {
    const int64_t cap = std::max<int64_t>(ng, b->gstream_cap * 2);
    if (grow(b->lcg, b->n_gstreams, cap) != cudaSuccess || grow(b->wca, b->n_gstreams, cap) != cudaSuccess ||
        grow(b->alpha, b->n_gstreams, cap) != cudaSuccess)
      return undo(bfail(b, FW2V_ERR_NOMEM, "batch stream state"));
    b->gstream_cap = cap;
  }
  std::vector<uint64_t> lcg(c.threads), zero(c.threads, 0);
  std::vector<float> alpha(c.threads, c.alpha);
  for (int i = 0; i < c.threads; i++) lcg[i] = (uint64_t)i + j.soff;
  if (cudaMemcpy(b->lcg + j.gfirst, lcg.data(), c.threads * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->wca + j.gfirst, zero.data(), c.threads * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->alpha + j.gfirst, alpha.data(), c.threads * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return undo(bfail(b, FW2V_ERR_CUDA, "batch stream state upload"));
  const int64_t J = (int64_t)b->jobs.size() + 1;
  if (J > b->job_cap) {
    const int64_t cap = std::max<int64_t>(J, b->job_cap * 2);
    const int64_t old = (int64_t)b->jobs.size();
    if (grow(b->job_uid, 0, cap) != cudaSuccess || grow(b->job_words, old, cap) != cudaSuccess ||
        grow(b->job_kept, old, cap) != cudaSuccess)
      return undo(bfail(b, FW2V_ERR_NOMEM, "batch job counters"));
    b->job_cap = cap;
  }
  if (cudaMemset(b->job_words + b->jobs.size(), 0, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(b->job_kept + b->jobs.size(), 0, sizeof(unsigned long long)) != cudaSuccess)
    return undo(bfail(b, FW2V_ERR_CUDA, "batch job counters"));
  if (b->negative < 0) {
    b->negative = c.negative;
    const int n_jump = 32 * (1 + c.negative) + 1;
    std::vector<uint64_t> ja(n_jump), jc(n_jump);
    for (int m = 0; m < n_jump; m++) {
      const Affine a = lcg_jump((uint64_t)m);
      ja[m] = a.a;
      jc[m] = a.c;
    }
    if (balloc(b->jump_a, n_jump) != cudaSuccess || balloc(b->jump_c, n_jump) != cudaSuccess ||
        cudaMemcpy(b->jump_a, ja.data(), n_jump * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->jump_c, jc.data(), n_jump * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      return undo(bfail(b, FW2V_ERR_NOMEM, "batch jump table"));
  }
  b->n_gstreams = ng;
  b->jobs.push_back(std::move(j));
  b->words_total.push_back(0);
  b->kept_total.push_back(0);
  b->words_snap.push_back(0);
  b->kept_snap.push_back(0);
  b->planned = false;
  if (job_out) *job_out = (int32_t)b->jobs.size() - 1;
  return FW2V_OK;
}

fw2v_status fw2v_batch_set_shape(fw2v_batch* b, int32_t job, int32_t lane_vec, int32_t lane_nv, int32_t stages,
                                 int32_t prefetch) {
  if (!b || job < 0 || job >= (int32_t)b->jobs.size()) return bfail(b, FW2V_ERR_ARGUMENT, "bad job");
  BatchJob& j = b->jobs[job];
  if (!valid_shape(j.cfg.layer_size, lane_vec, lane_nv, stages))
    return bfail(b, FW2V_ERR_ARGUMENT, "shape (%d x %d, %d stages) cannot train d = %d", lane_vec, lane_nv, stages,
                 j.cfg.layer_size);
  if (batch_family(lane_nv, stages) != j.family()) b->planned = false;  // the job moves to another family
  j.lane_vec = lane_vec;
  j.lane_nv = lane_nv;
  j.stages = stages;
  if (prefetch < 0 || prefetch > 3) return bfail(b, FW2V_ERR_ARGUMENT, "prefetch bits are 0..3");
  j.prefetch = prefetch;
  return FW2V_OK;
}

fw2v_status fw2v_batch_get_shape(fw2v_batch* b, int32_t job, int32_t* lane_vec, int32_t* lane_nv, int32_t* stages,
                                 int32_t* prefetch) {
  if (!b || job < 0 || job >= (int32_t)b->jobs.size() || !lane_vec || !lane_nv || !stages || !prefetch)
    return bfail(b, FW2V_ERR_ARGUMENT, "bad job");
  *lane_vec = b->jobs[job].lane_vec;
  *lane_nv = b->jobs[job].lane_nv;
  *stages = b->jobs[job].stages;
  *prefetch = b->jobs[job].prefetch;
  return FW2V_OK;
}

fw2v_status fw2v_batch_set_launch(fw2v_batch* b, int32_t family, int32_t warps_per_block, int32_t blocks_per_sm) {
  if (!b || family < 0 || family >= kBatchFamilies || warps_per_block < 0 ||
      warps_per_block > batch_max_warps(family) || blocks_per_sm < 0)
    return bfail(b, FW2V_ERR_ARGUMENT,
                 "family 0..2, warps per block 0 (automatic) or 1..8, 1..6, 1..4 (families 0, 1, 2), blocks per SM >= 0");
  b->warps_per_block[family] = warps_per_block;
  b->blocks_per_sm[family] = blocks_per_sm;
  return FW2V_OK;
}

fw2v_status fw2v_batch_get_launch(fw2v_batch* b, int32_t family, int32_t* warps_per_block, int32_t* blocks_per_sm) {
  if (!b || family < 0 || family >= kBatchFamilies || !warps_per_block || !blocks_per_sm) return FW2V_ERR_ARGUMENT;
  *warps_per_block = b->warps_per_block[family];
  *blocks_per_sm = b->blocks_per_sm[family];
  return FW2V_OK;
}

fw2v_status fw2v_batch_train_epochs(fw2v_batch* b, int32_t n_epochs, fw2v_batch_stats* stats) {
  if (!b || n_epochs < 0) return bfail(b, FW2V_ERR_ARGUMENT, "epochs >= 0");
  BCK(b, cudaSetDevice(b->cfg.device));
  fw2v_status s = plan(b);
  if (s != FW2V_OK) return s;
  s = upload_params(b);
  if (s != FW2V_OK) return s;
  std::vector<int> all(b->jobs.size());
  for (size_t i = 0; i < all.size(); i++) all[i] = (int)i;
  Grid g[kBatchFamilies];
  for (int fam = 0; fam < kBatchFamilies; fam++) {
    s = grid_for(b, all, fam, b->warps_per_block[fam], b->blocks_per_sm[fam], &g[fam]);
    if (s != FW2V_OK) return s;
  }
  int max_epochs = 0;
  for (const BatchJob& j : b->jobs) max_epochs = std::max(max_epochs, j.cfg.epochs);
  const int e0 = b->epochs_run;
  const int epochs = std::min(n_epochs, std::max(0, max_epochs - e0));
  if (epochs == 0) {
    if (stats) *stats = fw2v_batch_stats{};
    return FW2V_OK;
  }
  const size_t J = b->jobs.size();
  const size_t launches = (size_t)epochs * b->rounds.size();
  while (b->round_ev.size() < 2 * launches) {
    cudaEvent_t ev;
    BCK(b, cudaEventCreate(&ev));
    b->round_ev.push_back(ev);
  }
  BCK(b, cudaStreamSynchronize(b->st));
  BCK(b, cudaEventRecord(b->ev_start, b->st));
  if (b->cfg.use_graph) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    BCK(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    const cudaError_t e = enqueue_epochs(b, e0, epochs, g, true);
    const cudaError_t e2 = cudaStreamEndCapture(b->st, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();  // the failed capture's error is reported here, not by a later call
    }
    BCK(b, e);
    BCK(b, e2);
    cudaError_t e3 = cudaGraphInstantiate(&exec, graph, 0);
    if (e3 == cudaSuccess) e3 = cudaGraphLaunch(exec, b->st);
    if (e3 == cudaSuccess) e3 = cudaEventRecord(b->ev_end, b->st);
    if (e3 == cudaSuccess) e3 = cudaStreamSynchronize(b->st);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    BCK(b, e3);
  } else {
    BCK(b, enqueue_epochs(b, e0, epochs, g, false));
    BCK(b, cudaEventRecord(b->ev_end, b->st));
    BCK(b, cudaStreamSynchronize(b->st));
  }
  b->next_buf = (int)((b->next_buf + (int64_t)epochs * (int64_t)b->rounds.size()) % 2);
  s = check_error_flag(b, "batch train");
  if (s != FW2V_OK) return s;
  // the job counters are cumulative: this call's words are the change
  std::vector<unsigned long long> w(J), k(J);
  BCK(b, cudaMemcpy(w.data(), b->job_words, J * 8, cudaMemcpyDeviceToHost));
  BCK(b, cudaMemcpy(k.data(), b->job_kept, J * 8, cudaMemcpyDeviceToHost));
  fw2v_batch_stats out{};
  for (size_t i = 0; i < J; i++) {
    out.words_read += w[i] - b->words_snap[i];
    out.words_kept += k[i] - b->kept_snap[i];
    b->words_total[i] = w[i];
    b->kept_total[i] = k[i];
  }
  b->words_snap = w;
  b->kept_snap = k;
  b->epochs_run += epochs;
  BCK(b, cudaEventElapsedTime(&out.ms, b->ev_start, b->ev_end));
  for (size_t i = 0; i < launches; i++) {
    float t = 0;
    if (cudaEventElapsedTime(&t, b->round_ev[2 * i], b->round_ev[2 * i + 1]) != cudaSuccess) {
      cudaGetLastError();
      out.train_ms = -1.0f;  // not timed
      break;
    }
    out.train_ms += t;
  }
  out.train_launches = (int32_t)launches;
  out.epochs = epochs;
  out.rounds = (int32_t)b->rounds.size();
  if (stats) *stats = out;
  return FW2V_OK;
}

fw2v_status fw2v_batch_train(fw2v_batch* b, fw2v_batch_stats* stats) {
  return fw2v_batch_train_epochs(b, INT32_MAX, stats);
}

}  // extern "C"

// ---- autotuner ----
namespace {

// A round of the first epoch's training order restricted to `jobs`, up to
// `tokens` readable tokens (at least one stream), within the buffer capacity.
fw2v_status tuning_round(fw2v_batch* b, const std::vector<int>& jobs, int64_t tokens, RoundPlan* r) {
  std::vector<char> in(b->jobs.size(), 0);
  for (int j : jobs) in[j] = 1;
  std::vector<int32_t> job, local;
  std::vector<int64_t> gs, kb(1, 0);
  for (const StreamItem& it : stream_order(b, in)) {
    if (!job.empty() && (kb.back() + it.tokens > std::min(tokens, b->buf_kept_cap) ||
                         (int64_t)job.size() >= b->buf_stream_cap))
      continue;
    job.push_back(it.job);
    local.push_back(it.local);
    gs.push_back(it.gstream);
    kb.push_back(kb.back() + it.tokens);
    r->max_region = std::max(r->max_region, it.tokens);
  }
  r->n = (int)job.size();
  r->kept = kb.back();
  if (r->n == 0 || r->kept > b->buf_kept_cap) return bfail(b, FW2V_ERR_STATE, "tuning sample does not fit");
  BCK(b, cudaMalloc(&r->dev, (size_t)r->n * 32 + 8));
  int64_t* d_gs = (int64_t*)r->dev;
  int64_t* d_kb = d_gs + r->n;
  int32_t* d_job = (int32_t*)(d_kb + r->n + 1);
  int32_t* d_local = d_job + r->n;
  BCK(b, cudaMemcpy(d_gs, gs.data(), r->n * 8, cudaMemcpyHostToDevice));
  BCK(b, cudaMemcpy(d_kb, kb.data(), (r->n + 1) * 8, cudaMemcpyHostToDevice));
  BCK(b, cudaMemcpy(d_job, job.data(), r->n * 4, cudaMemcpyHostToDevice));
  BCK(b, cudaMemcpy(d_local, local.data(), r->n * 4, cudaMemcpyHostToDevice));
  r->view = BatchRound{d_job, d_local, d_gs, d_kb, r->n};
  return FW2V_OK;
}

// Train the round sampled in buf[0] (jobs of kernel family `fam`) `reps`
// times after one warm-up; the fastest time in ms.
fw2v_status time_round(fw2v_batch* b, const RoundPlan& r, const std::vector<int>& active, int fam, int wpb, int cap,
                       int reps, float* best_ms) {
  fw2v_status s = upload_params(b);
  if (s != FW2V_OK) return s;
  Grid g;
  s = grid_for(b, active, fam, wpb, cap, &g);
  if (s != FW2V_OK) return s;
  *best_ms = 1e30f;
  for (int i = 0; i <= reps; i++) {
    BCK(b, cudaMemsetAsync(b->counter, 0, sizeof(unsigned long long), b->st));
    BCK(b, cudaEventRecord(b->ev_start, b->st));
    BCK(b, launch_train_round(b, fam, train_args(b, b->buf[0], r.view, 0, g), g, b->st));
    BCK(b, cudaEventRecord(b->ev_end, b->st));
    BCK(b, cudaStreamSynchronize(b->st));
    float ms = 0;
    BCK(b, cudaEventElapsedTime(&ms, b->ev_start, b->ev_end));
    if (i > 0) *best_ms = std::min(*best_ms, ms);
  }
  return FW2V_OK;
}

}  // namespace

extern "C" fw2v_status fw2v_batch_tune(fw2v_batch* b, int64_t sample_tokens, fw2v_batch_tune_report* report) {
  if (!b) return FW2V_ERR_ARGUMENT;
  if (b->cfg.deterministic) return bfail(b, FW2V_ERR_STATE, "tuning needs the concurrent mode");
  BCK(b, cudaSetDevice(b->cfg.device));
  fw2v_status s = plan(b);
  if (s != FW2V_OK) return s;
  if (sample_tokens <= 0) sample_tokens = (int64_t)1 << 23;
  const size_t J = b->jobs.size();
  // classes of jobs with the same (layout class of d, window); a class's
  // layouts all belong to one kernel family
  std::vector<std::pair<int, int>> keys;
  std::vector<std::vector<int>> members;
  for (size_t i = 0; i < J; i++) {
    const std::pair<int, int> k{layout_class(b->jobs[i].pitch), b->jobs[i].cfg.window};
    size_t c = std::find(keys.begin(), keys.end(), k) - keys.begin();
    if (c == keys.size()) {
      keys.push_back(k);
      members.emplace_back();
    }
    members[c].push_back((int)i);
  }
  if (keys.size() > 16) return bfail(b, FW2V_ERR_ARGUMENT, "more than 16 job classes to tune");
  // snapshot of everything tuning changes: tables and stream state
  size_t tbytes = 0;
  for (const BatchJob& j : b->jobs) tbytes += 2 * (size_t)j.V * j.pitch * b->elem;
  char* snap = nullptr;
  uint64_t* s_lcg = nullptr;
  uint64_t* s_wca = nullptr;
  float* s_alpha = nullptr;
  BCK(b, cudaStreamSynchronize(b->st));
  BCK(b, cudaMalloc(&snap, tbytes));
  auto restore = [&]() {
    size_t off = 0;
    for (const BatchJob& j : b->jobs) {
      const size_t tb = (size_t)j.V * j.pitch * b->elem;
      cudaMemcpy(j.syn0, snap + off, tb, cudaMemcpyDeviceToDevice);
      cudaMemcpy(j.syn1neg, snap + off + tb, tb, cudaMemcpyDeviceToDevice);
      off += 2 * tb;
    }
    if (s_lcg && s_wca && s_alpha) {
      cudaMemcpy(b->lcg, s_lcg, b->n_gstreams * 8, cudaMemcpyDeviceToDevice);
      cudaMemcpy(b->wca, s_wca, b->n_gstreams * 8, cudaMemcpyDeviceToDevice);
      cudaMemcpy(b->alpha, s_alpha, b->n_gstreams * 4, cudaMemcpyDeviceToDevice);
    }
    const cudaError_t e = cudaDeviceSynchronize();
    bfree(snap);
    bfree(s_lcg);
    bfree(s_wca);
    bfree(s_alpha);
    return e;
  };
  {
    size_t off = 0;
    cudaError_t e = cudaSuccess;
    for (const BatchJob& j : b->jobs) {
      const size_t tb = (size_t)j.V * j.pitch * b->elem;
      if (e == cudaSuccess) e = cudaMemcpy(snap + off, j.syn0, tb, cudaMemcpyDeviceToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(snap + off + tb, j.syn1neg, tb, cudaMemcpyDeviceToDevice);
      off += 2 * tb;
    }
    if (e == cudaSuccess) e = balloc(s_lcg, b->n_gstreams);
    if (e == cudaSuccess) e = balloc(s_wca, b->n_gstreams);
    if (e == cudaSuccess) e = balloc(s_alpha, b->n_gstreams);
    if (e == cudaSuccess) e = cudaMemcpy(s_lcg, b->lcg, b->n_gstreams * 8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s_wca, b->wca, b->n_gstreams * 8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s_alpha, b->alpha, b->n_gstreams * 4, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      bfree(snap);
      bfree(s_lcg);
      bfree(s_wca);
      bfree(s_alpha);
      return bfail(b, FW2V_ERR_NOMEM, "tuning snapshot: %s", cudaGetErrorString(e));
    }
  }

  std::vector<unsigned long long> words0(J), kept0(J);  // tuning samples must not count
  BCK(b, cudaMemcpy(words0.data(), b->job_words, J * 8, cudaMemcpyDeviceToHost));
  BCK(b, cudaMemcpy(kept0.data(), b->job_kept, J * 8, cudaMemcpyDeviceToHost));
  fw2v_batch_tune_report rep{};
  rep.n_classes = (int32_t)keys.size();
  auto sample_into_buf0 = [&](const RoundPlan& r) -> fw2v_status {
    fw2v_status s2 = upload_params(b);
    if (s2 != FW2V_OK) return s2;
    BCK(b, cudaMemsetAsync(b->job_uid, 0, J * sizeof(int64_t), b->sst));
    BCK(b, enqueue_sample(b, b->buf[0], r.view, r.max_region, 0));
    BCK(b, cudaStreamSynchronize(b->sst));
    return check_error_flag(b, "batch tune sampling");
  };
  auto kept_of = [&](const RoundPlan& r, double* kept) -> fw2v_status {
    std::vector<int64_t> nk(r.n);
    BCK(b, cudaMemcpy(nk.data(), b->buf[0].n_kept, r.n * 8, cudaMemcpyDeviceToHost));
    *kept = 0;
    for (int64_t x : nk) *kept += (double)x;
    return FW2V_OK;
  };
  fw2v_status result = FW2V_OK;
  for (size_t c = 0; c < keys.size() && result == FW2V_OK; c++) {
    RoundPlan r;
    result = tuning_round(b, members[c], sample_tokens, &r);
    if (result == FW2V_OK) result = sample_into_buf0(r);
    double kept = 0;
    if (result == FW2V_OK) result = kept_of(r, &kept);
    int d_max = 0;
    for (int j : members[c]) d_max = std::max(d_max, b->jobs[j].cfg.layer_size);
    const BatchJob& j0 = b->jobs[members[c][0]];
    const int def_vec = j0.pitch <= 64 ? 2 : 4, def_nv = j0.pitch <= 128 ? 1 : (j0.pitch <= 256 ? 2 : 3);
    const int def_st = default_stages(b->negative, def_nv);
    double best = -1, def_wps = 0;
    int best_vec = def_vec, best_nv = def_nv, best_st = def_st, best_pre = 0;
    for (int vec : {2, 4}) {
      for (int st : kBatchStages) {
        for (int pre : {0, 1, 2, 3}) {
          if (result != FW2V_OK || !valid_shape(d_max, vec, def_nv, st)) continue;
          for (int j : members[c]) {
            b->jobs[j].lane_vec = vec;
            b->jobs[j].lane_nv = def_nv;
            b->jobs[j].stages = st;
            b->jobs[j].prefetch = pre;
          }
          float ms = 0;
          const int fam = batch_family(def_nv, st);
          result = time_round(b, r, members[c], fam, b->warps_per_block[fam], b->blocks_per_sm[fam], 2, &ms);
          if (result != FW2V_OK) break;
          const double wps = kept / (ms / 1e3);
          if (vec == def_vec && st == def_st && !pre) def_wps = wps;
          if (wps > best) {
            best = wps;
            best_vec = vec;
            best_st = st;
            best_pre = pre;
          }
        }
      }
    }
    for (int j : members[c]) {
      b->jobs[j].lane_vec = best_vec;
      b->jobs[j].lane_nv = best_nv;
      b->jobs[j].stages = best_st;
      b->jobs[j].prefetch = best_pre;
    }
    rep.class_d[c] = d_max;
    rep.class_window[c] = keys[c].second;
    rep.class_lane_vec[c] = best_vec;
    rep.class_lane_nv[c] = best_nv;
    rep.class_stages[c] = best_st;
    rep.class_prefetch[c] = best_pre;
    rep.tuned_wps[c] = best;
    rep.default_wps[c] = def_wps;
    bfree(r.dev);
  }
  // grid of each kernel family: warps per block over all its jobs together
  for (int fam = 0; fam < kBatchFamilies && result == FW2V_OK; fam++) {
    std::vector<int> act;
    for (size_t i = 0; i < J; i++)
      if (b->jobs[i].family() == fam) act.push_back((int)i);
    if (act.empty()) continue;
    int n_cls = 0;
    for (size_t c = 0; c < keys.size(); c++) n_cls += b->jobs[members[c][0]].family() == fam;
    RoundPlan r;
    result = tuning_round(b, act, sample_tokens * (int64_t)std::max(n_cls, 1), &r);
    if (result == FW2V_OK) result = sample_into_buf0(r);
    double best = -1;
    int best_w = b->warps_per_block[fam];
    for (int w : {2, 4, 6, 8}) {
      if (result != FW2V_OK) break;
      if (w > batch_max_warps(fam)) continue;
      Grid g;
      if (grid_for(b, act, fam, w, 0, &g) != FW2V_OK) continue;  // does not fit: skip
      float ms = 0;
      result = time_round(b, r, act, fam, w, 0, 2, &ms);
      if (result == FW2V_OK && 1.0 / ms > best) {
        best = 1.0 / ms;
        best_w = w;
      }
    }
    b->warps_per_block[fam] = best_w;
    b->blocks_per_sm[fam] = 0;
    bfree(r.dev);
  }
  for (int fam = 0; fam < kBatchFamilies; fam++) {
    rep.warps_per_block[fam] = b->warps_per_block[fam];
    rep.blocks_per_sm[fam] = b->blocks_per_sm[fam];
  }
  b->planned = false;  // shapes may have moved jobs between families
  cudaStreamSynchronize(b->sst);
  cudaMemcpy(b->job_words, words0.data(), J * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(b->job_kept, kept0.data(), J * 8, cudaMemcpyHostToDevice);
  const cudaError_t e = restore();
  if (result != FW2V_OK) return result;
  BCK(b, e);
  if (report) *report = rep;
  return check_error_flag(b, "batch tune");
}

extern "C" {

fw2v_status fw2v_batch_job_words(fw2v_batch* b, int32_t job, uint64_t* words_read, uint64_t* words_kept) {
  if (!b || job < 0 || job >= (int32_t)b->jobs.size()) return bfail(b, FW2V_ERR_ARGUMENT, "bad job");
  if (words_read) *words_read = b->words_total[job];
  if (words_kept) *words_kept = b->kept_total[job];
  return FW2V_OK;
}

fw2v_status fw2v_batch_get_syn0(fw2v_batch* b, int32_t job, float* out, int64_t ld) {
  return copy_table(b, job, false, out, ld);
}

fw2v_status fw2v_batch_get_syn1neg(fw2v_batch* b, int32_t job, float* out, int64_t ld) {
  return copy_table(b, job, true, out, ld);
}

}  // extern "C"
