/*
 * fw2v.h — C ABI of libfw2v.so, the B200 SGNS (skip-gram negative sampling)
 * trainer that replaces the FULL-W2V training path.
 *
 * Plain C types only; every call returns an fw2v_status and never exits the
 * process.  A handle owns all device memory it allocates and must be used from
 * one host thread at a time.  Streams and graphs are internal.
 *
 * What each entry point replaces in the reference (tlranda/FULL-W2V, paths
 * relative to its root):
 *
 *   fw2v_create / fw2v_destroy     global configuration + teardown,
 *                                  src/FULL-W2V/FULL-W2V-driver.cu:42-73, 453-470
 *   fw2v_set_vocab                 InitNet: syn0 LCG init, syn1neg zero, unigram
 *                                  table, subsampling table,
 *                                  src/FULL-W2V/improved_driver_functions.cpp:1-83
 *   fw2v_load_corpus               the global token stream and its sentence
 *                                  table (createGlobalStream / readCorpusCache),
 *                                  improved_driver_functions.cpp:244-281, 320-401
 *   fw2v_sample_epoch              the host batch builder of Train_SGNS (LCG
 *                                  subsampling + negatives + alpha schedule),
 *                                  FULL-W2V-driver.cu:166-302, moved on-device
 *   fw2v_train_sampled             the kernel launches of Train_SGNS,
 *                                  FULL-W2V-driver.cu:284-299, 305-319
 *   fw2v_train_epoch / fw2v_train  one / all epochs of Train_SGNS,
 *                                  FULL-W2V-driver.cu:80-354, 438-446
 *   fw2v_kernel_batch              the `cuda_kernel` function-pointer seam
 *                                  (FULL-W2V-kernels.cu:11-12, bound at :24,
 *                                  called at FULL-W2V-driver.cu:293, 317) with
 *                                  the same arguments: device sentence, negative,
 *                                  length and alpha arrays laid out per block
 *   fw2v_get_syn0 / fw2v_get_syn1neg
 *                                  the device-to-host copy of saveModel,
 *                                  improved_driver_functions.cpp:225-228
 *   fw2v_words_trained             word_count_actual, the numerator of
 *                                  "Overall Words Per Second", FULL-W2V-driver.cu:450-451
 */
#ifndef FW2V_H
#define FW2V_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fw2v_status {
  FW2V_OK = 0,
  FW2V_ERR_ARGUMENT = 1,     /* invalid argument or unsupported size */
  FW2V_ERR_CUDA = 2,         /* a CUDA runtime call failed; see fw2v_last_error */
  FW2V_ERR_NOMEM = 3,        /* device or pinned host allocation failed */
  FW2V_ERR_STATE = 4,        /* call out of order (e.g. train before set_vocab) */
  FW2V_ERR_BOUNDS = 5,       /* a token or negative id outside [0, V) was found */
  FW2V_ERR_NO_DEVICE = 6,    /* no CUDA device or the library was built for another arch */
  FW2V_ERR_TOO_LARGE = 7     /* the request does not fit a fixed-size library buffer */
} fw2v_status;

typedef enum fw2v_sigmoid {
  FW2V_SIGMOID_TABLE = 0,    /* the reference's 1000-entry table (expTable.h) */
  FW2V_SIGMOID_EXACT = 1     /* 1/(1+expf(-x)) */
} fw2v_sigmoid;

typedef enum fw2v_precision {
  FW2V_FP32 = 0,             /* FP32 tables, FP32 math */
  FW2V_BF16 = 1              /* BF16 tables, FP32 math, stochastic-rounded write-back */
} fw2v_precision;

typedef struct fw2v_config {
  int32_t layer_size;        /* -size  d, 1..1024 */
  int32_t window;            /* -window W, 1..15 */
  int32_t negative;          /* -negative K, 0..31 */
  int32_t epochs;            /* -iter E */
  int32_t threads;           /* -threads T: sampling streams, each seeded with its id */
  int32_t msl;               /* -msl: maximum kept words per sentence */
  float alpha;               /* -alpha: starting learning rate */
  float sample;              /* -sample: subsampling threshold (0 disables) */
  int32_t sigmoid;           /* fw2v_sigmoid */
  int32_t precision;         /* fw2v_precision */
  int32_t deterministic;     /* 1: sentences trained one at a time in stream order */
  int32_t device;            /* CUDA device ordinal */
  uint64_t seed;             /* 0: the reference's seeds (syn0 from LCG state 1,
                                stream s from state s); otherwise syn0's start
                                state, every stream's LCG and the stochastic-
                                rounding seeds are offset by fw2v_seed_offset(seed) */
} fw2v_config;

typedef struct fw2v_handle fw2v_handle;

typedef struct fw2v_epoch_stats {
  uint64_t words_read;       /* tokens read this epoch, subsampled-away and EOS included */
  uint64_t words_kept;       /* tokens that survived subsampling in trained sentences */
  uint64_t sentences;        /* batch entries recorded (zero-length ones included) */
  float sampler_ms;          /* device time of the sampling kernel */
  float train_ms;            /* device time of the training kernel */
} fw2v_epoch_stats;

/* Fill *cfg with the reference defaults (FULL-W2V-driver.cu:49-55,
 * improved_driver_functions.cpp:475-501). */
void fw2v_config_default(fw2v_config* cfg);

fw2v_status fw2v_create(const fw2v_config* cfg, fw2v_handle** out);
void fw2v_destroy(fw2v_handle* h);

/* Vocabulary in reference order (index 0 = "</s>", then descending count).
 * train_words is the reference's train_words (sum of kept counts, +1 when
 * learned from a text file).  Allocates and initialises the embedding tables. */
fw2v_status fw2v_set_vocab(fw2v_handle* h, const uint32_t* counts, int64_t vocab_size,
                           uint64_t train_words);

/* Token stream (host memory; ids in [0, V), the trailing 0 included) and the
 * start offset of each stored sentence chunk, in the order the streams read
 * them (any order; a chunk is read from its offset up to msl tokens or up to
 * and including its first 0).  Requires threads <= n_chunks.  Resets the
 * streams' LCG and learning-rate state and the epoch count. */
fw2v_status fw2v_load_corpus(fw2v_handle* h, const int32_t* stream, int64_t stream_len,
                             const int64_t* chunk_off, int64_t n_chunks);
/* The same from device memory (both arrays device pointers, e.g. a corpus
 * generated on the GPU): checked by a kernel (trailing 0, chunk offsets inside
 * the stream, ids in [0, V)) and copied on the device; no host round trip.
 * The replacement of createGlobalStream's host array for corpora that already
 * live on the GPU (improved_driver_functions.cpp:244-281). */
fw2v_status fw2v_load_corpus_device(fw2v_handle* h, const int32_t* stream, int64_t stream_len,
                                    const int64_t* chunk_off, int64_t n_chunks);

/* Replace the order of the stored chunks without touching the streams' LCG and
 * learning-rate state: the reference's -epoch-shuffle, which permutes its
 * sentence pointers between epochs (FULL-W2V-driver.cu:249-266,
 * improved_driver_functions.cpp:283-291).  Same chunk count; call between
 * epochs (no sampled epoch waiting to be trained). */
fw2v_status fw2v_reorder_chunks(fw2v_handle* h, const int64_t* chunk_off, int64_t n_chunks);

/* A seeded shuffle of the stored chunks on the device, in place of the
 * reference's libc rand() shuffle (shuffleSentences,
 * improved_driver_functions.cpp:283-291; -pre-shuffle / -epoch-shuffle,
 * FULL-W2V-driver.cu:249-266, 423): Fisher-Yates from the last chunk down,
 * chunk i swapped with j = high 64 bits of mix64(key ^ mix64(i)) * (i + 1)
 * (mix64: the SplitMix64 finaliser).  The same key gives the same order on any
 * device; fw2v_get_chunks reads the order back (n_chunks offsets).  Same
 * calling rules as fw2v_reorder_chunks. */
fw2v_status fw2v_shuffle_chunks(fw2v_handle* h, uint64_t key);
fw2v_status fw2v_get_chunks(fw2v_handle* h, int64_t* chunk_off);

/* Run the on-device batch builder for the next epoch only. */
fw2v_status fw2v_sample_epoch(fw2v_handle* h);
/* Sizes of the last sampled epoch: entries and kept ids summed over streams. */
fw2v_status fw2v_epoch_sample_sizes(fw2v_handle* h, int64_t* n_entries, int64_t* n_kept);
/* Copy the last sampled epoch to host memory, streams in order.  Per stream s:
 * entries_per_stream[s] entries (lens, alphas) and kept_per_stream[s] kept ids
 * (ids) with `negative` negatives each (negs); words_per_stream[s] tokens read.
 * Any output pointer may be NULL. */
fw2v_status fw2v_epoch_samples(fw2v_handle* h, int32_t* lens, float* alphas, int32_t* ids,
                               int32_t* negs, int64_t* entries_per_stream,
                               int64_t* kept_per_stream, uint64_t* words_per_stream);
/* Train the sentences of the last sampled epoch. */
fw2v_status fw2v_train_sampled(fw2v_handle* h, fw2v_epoch_stats* stats);

/* Sample + train one epoch; stats may be NULL. */
fw2v_status fw2v_train_epoch(fw2v_handle* h, fw2v_epoch_stats* stats);
/* Run the remaining epochs of the configured E. */
fw2v_status fw2v_train(fw2v_handle* h, uint64_t* words_read);

/* Total tokens read over all epochs trained so far. */
fw2v_status fw2v_words_trained(fw2v_handle* h, uint64_t* words);

/* Copy tables to/from host memory, rows of layer_size floats spaced by
 * row_stride floats (row_stride >= layer_size). */
fw2v_status fw2v_get_syn0(fw2v_handle* h, float* out, int64_t row_stride);
fw2v_status fw2v_get_syn1neg(fw2v_handle* h, float* out, int64_t row_stride);
fw2v_status fw2v_set_tables(fw2v_handle* h, const float* syn0, const float* syn1neg,
                            int64_t row_stride);

/* Train explicit sentences from host memory (deterministic order when the
 * handle is deterministic): sentence s has lens[s] ids starting at
 * ids[starts[s]] and negatives at negs[starts[s] * K]. */
fw2v_status fw2v_train_sentences(fw2v_handle* h, const int32_t* ids, const int32_t* negs,
                                 const int64_t* starts, const int32_t* lens, const float* alphas,
                                 int64_t n_sentences);

/* Held-out SGNS loss summed in FP64 on the device over every (context, centre)
 * pair of the given sentences: -log s(<v_c,o_w>) - sum_k log s(-<v_c,o_nk>). */
fw2v_status fw2v_heldout_loss(fw2v_handle* h, const int32_t* ids, const int32_t* negs,
                              const int64_t* starts, const int32_t* lens, int64_t n_sentences,
                              double* loss_sum, int64_t* pairs);

/* The reference kernel seam: FP32 tables with `pitch` floats per row, block b
 * trains sen[b*msl .. +len[b]] with negatives neg[b*msl*K ...] at alpha[b].
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL: default).
 * The launch is asynchronous; errors found by the kernel (ids outside
 * [0, vocab_size)) are reported by the next call on the same handle-less seam
 * through fw2v_kernel_batch_error. */
fw2v_status fw2v_kernel_batch(float* syn0, float* syn1neg, const int32_t* sen, const int32_t* neg,
                              const int32_t* len, const float* alpha, int32_t n_blocks,
                              int32_t layer_size, int32_t window, int32_t negative, int32_t msl,
                              uint32_t pitch, int64_t vocab_size, void* stream);
/* fw2v_kernel_batch without any device allocation.  No counterpart in the
 * reference: FULL-W2V allocates all of its buffers up front in its driver.
 *
 * For callers that cannot allocate device memory: a host program whose device
 * memory is owned entirely by a framework's pooling allocator (a direct
 * cudaMalloc would bypass the pool's accounting and can fail once the pool
 * holds the device), a plugin host that hands the library its buffers under a
 * fixed memory budget, and latency-bound loops in which cudaMalloc/cudaFree
 * would stall or synchronise the device.  Arguments and results are those of
 * fw2v_kernel_batch.  The per-warp scratch the kernel needs (each context row's
 * value when it entered the window) lives in a fixed array of
 * FW2V_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the
 * library keeps until the process exits; (2*window+1) * pitch * 4 bytes per warp
 * of up to FW2V_NOALLOC_SCRATCH_BYTES in total cap the number of warps working
 * concurrently.  A request needing more than that for one block of 4 warps is
 * rejected with FW2V_ERR_TOO_LARGE, and one whose per-warp shared memory (the
 * ring of 2*window+1 rows and the staged target rows, about
 * (2*window + 12) * pitch * 4 bytes) does not fit a block with
 * FW2V_ERR_ARGUMENT, both before anything runs.
 *
 * The first call on a device looks up the array's device address and loads the
 * sigmoid table; make that first call before any stream capture.  All calls
 * share the one array and nothing in it needs to start at zero (every row is
 * written when it enters the window, before it is read), so its contents from
 * an earlier call are harmless; but calls that overlap on the GPU (other
 * streams, or another thread) race on it and must be serialised by the caller.
 * Out-of-range ids are reported by fw2v_kernel_batch_error, like the seam's. */
#define FW2V_NOALLOC_SCRATCH_BYTES (16u << 20)
fw2v_status fw2v_kernel_batch_noalloc(float* syn0, float* syn1neg, const int32_t* sen,
                                      const int32_t* neg, const int32_t* len, const float* alpha,
                                      int32_t n_blocks, int32_t layer_size, int32_t window,
                                      int32_t negative, int32_t msl, uint32_t pitch,
                                      int64_t vocab_size, void* stream);
/* Returns FW2V_ERR_BOUNDS (and clears it) if an earlier fw2v_kernel_batch launch
 * on this device skipped a block with an out-of-range id; synchronises `stream`. */
fw2v_status fw2v_kernel_batch_error(void* stream);

/* Host-only helpers (no device needed).
 * fw2v_lane_layout: the device row layout for a layer size: rows hold `pitch`
 * values (FP32: layer_size rounded up to 8) and lane l of a warp owns elements
 * ((i*32+l)*vec + j), i < nv, j < vec; dot products sum each lane's elements in
 * that order and combine lanes with an xor tree (16, 8, 4, 2, 1).
 * fw2v_exp_table: the 1000-entry sigmoid table of generate_expTable_h.cpp:46-55.
 * fw2v_unigram_firsts: first index of words 1..V-1 in the reference unigram
 * table of `table_size` entries (improved_driver_functions.cpp:44-58); words
 * never reached get table_size.  Returns 0, or -1 if V < 2. */
void fw2v_lane_layout(int32_t layer_size, int32_t precision, int32_t* vec, int32_t* nv,
                      int64_t* pitch);
void fw2v_exp_table(float* table);
int fw2v_unigram_firsts(const uint32_t* counts, int64_t vocab_size, int64_t table_size,
                        int64_t* firsts);
/* Copy n entries of the device unigram table starting at index `first`. */
fw2v_status fw2v_get_unigram(fw2v_handle* h, int64_t first, int64_t n, int32_t* out);

/* Nearest neighbours by cosine similarity, the evaluator behind same-label
 * precision@10 (the reference scores its vectors offline with public
 * word-similarity sets, analysis/hyperwords; the synthetic corpora carry a
 * planted label per word instead).  `table` holds rows of `pitch` elements
 * (FP32, or bfloat16 bits with FW2V_BF16), the first layer_size (<= 512) used;
 * cand[0..n_cand) are the rows searched; query q is candidate queries[q].  For
 * each query: the k (<= 32, < n_cand) most similar other candidates, most
 * similar first, as candidate indices in out_idx[q*k..] and cosines in
 * out_sim[q*k..]; ties go to the lower candidate index.  Device pointers;
 * asynchronous on `stream` (a cudaStream_t); takes its scratch from the
 * stream-ordered allocator. */
fw2v_status fw2v_neighbours(const void* table, int32_t precision, int64_t pitch, int32_t layer_size,
                            const int32_t* cand, int64_t n_cand, const int32_t* queries,
                            int64_t n_queries, int32_t k, int32_t* out_idx, float* out_sim,
                            void* stream);

/* Graph-walk corpora generated on the device (the reference reads walk
 * corpora as text, one walk per line with -cache-eos, through
 * createGlobalStream, improved_driver_functions.cpp:244-281; these write the
 * same token stream in device memory).
 * fw2v_random_walks: n_walks uniform random walks of walk_len nodes on a graph
 * in CSR form (offs[0..nodes], dst[offs[0]..offs[nodes]), device pointers),
 * walk w starting at starts[w]; each step takes a uniform neighbour chosen by
 * a counter-based hash of (seed, w, step), a node without neighbours stays.
 * Writes node ids, walk w at out[w*(walk_len+1) ..], then -1 after each walk.
 * fw2v_relabel_stream: such a stream in place: node x -> vocab_of[x], every
 * negative entry -> 0 (</s>). */
fw2v_status fw2v_random_walks(const int64_t* offs, const int32_t* dst, int64_t nodes, const int32_t* starts,
                              int64_t n_walks, int32_t walk_len, uint64_t seed, int32_t* out, void* stream);
fw2v_status fw2v_relabel_stream(int32_t* stream, int64_t n, const int32_t* vocab_of, int64_t nodes,
                                void* cuda_stream);

/* The handle's CUDA stream (a cudaStream_t), on which every kernel of the
 * handle runs; lets a caller time or order its own work against the epochs. */
void* fw2v_stream(fw2v_handle* h);

const char* fw2v_status_string(fw2v_status s);
/* Detail of the last error on this handle (empty string if none). */
const char* fw2v_last_error(fw2v_handle* h);
/* Library build information, e.g. "fw2v sm_100a". */
const char* fw2v_version(void);

/* ---- Batched training of many independent jobs ------------------------------
 * No counterpart in the reference, which trains one corpus per process.  A
 * batch holds many independent SGNS jobs (each its own vocabulary, corpus,
 * layer size, window, seed and tables) and trains all of them on one GPU with
 * one persistent training kernel per round: every epoch is cut into rounds of
 * whole sampling streams of all jobs, sampled on the device (the same method,
 * and for each job the same ids, negatives, learning rates and stochastic
 * rounding seeds as a single-job handle with the same configuration) and then
 * drained from one work queue of (job, sentence) items.  Sampling of round
 * r+1 overlaps training of round r; with use_graph the whole call is captured
 * and replayed as one CUDA graph.
 *
 * Jobs: layer_size <= 384, sigmoid FW2V_SIGMOID_TABLE, the same `negative` in
 * every job of a batch; the batch's precision and deterministic flags replace
 * the jobs' own.  Jobs run in rounds of one kernel family each: one vector per
 * lane (d <= 128), and wide rows (2 or 3 vectors per lane) with light or deep
 * pipelines, each family compiled for its own register budget. */
typedef struct fw2v_batch fw2v_batch;

typedef struct fw2v_batch_config {
  int32_t precision;      /* fw2v_precision of every job's tables */
  int32_t device;
  int32_t use_graph;      /* 1: each fw2v_batch_train call runs as one CUDA graph */
  int32_t deterministic;  /* 1: one warp trains every round's sentences in order */
  int64_t round_tokens;   /* readable tokens sampled per round (buffer size); 0: 2^27 */
  int64_t group_bytes;    /* table bytes of a group of jobs trained side by side; 0: half
                             the device's L2 cache; < 0: all jobs of a family in one group */
} fw2v_batch_config;

typedef struct fw2v_batch_stats {
  uint64_t words_read;    /* tokens read by all jobs' streams in the call */
  uint64_t words_kept;
  float ms;               /* device time of the call (sampling and training) */
  int32_t epochs;         /* epochs run in the call */
  int32_t rounds;         /* rounds per epoch */
  float train_ms;         /* device time of the training kernel launches, summed (-1: not timed) */
  int32_t train_launches; /* training kernel launches in the call */
} fw2v_batch_stats;

void fw2v_batch_config_default(fw2v_batch_config* cfg);
fw2v_status fw2v_batch_create(const fw2v_batch_config* cfg, fw2v_batch** out);
void fw2v_batch_destroy(fw2v_batch* b);
const char* fw2v_batch_last_error(fw2v_batch* b);

/* Add a job: its configuration, vocabulary (as fw2v_set_vocab) and corpus (as
 * fw2v_load_corpus, host memory).  Allocates and initialises its tables.
 * *job receives its index (0, 1, ...). */
fw2v_status fw2v_batch_add_job(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts, int64_t vocab_size,
                               uint64_t train_words, const int32_t* stream, int64_t stream_len,
                               const int64_t* chunk_off, int64_t n_chunks, int32_t* job);
/* fw2v_batch_add_job with the corpus in device memory (stream and chunk_off
 * device pointers, checked on the device as fw2v_load_corpus_device does);
 * counts stay in host memory. */
fw2v_status fw2v_batch_add_job_device(fw2v_batch* b, const fw2v_config* cfg, const uint32_t* counts,
                                      int64_t vocab_size, uint64_t train_words, const int32_t* stream,
                                      int64_t stream_len, const int64_t* chunk_off, int64_t n_chunks, int32_t* job);

/* A job's kernel shape: the lane vector width and vectors per lane (2 x 1:
 * 32 lanes of 2 floats cover d <= 64; 4 x 1: d <= 128, 16 lanes suffice for
 * d <= 64; 4 x 2: d <= 256; 4 x 3: d <= 384), the pipeline stages (2, 3, 4
 * or 6 targets in flight; 4 at most with 3 vectors per lane) and the staging
 * bits `prefetch`: bit 0, the target rows of each group of `stages` targets
 * are copied into shared memory while the previous group trains; bit 1, the
 * entering context row and the leaving row's original are staged by
 * cp.async.bulk copies from one lane (completion on an mbarrier) instead of
 * per-lane cp.async.  Defaults follow d and negative, both bits off;
 * fw2v_batch_tune picks them by measurement. */
fw2v_status fw2v_batch_set_shape(fw2v_batch* b, int32_t job, int32_t lane_vec, int32_t lane_nv, int32_t stages,
                                 int32_t prefetch);
fw2v_status fw2v_batch_get_shape(fw2v_batch* b, int32_t job, int32_t* lane_vec, int32_t* lane_nv,
                                 int32_t* stages, int32_t* prefetch);

/* The training grid of a kernel family (0: one vector per lane; 1: wide rows
 * with 2 or 3 stages (2 vectors per lane) or 2 stages (3 vectors); 2: other
 * wide rows): warps per block (sentences trained side by side in one block:
 * 1..8 in family 0, 1..6 in family 1, 1..4 in family 2; 0, the default: the
 * count of 8, 6, 4 or 2 that keeps the most warps resident per SM) and a cap
 * on blocks per SM (0: as many as fit). */
fw2v_status fw2v_batch_set_launch(fw2v_batch* b, int32_t family, int32_t warps_per_block, int32_t blocks_per_sm);
fw2v_status fw2v_batch_get_launch(fw2v_batch* b, int32_t family, int32_t* warps_per_block,
                                  int32_t* blocks_per_sm);

/* Autotuner: for every class of jobs with the same (lane-vector class of d,
 * window), time every shape on a sample of up to sample_tokens of the class's
 * first-epoch sentences and keep the fastest; then time the grid shapes on
 * all classes together.  Tables and sampler state are restored afterwards, so
 * training is unchanged apart from speed.  Report: per class, the fastest
 * words/s (tuned_wps) and the default shape's (default_wps), n_classes. */
typedef struct fw2v_batch_tune_report {
  int32_t n_classes;
  int32_t class_d[16], class_window[16], class_lane_vec[16], class_lane_nv[16], class_stages[16];
  int32_t class_prefetch[16];
  double tuned_wps[16], default_wps[16];
  int32_t warps_per_block[3], blocks_per_sm[3];  /* per kernel family */
} fw2v_batch_tune_report;
fw2v_status fw2v_batch_tune(fw2v_batch* b, int64_t sample_tokens, fw2v_batch_tune_report* report);

/* Train every job until it has trained its configured epochs (as fw2v_train:
 * a second call trains nothing). */
fw2v_status fw2v_batch_train(fw2v_batch* b, fw2v_batch_stats* stats);

/* Train the next n_epochs epochs of every job that has epochs left (as that
 * many fw2v_train_epoch calls); with use_graph, as one graph. */
fw2v_status fw2v_batch_train_epochs(fw2v_batch* b, int32_t n_epochs, fw2v_batch_stats* stats);

/* Words read and kept by one job since it was added. */
fw2v_status fw2v_batch_job_words(fw2v_batch* b, int32_t job, uint64_t* words_read, uint64_t* words_kept);

/* A job's tables as FP32 rows of ld floats (ld >= its layer_size). */
fw2v_status fw2v_batch_get_syn0(fw2v_batch* b, int32_t job, float* out, int64_t ld);
fw2v_status fw2v_batch_get_syn1neg(fw2v_batch* b, int32_t job, float* out, int64_t ld);

#ifdef __cplusplus
}
#endif
#endif
