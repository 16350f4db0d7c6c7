/*
 * TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the FULL-W2V hot path, used as the checker for the CUDA
 * library (libfw2v) in tests/, in __graft_entry__.smoke() and as the timed CPU
 * baseline in bench.py.  The product never links, loads or calls this code.
 *
 * Every function cites the reference file:line it restates (paths are relative
 * to the reference repository root, tlranda/FULL-W2V).  Integer work (LCG,
 * subsampling, unigram table, batch builder) is a literal restatement and is
 * pinned against golden dumps produced by the reference's own host code
 * (tests/golden/).  The SGNS update has two arithmetic modes:
 *   - ORC_F64: textbook FP64 arithmetic, the accuracy yardstick;
 *   - ORC_F32: FP32 with the CUDA kernel's exact operation order (per-lane FMA
 *     partials over a 32-lane layout, xor-tree reduction 16,8,4,2,1, FMA
 *     updates), so table-sigmoid runs can be compared bit for bit.
 */
#ifndef FW2V_ORACLE_H
#define FW2V_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_UNIGRAM_TABLE_SIZE 100000000LL
#define ORC_EXP_TABLE_SIZE 1000

/* word2vec linear congruential generator step (FULL-W2V-driver.cu:217,225). */
uint64_t orc_lcg_next(uint64_t r);

/* 1000-entry sigmoid tables as generate_expTable_h.cpp:46-71 builds them:
 * exp_table[i] = sigma((i/1000*2-1)*6) with [0]=0, [999]=1. */
void orc_exp_table(float* exp_table);

/* syn0 initialisation (improved_driver_functions.cpp:27-31): element i of the
 * V*d row-major matrix takes ((r_i & 0xFFFF)/65536 - 0.5)/d with r_i the
 * (i+1)-th LCG state from seed 1.  Rows are written with `pitch` floats. */
void orc_init_syn0(float* syn0, int64_t V, int d, int64_t pitch);
void orc_init_syn0_from(float* syn0, int64_t V, int d, int64_t pitch, uint64_t start);

/* Subsampling keep threshold (improved_driver_functions.cpp:71-77). */
void orc_subsample_table(const uint32_t* counts, int64_t V, float sample, uint64_t train_words,
                         float* p_keep);

/* Unigram table (improved_driver_functions.cpp:44-58) run by the literal
 * sequential fill loop over `table_size` entries, returned as runs: run j covers
 * table entries [run_start[j], run_start[j+1]) and holds word run_word[j]
 * (run_start[n_runs] = table_size).  Capacity of run arrays: V+1.
 * Returns the number of runs. If `table` is non-NULL the full table is also written. */
int64_t orc_unigram_runs(const uint32_t* counts, int64_t V, int64_t table_size, int64_t* run_start,
                         int32_t* run_word, int32_t* table);
int32_t orc_unigram_lookup(const int64_t* run_start, const int32_t* run_word, int64_t n_runs,
                           int64_t index);

/* ---- batch builder (FULL-W2V-driver.cu:103-114, 166-302) ---- */
typedef struct {
  const int32_t* stream;    /* token ids, trailing 0 included */
  int64_t stream_len;
  const int64_t* chunk_off; /* start of each stored chunk ("sentence") in `stream` */
  int64_t n_chunks;
  const float* p_keep;      /* subsampling thresholds, used when sample > 0 */
  float sample;
  const int64_t* run_start; /* unigram runs from orc_unigram_runs */
  const int32_t* run_word;
  int64_t n_runs;
  int64_t table_size;       /* unigram table size, 1e8 in the reference */
  int threads;              /* T: number of sampling streams */
  int msl;
  int negative;             /* K */
  int epochs;               /* E */
  float alpha0;
  uint64_t train_words;
} orc_sampler_cfg;

/* State a stream carries across epochs. */
typedef struct {
  uint64_t lcg;       /* next_random, seeded with the stream id */
  uint64_t wca_own;   /* words this stream has added to word_count_actual */
  float alpha;        /* current learning rate */
} orc_stream_state;

void orc_stream_init(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st);
void orc_stream_range(const orc_sampler_cfg* cfg, int stream_id, int64_t* first_chunk,
                      int64_t* end_chunk);

/* One epoch of stream `stream_id`.  Appends every recorded batch entry
 * (including zero-length ones: epoch-end drops and empty sentences) to
 * lens/alphas and the kept ids / K negatives per kept id to ids/negs.
 * Returns 0 on success, -1 if a capacity is exceeded, -2 on a read outside
 * the stream.  *words_read receives the tokens read this epoch. */
int orc_sample_epoch(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st,
                     int64_t cap_entries, int32_t* lens, float* alphas, int64_t cap_kept,
                     int32_t* ids, int32_t* negs, int64_t* n_entries, int64_t* n_kept,
                     uint64_t* words_read);

/* The first max_entries entries of that epoch (fewer if it ends before), with
 * *words_read the tokens they consumed: a bounded sample of the workload.  The
 * stream state is left mid-epoch. */
int orc_sample_epoch_prefix(const orc_sampler_cfg* cfg, int stream_id, orc_stream_state* st,
                            int64_t max_entries, int64_t cap_entries, int32_t* lens, float* alphas,
                            int64_t cap_kept, int32_t* ids, int32_t* negs, int64_t* n_entries,
                            int64_t* n_kept, uint64_t* words_read);

/* ---- SGNS update (FULL-W2V-kernels.cu:106-250, textbook windows) ---- */
enum { ORC_F64 = 64, ORC_F32 = 32 };
enum { ORC_SIGMOID_TABLE = 0, ORC_SIGMOID_EXACT = 1 };

typedef struct {
  int d;
  int64_t pitch;   /* floats per row */
  int window;      /* W */
  int negative;    /* K */
  int sigmoid;     /* ORC_SIGMOID_* */
  int vec, nv;     /* ORC_F32 lane layout: lane l holds elements ((i*32+l)*vec + j) */
  const float* exp_table;
} orc_train_cfg;

/* Train sentences serially in the given order.  Sentence s has lens[s] kept ids
 * at ids[starts[s]...] and negatives at negs[starts[s]*K ...], learning rate
 * alphas[s].  Tables are V x pitch. */
int orc_train_f32(const orc_train_cfg* cfg, float* syn0, float* syn1neg, int64_t V,
                  int64_t n_sent, const int64_t* starts, const int32_t* lens, const float* alphas,
                  const int32_t* ids, const int32_t* negs);
int orc_train_f64(const orc_train_cfg* cfg, double* syn0, double* syn1neg, int64_t V,
                  int64_t n_sent, const int64_t* starts, const int32_t* lens, const float* alphas,
                  const int32_t* ids, const int32_t* negs);

/* The same on bfloat16 tables (uint16 bit patterns): loads widen exactly, math
 * is the FP32 mode's, every write-back is row = SR(row + delta) with the
 * library's counter-based bits: seed of the training launch, sentence s as
 * uid, target k of centre w as event w*(K+1)+k, leaving position q as event
 * L*(K+1)+q; 16 bits per element from the element's vector (cfg->vec wide). */
int orc_train_bf16(const orc_train_cfg* cfg, uint16_t* syn0, uint16_t* syn1neg, int64_t V, int64_t n_sent,
                   const int64_t* starts, const int32_t* lens, const float* alphas, const int32_t* ids,
                   const int32_t* negs, uint64_t seed);
uint16_t orc_bf16_nearest(float x);
/* One element of the bfloat16 write-back: `stored` after its row moved from b
 * to a, with 16 random bits r16 (increment to the stochastic rounding of a,
 * added with round-to-nearest). */
uint16_t orc_bf16_writeback1(uint16_t stored, float a, float b, uint32_t r16);

/* Held-out SGNS loss in FP64: for every centre w and context c of every
 * sentence, -log sigma(<v_c, o_w>) - sum_k log sigma(-<v_c, o_nk>), negatives
 * given per centre.  Returns the sum; *pairs gets the number of (c, w) pairs. */
double orc_heldout_loss(const float* syn0, const float* syn1neg, int64_t pitch, int d, int window,
                        int negative, int64_t n_sent, const int64_t* starts, const int32_t* lens,
                        const int32_t* ids, const int32_t* negs, int64_t* pairs);

/* Timed CPU baseline (fw2v_cpu_sgns.c): every stream sampled and trained by
 * n_threads host threads on shared tables (Hogwild), FP32. */
int orc_cpu_sgns(const orc_sampler_cfg* scfg, const orc_train_cfg* tcfg, float* syn0, float* syn1neg,
                 int n_threads, int64_t max_entries_per_stream, uint64_t* words_read,
                 uint64_t* words_kept);

#ifdef __cplusplus
}
#endif
#endif
