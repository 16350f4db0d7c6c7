// full-w2v: drop-in command line for the FULL-W2V training program
// (src/FULL-W2V/FULL-W2V-driver.cu + improved_driver_functions.cpp +
// legacy_driver_functions.cpp), training on a B200 through libfw2v.
//
// Same flags and defaults (improved_driver_functions.cpp:403-501), same text
// front end (word reader, vocabulary, global token stream, vocabulary and corpus
// cache files), same .vec output (improved_driver_functions.cpp:225-242) and the
// same closing lines "Overall Words Per Second / Overall Words / Overall time"
// (FULL-W2V-driver.cu:450-451) that replication/sweep.py parses.
//
// Flags the GPU path has no use for (-streams, -kernel-batch-size) are accepted
// and ignored.  Added flags: -sigmoid table|exact, -deterministic 0|1,
// -device N.  Without -threads the number of sampling streams is chosen for the
// GPU (one stream per 256 stored sentences, at least 1, at most 4096) instead of
// the reference's CPU-thread default of 12.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fw2v.h"

namespace {

constexpr int kMaxString = 800;               // FULL-W2V-driver.cu:16
constexpr int64_t kVocabHashSize = 30000000;  // FULL-W2V-driver.cu:60 (reduce threshold 0.7x)

struct Options {
  std::string train, output, save_vocab, read_vocab, save_corpus, save_corpus_cache, read_corpus_cache;
  bool do_export = true, recount = false, cache_eos = false, pre_shuffle = false, epoch_shuffle = false;
  int binary = 0, debug = 2, min_count = 5, layer_size = 100, epochs = 5, window = 5, negative = 5;
  int threads = -1, msl = 1000, sigmoid = FW2V_SIGMOID_TABLE, deterministic = 0, device = 0;
  int precision = FW2V_FP32, tune = 1;
  int read_threads = 0;  // text reader threads (0: one per core, segments of >= 4 MB)
  unsigned long long seed = 0;
  float alpha = 0.025f, sample = 1e-3f;
  std::string jobs;  // manifest: one job's arguments per line, trained together
};

// ---------------------------------------------------------------------------
// Mapped files and the word reader
// ---------------------------------------------------------------------------
struct Mapped {
  const char* data = nullptr;
  uint64_t size = 0;
  bool open(const std::string& path) {
    int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) < 0) {
      ::close(fd);
      return false;
    }
    size = (uint64_t)st.st_size;
    if (size > 0) {
      void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (p == MAP_FAILED) {
        ::close(fd);
        return false;
      }
      data = (const char*)p;
    }
    ::close(fd);
    return true;
  }
  ~Mapped() {
    if (data) munmap((void*)data, size);
  }
};

// One word from a mapped file (improved_driver_functions.cpp:86-124): CR is
// skipped, a newline alone reads as "</s>", blanks and tabs separate words,
// words are cut at 799 bytes and the rest of an over-long word is skipped.
void read_word(std::string& word, const char* m, uint64_t max, uint64_t* cur) {
  word.clear();
  char c = 0;
  uint64_t pos = *cur;
  while (pos < max) {
    c = m[pos++];
    if (c == 13) continue;
    if (c == '\n') {
      if (!word.empty()) {
        pos--;
        break;
      }
      word = "</s>";
      *cur = pos;
      return;
    }
    if (c == ' ' || c == '\t') {
      if (!word.empty()) break;
      continue;
    }
    word.push_back(c);
    if ((int)word.size() >= kMaxString - 1) break;
  }
  if (pos == max || c == ' ' || c == '\t' || c == '\n') {
    *cur = pos;
    return;
  }
  while (pos < max && c != ' ' && c != '\t' && c != '\n') c = m[pos++];
  *cur = pos - 1;
}

// ---------------------------------------------------------------------------
// Vocabulary (legacy_driver_functions.cpp:26-124, improved_driver_functions.cpp:136-223)
// ---------------------------------------------------------------------------
struct Vocab {
  std::vector<std::string> words;
  std::vector<uint64_t> counts;
  std::unordered_map<std::string, int> index;
  int64_t min_reduce = 1;

  int find(const std::string& w) const {
    auto it = index.find(w);
    return it == index.end() ? -1 : it->second;
  }
  int add(const std::string& w) {
    words.push_back(w.substr(0, kMaxString - 1));
    counts.push_back(0);
    index[words.back()] = (int)words.size() - 1;
    return (int)words.size() - 1;
  }
  void rebuild_index() {
    index.clear();
    for (size_t i = 0; i < words.size(); i++) index.emplace(words[i], (int)i);
  }
  // Drop words seen at most min_reduce times (ReduceVocab).
  void reduce() {
    size_t k = 0;
    for (size_t i = 0; i < words.size(); i++) {
      if (counts[i] > (uint64_t)min_reduce) {
        words[k] = words[i];
        counts[k] = counts[i];
        k++;
      }
    }
    words.resize(k);
    counts.resize(k);
    rebuild_index();
    min_reduce++;
  }
  // Sort by count, "</s>" kept at 0, cut below min_count; returns the sum of the
  // remaining counts (SortVocab).  Ties keep their order: the reference's qsort
  // is glibc's stable merge sort.
  uint64_t sort_and_cut(int min_count) {
    std::vector<size_t> order(words.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    if (order.size() > 1)
      std::stable_sort(order.begin() + 1, order.end(),
                       [&](size_t a, size_t b) { return counts[a] > counts[b]; });
    std::vector<std::string> w2;
    std::vector<uint64_t> c2;
    uint64_t total = 0;
    for (size_t k = 0; k < order.size(); k++) {
      size_t i = order[k];
      if (counts[i] < (uint64_t)min_count && k != 0) continue;
      w2.push_back(words[i]);
      c2.push_back(counts[i]);
      total += counts[i];
    }
    words.swap(w2);
    counts.swap(c2);
    rebuild_index();
    return total;
  }
};

// LearnVocabFromTrainFile (improved_driver_functions.cpp:136-164).  The word
// that ends exactly at the end of the file is not counted.
uint64_t learn_vocab(Vocab& v, const Mapped& f, int min_count) {
  v.add("</s>");
  std::string w;
  uint64_t train_words = 0;
  for (uint64_t pos = 0; pos < f.size;) {
    read_word(w, f.data, f.size, &pos);
    if (pos == f.size) break;
    train_words++;
    int i = v.find(w);
    if (i < 0) {
      i = v.add(w);
      v.counts[i] = 1;
    } else {
      v.counts[i]++;
    }
    if ((int64_t)v.words.size() > (int64_t)(kVocabHashSize * 0.7)) v.reduce();
  }
  (void)train_words;
  return v.sort_and_cut(min_count) + 1;
}

// ReadVocab (improved_driver_functions.cpp:167-196): "word count" per line.
bool read_vocab(Vocab& v, const std::string& path, int min_count, uint64_t* train_words) {
  Mapped f;
  if (!f.open(path)) return false;
  std::string w, c;
  for (uint64_t pos = 0; pos < f.size; pos++) {
    read_word(w, f.data, f.size, &pos);
    int i = v.add(w);
    read_word(c, f.data, f.size, &pos);
    v.counts[i] = (uint64_t)(uint32_t)atoi(c.c_str());
  }
  *train_words = v.sort_and_cut(min_count);
  return true;
}

// recountVocab (improved_driver_functions.cpp:199-223).
uint64_t recount_vocab(Vocab& v, const Mapped& f, int min_count) {
  std::fill(v.counts.begin(), v.counts.end(), 0);
  std::string w;
  for (uint64_t pos = 0; pos < f.size;) {
    read_word(w, f.data, f.size, &pos);
    int i = v.find(w);
    if (i >= 0) v.counts[i]++;
  }
  return v.sort_and_cut(min_count);
}

bool save_vocab(const Vocab& v, const std::string& path) {
  FILE* fo = fopen(path.c_str(), "wb");
  if (!fo) return false;
  for (size_t i = 0; i < v.words.size(); i++) fprintf(fo, "%s %d\n", v.words[i].c_str(), (int)v.counts[i]);
  fclose(fo);
  return true;
}

// ---------------------------------------------------------------------------
// Corpus: the global token stream cut into stored chunks
// ---------------------------------------------------------------------------
struct Corpus {
  std::vector<int32_t> stream;     // trailing 0 included
  std::vector<int64_t> chunk_off;  // start of each stored chunk
};

// createGlobalStream (improved_driver_functions.cpp:244-281): in-vocabulary
// words only, "</s>" kept with -cache-eos, a chunk ends after msl words or at
// "</s>".  A run of out-of-vocabulary words reaching the end of the file stores
// nothing (the reference stores -1 there).
void create_stream(Corpus& c, const Vocab& v, const Mapped& f, int msl, bool cache_eos) {
  std::string w;
  int64_t sent_length = 0;
  for (uint64_t pos = 0; pos < f.size;) {
    int id = -1;
    while (pos < f.size && id == -1) {
      read_word(w, f.data, f.size, &pos);
      id = v.find(w);
    }
    if (id == -1) break;
    if (!cache_eos && id == 0) continue;
    if (sent_length == 0) c.chunk_off.push_back((int64_t)c.stream.size());
    c.stream.push_back(id);
    sent_length++;
    if (id == 0 || sent_length >= msl) sent_length = 0;
  }
  c.stream.push_back(0);
}

// ---------------------------------------------------------------------------
// Parallel text reader: the same vocabulary and token stream as learn_vocab /
// create_stream, with the file cut into segments at line starts and each
// segment read by its own thread.  The word reader keeps no state across a
// line start, so every segment reads the words the serial pass reads there.
// Each thread counts its words with the position of their first occurrence;
// merged, the insertion order of the serial pass is the order of first
// occurrence, which the stable sort by count keeps for ties.  A vocabulary
// that would reach the serial pass's ReduceVocab threshold is read serially.
// ---------------------------------------------------------------------------
struct Segments {
  std::vector<uint64_t> begin, end;
};

// n segments of f starting at line starts (fewer if lines are long).
Segments cut_segments(const Mapped& f, int n) {
  Segments s;
  uint64_t pos = 0;
  for (int k = 0; k < n && pos < f.size; k++) {
    uint64_t e = k + 1 == n ? f.size : std::max(pos, f.size / n * (k + 1));
    while (e < f.size && f.data[e - 1] != '\n') e++;
    if (e <= pos) continue;
    s.begin.push_back(pos);
    s.end.push_back(e);
    pos = e;
  }
  return s;
}

int reader_threads(const Options& o, const Mapped& f) {
  if (o.read_threads > 0) return o.read_threads;
  const int cores = (int)std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)cores, f.size / (4u << 20)));
}

struct SegmentCounts {
  std::unordered_map<std::string, std::pair<uint64_t, uint64_t>> words;  // count, first token index
  uint64_t tokens = 0;
};

// Returns false (and leaves v untouched) when the vocabulary is too large for
// the parallel pass.
bool learn_vocab_parallel(Vocab& v, const Mapped& f, int min_count, int n, uint64_t* train_words) {
  const Segments seg = cut_segments(f, n);
  const size_t ns = seg.begin.size();
  std::vector<SegmentCounts> part(ns);
  std::vector<std::thread> pool;
  for (size_t k = 0; k < ns; k++)
    pool.emplace_back([&, k] {
      std::string w;
      SegmentCounts& c = part[k];
      const uint64_t end = seg.end[k];
      for (uint64_t pos = seg.begin[k]; pos < end;) {
        read_word(w, f.data, end, &pos);
        // the word that ends exactly at the end of the file is not counted
        if (pos == end && end == f.size) break;
        auto it = c.words.find(w);
        if (it == c.words.end()) c.words.emplace(w, std::make_pair(1ull, c.tokens));
        else it->second.first++;
        c.tokens++;
      }
    });
  for (auto& t : pool) t.join();
  std::unordered_map<std::string, std::pair<uint64_t, uint64_t>> all;
  uint64_t base = 0;
  for (size_t k = 0; k < ns; k++) {
    for (auto& kv : part[k].words) {
      auto it = all.find(kv.first);
      const uint64_t first = base + kv.second.second;
      if (it == all.end()) all.emplace(kv.first, std::make_pair(kv.second.first, first));
      else {
        it->second.first += kv.second.first;
        it->second.second = std::min(it->second.second, first);
      }
    }
    base += part[k].tokens;
    part[k].words.clear();
  }
  if ((int64_t)all.size() + 1 > (int64_t)(kVocabHashSize * 0.7)) return false;
  std::vector<std::pair<uint64_t, const std::string*>> order;  // first occurrence, word
  order.reserve(all.size());
  for (auto& kv : all)
    if (kv.first != "</s>") order.emplace_back(kv.second.second, &kv.first);
  std::sort(order.begin(), order.end());
  v.add("</s>");
  auto eos = all.find("</s>");
  v.counts[0] = eos == all.end() ? 0 : eos->second.first;
  for (auto& o : order) {
    const int i = v.add(*o.second);
    v.counts[i] = all[*o.second].first;
  }
  *train_words = v.sort_and_cut(min_count) + 1;
  return true;
}

// create_stream over segments read in parallel: each thread maps its words to
// ids (in-vocabulary words only, "</s>" kept with -cache-eos); the chunk cuts,
// which carry across segments, are made in one pass over the joined stream.
void create_stream_parallel(Corpus& c, const Vocab& v, const Mapped& f, int msl, bool cache_eos, int n) {
  const Segments seg = cut_segments(f, n);
  const size_t ns = seg.begin.size();
  std::vector<std::vector<int32_t>> part(ns);
  std::vector<std::thread> pool;
  for (size_t k = 0; k < ns; k++)
    pool.emplace_back([&, k] {
      std::string w;
      const uint64_t end = seg.end[k];
      for (uint64_t pos = seg.begin[k]; pos < end;) {
        read_word(w, f.data, end, &pos);
        const int id = v.find(w);
        if (id < 0 || (!cache_eos && id == 0)) continue;
        part[k].push_back(id);
      }
    });
  for (auto& t : pool) t.join();
  size_t total = 1;
  for (auto& p : part) total += p.size();
  c.stream.reserve(total);
  for (auto& p : part) {
    c.stream.insert(c.stream.end(), p.begin(), p.end());
    std::vector<int32_t>().swap(p);
  }
  int64_t sent_length = 0;
  for (size_t i = 0; i < c.stream.size(); i++) {
    if (sent_length == 0) c.chunk_off.push_back((int64_t)i);
    sent_length++;
    if (c.stream[i] == 0 || sent_length >= msl) sent_length = 0;
  }
  c.stream.push_back(0);
}

// saveCorpusCache / saveCorpus (improved_driver_functions.cpp:293-318).
bool save_corpus(const Corpus& c, const Vocab& v, uint64_t train_words, int msl, const std::string& path,
                 bool as_words) {
  FILE* fo = fopen(path.c_str(), "w");
  if (!fo) return false;
  if (!as_words) fprintf(fo, "%llu %llu\n", (unsigned long long)c.chunk_off.size(), (unsigned long long)train_words);
  for (int64_t off : c.chunk_off) {
    int w = 0;
    for (; w < msl && c.stream[off + w] != 0; w++) {
      if (as_words) fprintf(fo, "%s ", v.words[c.stream[off + w]].c_str());
      else fprintf(fo, "%u ", (unsigned)c.stream[off + w]);
    }
    if (w > 0) fprintf(fo, "\n");
  }
  fclose(fo);
  return true;
}

// readCorpusCache (improved_driver_functions.cpp:320-401): "S N" then ids; a
// "</s>" ends a chunk (stored with -cache-eos), and every msl+1-th id starts a
// new chunk after an inserted 0.
bool read_corpus_cache(Corpus& c, const std::string& path, int msl, bool cache_eos, uint64_t* train_words) {
  Mapped f;
  if (!f.open(path)) return false;
  std::string w;
  uint64_t pos = 0;
  read_word(w, f.data, f.size, &pos);
  read_word(w, f.data, f.size, &pos);
  *train_words = (uint64_t)atoi(w.c_str());
  pos++;
  c.chunk_off.push_back(0);
  uint64_t msl_trigger = 0;
  auto new_chunk = [&]() {
    c.stream.push_back(0);
    c.chunk_off.push_back((int64_t)c.stream.size());
    msl_trigger = 0;
  };
  while (pos < f.size) {
    read_word(w, f.data, f.size, &pos);
    if (w == "</s>") {
      if (cache_eos) new_chunk();
    } else {
      if (msl_trigger == (uint64_t)msl) new_chunk();
      else msl_trigger++;
      c.stream.push_back(atoi(w.c_str()));
    }
  }
  // The last chunk pointer points past the data (the reference's count is
  // sentence_pos - 1); drop it and close the stream.
  c.chunk_off.pop_back();
  c.stream.push_back(0);
  return true;
}

// shuffleSentences (improved_driver_functions.cpp:283-291) with the C library's
// rand(), unseeded as in the reference.
void shuffle_chunks(std::vector<int64_t>& off) {
  if (off.empty()) return;
  for (uint64_t i = off.size() - 1; i > 0; i--) {
    uint64_t j = (uint64_t)((rand() / (double)RAND_MAX) * (double)(i + 1));
    if (j >= off.size()) j = off.size() - 1;  // rand() == RAND_MAX picks i+1
    std::swap(off[j], off[i]);
  }
}

// saveModel (improved_driver_functions.cpp:225-242).
bool save_model(const std::string& path, const Vocab& v, const std::vector<float>& syn0, int d, int binary) {
  FILE* fo = fopen(path.c_str(), "wb");
  if (!fo) return false;
  fprintf(fo, "%d %d\n", (int)v.words.size(), d);
  for (size_t a = 0; a < v.words.size(); a++) {
    fprintf(fo, "%s ", v.words[a].c_str());
    const float* row = syn0.data() + a * d;
    if (binary) fwrite(row, sizeof(float), d, fo);
    else
      for (int b = 0; b < d; b++) fprintf(fo, "%f ", row[b]);
    fprintf(fo, "\n");
  }
  fclose(fo);
  return true;
}

double now_s() {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC_RAW, &t);
  return (double)t.tv_sec + t.tv_nsec / 1e9;
}

int arg_pos(const char* name, int argc, char** argv) {
  for (int a = 1; a < argc; a++)
    if (!strcmp(name, argv[a])) return a;
  return -1;
}

void usage(const char* prog) {
  printf("SGNS word2vec (FULL-W2V method) trained on an NVIDIA B200\n\nOptions:\n");
  printf("** FILES & I/O **\n");
  printf("\t-train <file>\t\tUse text data from <file> to train the model\n");
  printf("\t-output <file>\t\tUse <file> to save the resulting word vectors\n");
  printf("\t-no-export\t\tSkip exporting vectors after training\n");
  printf("\t-binary <int>\t\tSave the vectors in binary mode; default is 0 (off)\n");
  printf("\t-debug <int>\t\tDebug mode (default 2)\n");
  printf("\t-save-vocab <file>\tSave the vocabulary to <file>\n");
  printf("\t-read-vocab <file>\tRead the vocabulary from <file>\n");
  printf("\t-min-count <int>\tDiscard words that appear less than <int> times; default 5\n");
  printf("\t-recount\t\tRecount vocabulary counts from the training data\n");
  printf("\t-save-corpus <file>\tSave the corpus as interpreted\n");
  printf("\t-save-corpus-cache <file>\tSave the corpus cache\n");
  printf("\t-read-corpus-cache <file>\tRead the corpus cache instead of the training data\n");
  printf("\t-cache-eos\t\tKeep line ends as sentence ends\n");
  printf("\t-pre-shuffle\t\tShuffle sentences before the first epoch\n");
  printf("\t-epoch-shuffle\t\tShuffle sentences after each epoch\n");
  printf("** TRAINING PARAMETERS **\n");
  printf("\t-size <int>\t\tSize of word vectors; default 100\n");
  printf("\t-epoch(s), -iter(s) <int>\tNumber of epochs; default 5\n");
  printf("\t-alpha <float>\t\tStarting learning rate; default 0.025\n");
  printf("\t-window <int>\t\tMax skip length; default 5 (1..15)\n");
  printf("\t-sample <float>\t\tSubsampling threshold; default 1e-3\n");
  printf("\t-negative(s) <int>\tNegative examples; default 5 (0..31)\n");
  printf("\t-sigmoid table|exact\tSigmoid: the reference's 1000-entry table (default) or exact\n");
  printf("\t-deterministic 0|1\tTrain sentences one at a time in stream order\n");
  printf("\t-precision fp32|bf16\tEmbedding tables in FP32 (default) or bfloat16 with stochastic rounding\n");
  printf("\t-seed <int>\t\t0 (default): the reference's seeds; otherwise offsets every LCG start, and\n"
         "\t\t\t\t-pre-shuffle / -epoch-shuffle use the library's seeded shuffle on the GPU\n");
  printf("** MANY JOBS **\n");
  printf("\t-jobs <file>\t\tTrain the jobs listed in <file> (one job's options per line, '#' comments)\n");
  printf("\t\t\t\ttogether on one GPU; -precision, -device, -deterministic apply to all\n");
  printf("\t-tune 0|1\t\tWith -jobs, pick kernel shapes by measurement first (default 1)\n");
  printf("** PARALLEL UTILIZATION **\n");
  printf("\t-thread(s) <int>\tSampling streams (the reference's CPU threads); default: one per 256 sentences\n");
  printf("\t-max-sentence-length, -msl <int>\tMaximum sentence length; default 1000\n");
  printf("\t-read-threads <int>\tThreads reading the text file; default one per core (segments of >= 4 MB)\n");
  printf("\t-device <int>\t\tCUDA device; default 0\n");
  printf("\t-streams, -kernel-batch-size <int>\tAccepted for compatibility, unused\n");
  printf("\nExamples:\n%s -train data.txt -output vec.txt -size 128 -window 5 -sample 1e-4 -negative 5 -epoch 3\n\n",
         prog);
}

bool parse(int argc, char** argv, Options& o) {
  if (argc == 1 || arg_pos("-help", argc, argv) > 0) {
    usage(argv[0]);
    return false;
  }
  auto val = [&](const char* n) -> const char* {
    int i = arg_pos(n, argc, argv);
    return (i > 0 && i + 1 < argc) ? argv[i + 1] : nullptr;
  };
  auto first = [&](std::initializer_list<const char*> ns) -> const char* {
    for (const char* n : ns)
      if (const char* v = val(n)) return v;
    return nullptr;
  };
  if (const char* v = val("-output")) o.output = v;
  if (arg_pos("-no-export", argc, argv) > 0) o.do_export = false;
  if (const char* v = val("-binary")) o.binary = atoi(v);
  if (const char* v = val("-debug")) o.debug = atoi(v);
  if (const char* v = val("-save-vocab")) o.save_vocab = v;
  if (const char* v = val("-read-vocab")) o.read_vocab = v;
  if (const char* v = val("-train")) o.train = v;
  if (const char* v = val("-min-count")) o.min_count = atoi(v);
  if (arg_pos("-recount", argc, argv) > 0) o.recount = true;
  if (const char* v = val("-save-corpus")) o.save_corpus = v;
  if (const char* v = val("-save-corpus-cache")) o.save_corpus_cache = v;
  if (const char* v = val("-read-corpus-cache")) o.read_corpus_cache = v;
  if (arg_pos("-cache-eos", argc, argv) > 0) o.cache_eos = true;
  if (arg_pos("-pre-shuffle", argc, argv) > 0) o.pre_shuffle = true;
  if (arg_pos("-epoch-shuffle", argc, argv) > 0) o.epoch_shuffle = true;
  if (const char* v = val("-size")) o.layer_size = atoi(v);
  if (const char* v = first({"-epoch", "-epochs", "-iter", "-iters"})) o.epochs = atoi(v);
  if (const char* v = val("-alpha")) o.alpha = (float)atof(v);
  if (const char* v = val("-window")) o.window = atoi(v);
  if (const char* v = val("-sample")) o.sample = (float)atof(v);
  if (const char* v = first({"-negative", "-negatives"})) o.negative = atoi(v);
  if (const char* v = first({"-thread", "-threads"})) o.threads = atoi(v);
  if (const char* v = first({"-msl", "-max-sentence-length"})) o.msl = atoi(v);
  if (const char* v = val("-sigmoid")) o.sigmoid = !strcmp(v, "exact") ? FW2V_SIGMOID_EXACT : FW2V_SIGMOID_TABLE;
  if (const char* v = val("-deterministic")) o.deterministic = atoi(v);
  if (const char* v = val("-device")) o.device = atoi(v);
  if (const char* v = val("-precision")) o.precision = !strcmp(v, "bf16") ? FW2V_BF16 : FW2V_FP32;
  if (const char* v = val("-seed")) o.seed = strtoull(v, nullptr, 10);
  if (const char* v = val("-read-threads")) o.read_threads = atoi(v);
  if (const char* v = val("-jobs")) o.jobs = v;
  if (const char* v = val("-tune")) o.tune = atoi(v);
  return true;
}

// The options of one manifest line, on top of defaults.
bool parse_line(const std::string& line, Options& o) {
  std::vector<std::string> toks;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && isspace((unsigned char)line[i])) i++;
    size_t j = i;
    while (j < line.size() && !isspace((unsigned char)line[j])) j++;
    if (j > i) toks.push_back(line.substr(i, j - i));
    i = j;
  }
  if (toks.empty() || toks[0][0] == '#') return false;
  std::vector<char*> argv{(char*)"full-w2v"};
  for (std::string& t : toks) argv.push_back(&t[0]);
  return parse((int)argv.size(), argv.data(), o);
}

int fail_status(const char* what, fw2v_status s, fw2v_handle* h) {
  fprintf(stderr, "ERROR: %s: %s%s%s\n", what, fw2v_status_string(s), h ? ": " : "", h ? fw2v_last_error(h) : "");
  return 1;
}

}  // namespace

// SetupNetwork (FULL-W2V-driver.cu:356-425): vocabulary, corpus stream and
// chunks, the caches and the stream count.  Returns 0 to go on training, -1
// when there is nothing to train (preprocessing only), or a process exit code.
int prepare(Options& o, Vocab& vocab, Corpus& corpus, uint64_t& train_words) {
  if (!o.train.empty()) {
    Mapped f;
    if (!f.open(o.train)) {
      printf("ERROR: Training data not found!\n");
      return 1;
    }
    if (o.debug > 0) printf("Train file size = %lluK\n", (unsigned long long)(f.size / 1000));
    if (!o.read_vocab.empty()) {
      if (!read_vocab(vocab, o.read_vocab, o.min_count, &train_words)) {
        printf("Vocabulary file \"%s\" not found!\n", o.read_vocab.c_str());
        return 1;
      }
    } else {
      const int n = reader_threads(o, f);
      if (n <= 1 || !learn_vocab_parallel(vocab, f, o.min_count, n, &train_words))
        train_words = learn_vocab(vocab, f, o.min_count);
    }
    if (o.recount) train_words = recount_vocab(vocab, f, o.min_count);
    if (!o.save_vocab.empty()) save_vocab(vocab, o.save_vocab);
    if (!o.read_corpus_cache.empty()) {
      if (!read_corpus_cache(corpus, o.read_corpus_cache, o.msl, o.cache_eos, &train_words)) {
        printf("Corpus cache file \"%s\" not found!\n", o.read_corpus_cache.c_str());
        return 1;
      }
    } else {
      const int n = reader_threads(o, f);
      if (n > 1) create_stream_parallel(corpus, vocab, f, o.msl, o.cache_eos, n);
      else create_stream(corpus, vocab, f, o.msl, o.cache_eos);
    }
  } else {
    if (o.read_vocab.empty()) {
      printf("ERROR: No vocabulary or training file to generate vocabulary from! Please specify -train or -read-vocab\n");
      return 1;
    }
    if (!read_vocab(vocab, o.read_vocab, o.min_count, &train_words)) {
      printf("Vocabulary file \"%s\" not found!\n", o.read_vocab.c_str());
      return 1;
    }
    if (!o.save_vocab.empty()) save_vocab(vocab, o.save_vocab);
    if (o.read_corpus_cache.empty()) {
      printf("ERROR: No corpus cache or training file to learn from! Please specify -train or -read-corpus-cache\n");
      return 1;
    }
    if (!read_corpus_cache(corpus, o.read_corpus_cache, o.msl, o.cache_eos, &train_words)) {
      printf("Corpus cache file \"%s\" not found!\n", o.read_corpus_cache.c_str());
      return 1;
    }
  }
  if (!o.save_corpus_cache.empty()) save_corpus(corpus, vocab, train_words, o.msl, o.save_corpus_cache, false);
  if (!o.save_corpus.empty()) save_corpus(corpus, vocab, train_words, o.msl, o.save_corpus, true);
  const int64_t n_chunks = (int64_t)corpus.chunk_off.size();
  if (o.threads < 0) o.threads = (int)std::max<int64_t>(1, std::min<int64_t>(4096, n_chunks / 256));
  if (o.debug > 1)
    printf("%lld sentences spread across %d sampling streams == %lld sentences/stream\n", (long long)n_chunks,
           o.threads, (long long)(n_chunks / std::max(o.threads, 1)));
  if (o.output.empty()) return -1;
  if (n_chunks == 0) {
    printf("ERROR: the corpus holds no in-vocabulary words\n");
    return 1;
  }

  return 0;
}

fw2v_config job_config(const Options& o) {
  fw2v_config cfg;
  fw2v_config_default(&cfg);
  cfg.layer_size = o.layer_size;
  cfg.window = o.window;
  cfg.negative = o.negative;
  cfg.epochs = o.epochs;
  cfg.threads = o.threads;
  cfg.msl = o.msl;
  cfg.alpha = o.alpha;
  cfg.sample = o.sample;
  cfg.sigmoid = o.sigmoid;
  cfg.deterministic = o.deterministic;
  cfg.device = o.device;
  cfg.precision = o.precision;
  cfg.seed = o.seed;
  return cfg;
}

int batch_fail(const char* what, fw2v_status st, fw2v_batch* b) {
  fprintf(stderr, "ERROR: %s: %s: %s\n", what, fw2v_status_string(st), b ? fw2v_batch_last_error(b) : "");
  fw2v_batch_destroy(b);
  return 1;
}

// -jobs: every manifest line is one job's command line; all jobs train
// together in one libfw2v batch and each exports its own vectors.
int run_jobs(const Options& g) {
  std::FILE* f = std::fopen(g.jobs.c_str(), "r");
  if (!f) {
    printf("ERROR: job manifest \"%s\" not found!\n", g.jobs.c_str());
    return 1;
  }
  std::vector<Options> opts;
  char buf[1 << 14];
  while (std::fgets(buf, sizeof(buf), f)) {
    Options o;
    o.debug = 0;
    if (!parse_line(buf, o)) continue;
    o.precision = g.precision;  // batch-wide settings
    o.device = g.device;
    o.deterministic = g.deterministic;
    opts.push_back(o);
  }
  std::fclose(f);
  if (opts.empty()) {
    printf("ERROR: the job manifest lists no jobs\n");
    return 1;
  }
  fw2v_batch_config bc;
  fw2v_batch_config_default(&bc);
  bc.precision = g.precision;
  bc.device = g.device;
  bc.deterministic = g.deterministic;
  fw2v_batch* b = nullptr;
  fw2v_status st = fw2v_batch_create(&bc, &b);
  if (st != FW2V_OK) return fail_status("batch_create", st, nullptr);
  std::vector<Vocab> vocabs(opts.size());
  for (size_t j = 0; j < opts.size(); j++) {
    Corpus corpus;
    uint64_t train_words = 0;
    if (const int r = prepare(opts[j], vocabs[j], corpus, train_words)) {
      fw2v_batch_destroy(b);
      if (r < 0) printf("ERROR: job %zu has no -output\n", j + 1);
      return 1;
    }
    if (opts[j].pre_shuffle) shuffle_chunks(corpus.chunk_off);
    std::vector<uint32_t> counts(vocabs[j].counts.size());
    for (size_t i = 0; i < counts.size(); i++) counts[i] = (uint32_t)vocabs[j].counts[i];
    const fw2v_config cfg = job_config(opts[j]);
    int32_t id = 0;
    st = fw2v_batch_add_job(b, &cfg, counts.data(), (int64_t)counts.size(), train_words, corpus.stream.data(),
                            (int64_t)corpus.stream.size(), corpus.chunk_off.data(),
                            (int64_t)corpus.chunk_off.size(), &id);
    if (st != FW2V_OK) return batch_fail("add job", st, b);
  }
  if (g.tune && !g.deterministic) {
    fw2v_batch_tune_report rep;
    if ((st = fw2v_batch_tune(b, 0, &rep)) != FW2V_OK) return batch_fail("tune", st, b);
  }
  const double t0 = now_s();
  fw2v_batch_stats bs;
  if ((st = fw2v_batch_train(b, &bs)) != FW2V_OK) return batch_fail("train", st, b);
  const double t1 = now_s();
  for (size_t j = 0; j < opts.size(); j++) {
    uint64_t wr = 0, wk = 0;
    fw2v_batch_job_words(b, (int32_t)j, &wr, &wk);
    printf("Job %zu Words: %llu\n", j + 1, (unsigned long long)wr);
  }
  printf("\nOverall Words Per Second: %.4f\n", bs.words_read / (t1 - t0));
  printf("Overall Words: %llu\nOverall time: %f\n", (unsigned long long)bs.words_read, t1 - t0);
  for (size_t j = 0; j < opts.size(); j++) {
    if (!opts[j].do_export) continue;
    const int d = opts[j].layer_size;
    std::vector<float> syn0(vocabs[j].counts.size() * (size_t)d);
    if ((st = fw2v_batch_get_syn0(b, (int32_t)j, syn0.data(), d)) != FW2V_OK) return batch_fail("export", st, b);
    if (!save_model(opts[j].output, vocabs[j], syn0, d, opts[j].binary)) {
      fprintf(stderr, "ERROR: cannot write %s\n", opts[j].output.c_str());
      fw2v_batch_destroy(b);
      return 1;
    }
  }
  fw2v_batch_destroy(b);
  return 0;
}

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) return 0;
  if (o.debug > 0) {
    fprintf(stderr, "** FILES & I/O **\n");
    if (!o.do_export && !o.output.empty()) fprintf(stderr, "!!\tProcess will train but will not export a model!\n");
    else if (!o.output.empty()) fprintf(stderr, "Trained model will export to file: %s\n", o.output.c_str());
    else fprintf(stderr, "!!\tPreprocessing only -- no training.\n");
    fprintf(stderr, "layer size: %d, epochs: %d, alpha: %.5f, window: %d, sample: %f, negative: %d\n",
            o.layer_size, o.epochs, o.alpha, o.window, o.sample, o.negative);
  }

  Vocab vocab;
  Corpus corpus;
  uint64_t train_words = 0;
  if (!o.jobs.empty()) return run_jobs(o);
  if (const int r = prepare(o, vocab, corpus, train_words)) return r < 0 ? 0 : r;
  const int64_t n_chunks = (int64_t)corpus.chunk_off.size();
  // -seed 0: the reference's libc rand() shuffles on the host; another seed:
  // the library's seeded Fisher-Yates on the device, shuffle n keyed by
  // (seed, n)
  const bool device_shuffle = o.seed != 0;
  auto shuffle_key = [&](uint64_t n) { return (uint64_t)o.seed + 0x9E3779B97F4A7C15ULL * (n + 1); };
  if (o.pre_shuffle && !device_shuffle) shuffle_chunks(corpus.chunk_off);

  // InitNet + Train_SGNS through libfw2v
  const fw2v_config cfg = job_config(o);
  fw2v_handle* h = nullptr;
  fw2v_status st = fw2v_create(&cfg, &h);
  if (st != FW2V_OK) return fail_status("create", st, nullptr);
  std::vector<uint32_t> counts(vocab.counts.size());
  for (size_t i = 0; i < counts.size(); i++) counts[i] = (uint32_t)vocab.counts[i];
  if ((st = fw2v_set_vocab(h, counts.data(), (int64_t)counts.size(), train_words)) != FW2V_OK)
    return fail_status("set_vocab", st, h);
  if ((st = fw2v_load_corpus(h, corpus.stream.data(), (int64_t)corpus.stream.size(), corpus.chunk_off.data(),
                             n_chunks)) != FW2V_OK)
    return fail_status("load_corpus", st, h);
  uint64_t shuffles = 0;
  if (o.pre_shuffle && device_shuffle && (st = fw2v_shuffle_chunks(h, shuffle_key(shuffles++))) != FW2V_OK)
    return fail_status("shuffle_chunks", st, h);

  const double t0 = now_s();
  uint64_t words = 0;
  for (int e = 0; e < o.epochs; e++) {
    fw2v_epoch_stats es;
    if (o.epoch_shuffle) {
      if ((st = fw2v_sample_epoch(h)) != FW2V_OK || (st = fw2v_train_sampled(h, &es)) != FW2V_OK)
        return fail_status("train", st, h);
      if (e + 1 < o.epochs && device_shuffle) {
        if ((st = fw2v_shuffle_chunks(h, shuffle_key(shuffles++))) != FW2V_OK)
          return fail_status("shuffle_chunks", st, h);
      } else if (e + 1 < o.epochs) {
        shuffle_chunks(corpus.chunk_off);
        if ((st = fw2v_reorder_chunks(h, corpus.chunk_off.data(), n_chunks)) != FW2V_OK)
          return fail_status("reorder_chunks", st, h);
      }
    } else if ((st = fw2v_train_epoch(h, &es)) != FW2V_OK) {
      return fail_status("train", st, h);
    }
    words += es.words_read;
    if (o.debug > 0) {
      printf("%cEpoch %d/%d  Words: %llu  Words/sec: %.2fk", 13, e + 1, o.epochs, (unsigned long long)words,
             words / 1000.0 / std::max(now_s() - t0, 1e-9));
      fflush(stdout);
    }
  }
  const double t1 = now_s();
  printf("\nOverall Words Per Second: %.4f\n", words / (t1 - t0));
  printf("Overall Words: %llu\nOverall time: %f\n", (unsigned long long)words, t1 - t0);

  if (o.do_export) {
    std::vector<float> syn0(counts.size() * (size_t)o.layer_size);
    if ((st = fw2v_get_syn0(h, syn0.data(), o.layer_size)) != FW2V_OK) return fail_status("get_syn0", st, h);
    if (o.debug > 0) fprintf(stderr, "Saving model to: %s\n", o.output.c_str());
    if (!save_model(o.output, vocab, syn0, o.layer_size, o.binary)) {
      fprintf(stderr, "ERROR: cannot write %s\n", o.output.c_str());
      return 1;
    }
  }
  fw2v_destroy(h);
  return 0;
}
