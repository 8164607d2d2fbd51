// The B200 search engine (host C++): owns a device, a stream and grow-only device buffers; runs the
// level-synchronous gate-count search of the reference (src/cheese.cu:1249-1377, 1762-1849) on sm_100a kernels.
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "cz_spec.h"

namespace cz {

struct Options {
  int depth = -1;            // -1: the spec's budget
  bool dedupe = true;        // --no-dedupe
  bool sym = true;           // --no-sym
  int store64 = 0;           // 0: int32 residual limbs, promoted to int64 when a value leaves int32; 1: int64 from the start
  int profile = 0;           // device times (CUDA events on the engine's stream): 1 level kernels, 2 also the dedupe
  bool nogoal = false;       // never report the goal (distance-table build)
  int table_k = 0;           // --table K
  std::string cache_dir = "build";   // distance-table cache directory ("" : no cache)
  bool mitm = false;         // --mitm
};

struct LevelStats {
  int t = 0;
  long long parents = 0, prefixes = 0, cut_w3 = 0, cut_lb = 0, survivors = 0, distinct = 0;
  bool proved_unsat = false;
  double seconds = 0;
  int dir = 0;               // 0 a plain level; 1 a level of the distance-table build ("dir": "table"); 2 / 3 a
                             // forward / backward level of the meet-in-the-middle search ("dir": "fwd" / "bwd")
};

struct SearchResult {
  int rc = 1;                          // 0 circuit, 1 proof (or stopped), 4 overflow, 5 CUDA error
  bool depth0 = false;                 // the target equals the goal
  std::vector<int> circuit;            // candidate indices of the found circuit
  long long n_found = 0;
  int nsym = 0;
  bool store64 = false;                // the run used int64 limbs
  int levels = 0;
  long long prefixes = 0;              // sum of the per-level "prefixes" fields
  long long launches = 0;              // kernels launched by the engine
  long long t_evals = 0, children = 0; // T-bound evaluations, children evaluated past the window rules
  long long children_full = 0;         // children whose residual was computed (not decided from the parent)
  double expand_ms = 0, dedupe_ms = 0, total_ms = 0;   // device times (profile) / host wall time
  long long expand_launches = 0;       // level-kernel launches (the denominator of per-launch figures)
  long long h2d_bytes = 0, d2h_bytes = 0;   // host<->device traffic of the call
  // --table K
  int table_k = 0, table_split[2] = {0, 0};
  bool table_proof = false, table_loaded = false, table_built = false;
  long long table_classes = 0;
  int table_levels = 0;
  double table_seconds = 0;
  std::string table_path;
  // --mitm
  bool mitm_join = false;              // the join ran (its "dir": "join" line)
  long long mitm_forward = 0, mitm_backward = 0, mitm_hash_matches = 0;
  double mitm_seconds = 0;
  int mitm_split[2] = {0, 0};          // [forward levels, backward levels] of the found circuit or of the proof
  bool mitm_found = false, mitm_proof = false;
  std::string error;
};

// Largest CX table and size of the device array used by eval_bounds_noalloc (see there).
constexpr int NOALLOC_MAX_CXTABLE = 4096;
constexpr size_t NOALLOC_SCRATCH_BYTES = 86016;

// Bounds of `count` residuals held in the caller's device memory (entries: count x N^2 x 4 int64 limbs, 16-byte
// aligned; exponents: count ints; bounds: count x 4 ints, 16-byte aligned), on the caller's stream, without any
// device allocation: the spec's tables are staged in a static device array shared by all calls (calls that overlap
// on the GPU race on it). Each call copies the tables from host memory and waits for the caller's stream before
// it queues the kernel. The first call on a device looks the array up (cudaGetSymbolAddress); make that first
// call before any stream capture. The address is kept per device index: it assumes the primary context and no
// device reset in between.
int eval_bounds_noalloc(const HostSpec &hs, int count, const int64_t *d_entries, const int *d_k, int *d_bounds,
                        void *stream, std::string &err);

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;
  // the plain search (no --mitm / --table); on_level is called after each completed level, in order
  int search(const HostSpec &hs, const Options &opt, const std::function<void(const LevelStats &)> &on_level,
             SearchResult &res);
  void *stream() const;
  // bounds of `count` caller-given residuals (entries count x N^2 x (a, b, c, d), exponents k): per residual
  // (T bound, CX bound, H structure, support) into out4
  int eval_bounds(const HostSpec &hs, int count, const int64_t *entries, const int *k, int *out4, std::string &err);
  // sustained int32 multiply-add throughput of this device (ops/s, a multiply-add counted as 2), measured by a
  // register-resident IMAD loop timed with CUDA events
  double int32_peak();
  // sorts n (key, value) pairs held in device memory by bits [lo, hi) of the key (stable radix sort of the dedupe,
  // in place, on the engine's stream; synchronises); the sort's device time in ms into *ms; returns 0, RC_USAGE (a
  // bit range that is not whole bytes) or RC_CUDA
  int sort_pairs(uint64_t *keys, uint32_t *vals, size_t n, int lo, int hi, float *ms, std::string &err);
  int device() const { return dev_; }
  // release the cached work buffers (frontiers, survivor records, sort scratch, tree); resident distance tables and
  // spec tables stay; returns the bytes released
  size_t trim();

 private:
  struct Impl;
  Impl *impl_;
  int dev_;
};

// Many searches of one qubit count advanced together, one level per step, in shared launches (continuous batching):
// jobs join at the next step after submit and leave when they finish; each job's per-level statistics, exit code
// and circuit are those of Engine::search on the same spec and options. Jobs the batched kernels do not cover (int64
// limbs, --no-dedupe, distance-table builds) run through Engine::search inside step().
struct BatchJob {
  bool done = false;
  SearchResult res;
  std::vector<LevelStats> levels;
  int joined_step = -1, finished_step = -1;
  bool plain = false;                  // ran through Engine::search
};

// Launch and chunking parameters of a batch step (the batched search's tunables): survivor records a chunk of jobs
// may plan for, expand blocks per SM (a persistent grid over a work counter) and deferred-T blocks per SM.
struct BatchTuning {
  size_t chunk_bytes = (size_t)8 << 30;
  int expand_blocks_per_sm = 16;
  int tbound_blocks_per_sm = 4;
};

class BatchSession {
 public:
  BatchSession(Engine &engine, int nq);
  ~BatchSession();
  BatchSession(const BatchSession &) = delete;
  BatchSession &operator=(const BatchSession &) = delete;
  int nq() const;
  // the job's id; it joins at the next step
  int submit(const HostSpec &hs, const Options &opt);
  // one level of every running job (admitting the submitted ones first); returns the jobs still running
  int step();
  int running() const;
  const BatchJob &job(int id) const;
  int jobs() const;
  long long frontier() const;          // nodes in the batch frontier
  long long launches() const;          // kernels launched by the session
  long long steps() const;
  size_t device_bytes() const;         // device memory held by the session's buffers
  // the frontier-memory estimate of the next step: the frontier plus room for every running job's children
  size_t projected_bytes() const;
  // device bytes a step may plan for (default: 80% of the free memory when the session was made); jobs beyond it
  // wait a step, their nodes carried over
  void set_memory_budget(size_t bytes);
  long long waits() const;             // job-steps spent waiting for memory
  void set_tuning(const BatchTuning &t);
  BatchTuning tuning() const;
  struct Impl;
 private:
  Impl *impl_;
};

// A project-written autotuner for batch sessions: every candidate tuning of a fixed search space is timed on the
// same probe jobs (one session on `engine`, warmed up by a first untimed run, the probe jobs submitted again for each
// trial; host wall time from the first submit to the last job's end), one parameter at a time from the defaults
// (coordinate descent: chunk budget, then expand blocks, then deferred-T blocks). Returns the fastest; trials (may
// be null) receives each timed run's tuning and seconds in the order tried.
struct TuneTrial { BatchTuning t; double seconds; };
BatchTuning autotune_batch(Engine &engine, int nq, const std::vector<const HostSpec *> &probe, const Options &opt,
                           std::vector<TuneTrial> *trials);

}  // namespace cz
