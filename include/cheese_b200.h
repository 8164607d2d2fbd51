/* cheese_b200: C ABI of the B200-native rebuild of cheese's gate-count search.
 *
 * The reference (jkhav/cheese) has no in-process API: its boundary is the process interface of build/cheese
 * (spec file in, one JSON line per level on stdout, exit code). This ABI exposes exactly that interface as calls
 * on plain pointers and sizes, so the drop-in binary (cheese_b200/bin/cheese) and any FFI caller (ctypes, cgo,
 * JNI ...) run the same code. Every entry point returns 0 or one of the reference's exit codes:
 *   CZ_CIRCUIT 0, CZ_PROOF 1, CZ_ERR_SPEC 2, CZ_ERR_USAGE 3, CZ_ERR_OVERFLOW 4, CZ_ERR_CUDA 5
 * (src/cheese.cu:1023-1026, 1153-1220, 1284-1285, 1848-1891). No C++ exception crosses the boundary.
 * Threading: one engine per host thread; an engine owns one device and one stream.
 */
#ifndef CHEESE_B200_H
#define CHEESE_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CZ_CIRCUIT 0
#define CZ_PROOF 1
#define CZ_ERR_SPEC 2
#define CZ_ERR_USAGE 3
#define CZ_ERR_OVERFLOW 4
#define CZ_ERR_CUDA 5
#define CZ_MAX_DEPTH 48

typedef struct cz_spec cz_spec;
typedef struct cz_engine cz_engine;

/* Parses a spec in the reference's text grammar (replaces read_spec, src/cheese.cu:1149-1226; the writer is
 * python/cheese/spec.py:356-415). Returns 0, CZ_ERR_SPEC (malformed: "not a spec", "unknown spec field X", ...)
 * or CZ_ERR_USAGE (qubit count not built: n outside 1..3). err receives a one-line message. */
int cz_spec_parse(const char *text, size_t len, cz_spec **out, char *err, size_t errlen);
void cz_spec_free(cz_spec *spec);
/* qubits, candidates and the spec's own budget ("depth" field) */
int cz_spec_info(const cz_spec *spec, int *n, int *gates, int *depth);
/* candidate name, e.g. "L_cx_0_1" (NULL when out of range) */
const char *cz_spec_gate_name(const cz_spec *spec, int g);
/* 1 when the spec is a state-target spec ("mode states": the circuit must map every listed input basis state to
 * the target's image, cheese.cu:451-583). The reference's GPU binary refuses these (src/cheese.cu:1871-1876) and
 * only its CPU build searches them; cz_search searches them on the GPU with the CPU build's bounds and results. */
int cz_spec_is_states(const cz_spec *spec);

/* Search engine on CUDA device `device` (replaces the device setup of run<NQ>, src/cheese.cu:1762-1792). */
int cz_engine_create(int device, cz_engine **out, char *err, size_t errlen);
void cz_engine_destroy(cz_engine *engine);
/* Release the engine's cached device work buffers (frontiers, survivor records, sort scratch, search tree), which it
 * otherwise keeps at their peak size for the next call; resident distance tables stay. Returns the bytes released.
 * No reference counterpart: the reference's processes run one search each and free everything at exit. */
int64_t cz_engine_trim(cz_engine *engine);

/* flags of the reference CLI (src/cheese.cu:1859-1868) */
typedef struct {
  int depth;        /* --depth D; -1: the spec's budget */
  int dedupe;       /* 1; 0: --no-dedupe */
  int sym;          /* 1; 0: --no-sym */
  int store64;      /* 0: int32 limbs promoted to int64 on demand; 1: int64 limbs throughout */
  int profile;      /* 1: device time of the level kernels (cz_result.expand_ms); 2: also of the dedupe (dedupe_ms).
                     * Each timed phase adds two events per level to the stream. */
  int table_k;      /* --table K: 0 none; K > 0 the distance table of the last K gates (cheese.cu:1431-1593) */
  const char *cache_dir;   /* distance-table cache directory ("build" by default; NULL: no cache) */
  int mitm;         /* --mitm: meet in the middle (cheese.cu:1595-1760); symmetry classes off, like the reference */
} cz_options;
void cz_options_default(cz_options *opt);

/* one JSON stats line of the reference (src/cheese.cu:1354-1356) */
typedef struct {
  int t;
  int64_t parents, prefixes, cut_w3, cut_lb, survivors, distinct;
  int proved_unsat;
  double seconds;
  int dir;          /* the line's "dir" field: 0 none; 1 "table" (distance-table build); 2 "fwd" / 3 "bwd" (--mitm) */
} cz_level_stats;
typedef void (*cz_level_fn)(void *user, const cz_level_stats *level);

typedef struct {
  int rc;                      /* the exit code the reference binary would return */
  int depth0;                  /* 1: the target is already the goal ({"found": 0, "circuit": []}) */
  int found_len;               /* rc 0: gates in the lexicographically first shortest circuit */
  int found[CZ_MAX_DEPTH];     /* candidate indices (names: cz_spec_gate_name) */
  int64_t n_found;             /* circuits of that length found at that level ("found" field) */
  int nsym;                    /* symmetry group size */
  int store64;                 /* 1: the run used int64 limbs */
  int levels;                  /* levels completed */
  int64_t prefixes;            /* sum of the per-level "prefixes" fields */
  int64_t kernel_launches;     /* device kernels launched by this call */
  int64_t t_evals;             /* Walsh-Hadamard T-bound evaluations */
  int64_t children;            /* children evaluated past the window rules */
  double expand_ms, dedupe_ms; /* device time per phase (profile >= 1, profile = 2) */
  double total_ms;             /* host wall time of the call */
  int64_t expand_launches;     /* launches of the level kernel */
  int64_t h2d_bytes, d2h_bytes;/* host<->device bytes moved by the call */
  int64_t children_full;       /* children whose residual was computed (the rest were decided from the parent) */
  /* --table K */
  int table_k;                 /* 0: not a table run */
  int table_split[2];          /* rc 0 through the table: [search levels, table gates] (the "table" field) */
  int table_proof;             /* rc 1 through the table: {"depth": D, "proved_unsat": true, "table": K} */
  int64_t table_classes;       /* classes in the table */
  int table_levels;
  int table_loaded, table_built;
  double table_seconds;
  char table_path[256];
  /* --mitm */
  int mitm_join;               /* 1: the join ran: {"dir": "join", "forward", "backward", "hash_matches", "seconds"} */
  int64_t mitm_forward, mitm_backward, mitm_hash_matches;
  double mitm_seconds;
  int mitm_split[2];           /* [forward levels, backward levels]: the "mitm" field of the circuit or proof line */
  int mitm_found, mitm_proof;  /* rc 0 / rc 1 through the join */
  char error[256];
} cz_result;

/* The search of `cheese SPEC [flags]` without --mitm (replaces run<NQ> + levels<NQ>, src/cheese.cu:1249-1377,
 * 1762-1849, and with opt->table_k the distance-table mode, :1431-1593, 1804-1838). Calls on_level after every
 * completed level, table-build levels included (may be NULL). */
int cz_search(cz_engine *engine, const cz_spec *spec, const cz_options *opt, cz_level_fn on_level, void *user,
              cz_result *out);

/* ---------------- batched searches (no counterpart in the reference: it runs one search per process) ----------------
 * A batch session advances many searches of one qubit count together, one level per step, in shared launches
 * (continuous batching): a submitted job joins at the next step, a finished job leaves. Every job's level lines,
 * exit code and circuit equal cz_search's on the same spec and options. */
typedef struct cz_batch cz_batch;
typedef struct {
  int nq, jobs, running;
  int64_t frontier;                 /* nodes in the shared frontier */
  int64_t steps, kernel_launches;
  int64_t device_bytes;             /* device memory held by the session */
  int64_t waits;                    /* job-steps a job waited for memory */
} cz_batch_info;
int cz_batch_create(cz_engine *engine, int nq, cz_batch **out);
void cz_batch_destroy(cz_batch *batch);
/* Device memory a step may plan for (default: 80% of the free memory when the session was made). When a step's
 * jobs would need more, the later jobs wait that step (their nodes carried over); results do not change. */
int cz_batch_set_memory(cz_batch *batch, double gb);
/* Queue a search (the spec's qubit count must be the session's): the job id (>= 0), or -(exit code). */
int cz_batch_submit(cz_batch *batch, const cz_spec *spec, const cz_options *opt);
/* One level of every running job (admitting the queued ones first); *running = jobs not finished yet. */
int cz_batch_step(cz_batch *batch, int *running);
/* the message of the last failed cz_batch_step ("" if none) */
const char *cz_batch_error(const cz_batch *batch);
int cz_batch_info_get(const cz_batch *batch, cz_batch_info *out);
/* The batch step's tunables: survivor-record bytes a chunk of jobs may plan for, expand blocks per SM, deferred
 * T-bound blocks per SM (defaults 8 GiB, 16, 4). Results do not depend on them, only the time. */
typedef struct {
  int64_t chunk_bytes;
  int expand_blocks_per_sm, tbound_blocks_per_sm;
  int trials;                       /* cz_batch_autotune: probe runs timed */
  double trial_seconds[16];         /* their host wall times, in the order tried */
  double best_seconds;              /* the chosen tuning's probe time */
} cz_batch_tuning;
int cz_batch_set_tuning(cz_batch *batch, const cz_batch_tuning *t);
/* The autotuner (no counterpart in the reference): times every candidate of a fixed search space on the probe jobs
 * (nprobe specs of qubit count nq, run to their end on one session of the engine, once untimed and then once per
 * candidate; chunk budget {8, 1, 2, 4}
 * GiB, expand blocks per SM {16, 4, 8, 32}, deferred-T blocks per SM {4, 1, 2, 8}, one parameter at a time from the
 * defaults) and writes the fastest to *out, with the probe times. Apply it with cz_batch_set_tuning. */
int cz_batch_autotune(cz_engine *engine, int nq, const cz_spec *const *probe, int nprobe, const cz_options *opt,
                      cz_batch_tuning *out);
/* 1 when the job has finished. */
int cz_batch_done(const cz_batch *batch, int job);
/* A finished job: its level lines through on_level (in order) and its result, as cz_search gives them. */
int cz_batch_result(const cz_batch *batch, int job, cz_level_fn on_level, void *user, cz_result *out);

/* ---------------- serving (no counterpart in the reference) ----------------
 * A persistent request server on one GPU. Requests of three kinds arrive at any time; each kind has a worker thread
 * with its own engine and stream, so their device work overlaps: gate-count searches are continuously batched
 * (admitted at the next level step while the batch's frontier-memory estimate leaves room under memory_gb),
 * T-count queries and Clifford-segment jobs use their resident tables. A request's output text is the stdout the
 * reference program prints for it ("seconds" fields 0.00). */
typedef struct cz_server cz_server;
#define CZ_REQ_GATES 0            /* text: a cheese spec; depth: budget (-1: the spec's) */
#define CZ_REQ_TCOUNT 1           /* text: a tcount-spec */
#define CZ_REQ_CLIFFORD 2         /* text: a cliffopt job */
#define CZ_REQ_GATES_QASM 3       /* text: an OpenQASM target, its spec generated in the server (cz_spec_generate);
                                     depth: budget (-1: the circuit's gate count) */
#define CZ_REQ_TCOUNT_QASM 4      /* text: an OpenQASM target, its tcount-spec generated in the server */
typedef struct {
  int device;
  double memory_gb;               /* device memory the gate-count batch may plan for */
  int max_jobs;                   /* gate-count jobs running at once */
  int tcount_table_k;             /* --table K of T-count queries */
  int beam;                       /* --beam of Clifford jobs */
  const char *cache_dir;          /* T-count table cache directory (NULL: none) */
} cz_server_options;
typedef struct {
  int rc, kind;
  double latency_s, queued_s;     /* submit -> done, submit -> started */
  int64_t gpu_work;               /* prefixes (gate count), children (T count), placements (Clifford) */
  size_t text_len;
  char error[256];
} cz_server_result;
typedef struct {
  int64_t submitted, completed, batch_steps, batch_admitted, batch_deferred, batch_peak_running, batch_peak_bytes;
  int64_t queued[3];
} cz_server_stats;
void cz_server_options_default(cz_server_options *opt);
int cz_server_create(const cz_server_options *opt, cz_server **out, char *err, size_t errlen);
void cz_server_destroy(cz_server *server);
/* the request id (>= 0), or -(exit code) */
int cz_server_submit(cz_server *server, int kind, const char *text, size_t len, int depth);
/* 1 done (out and text filled), 0 still running, < 0 unknown id */
int cz_server_poll(cz_server *server, int id, cz_server_result *out, char *text, size_t text_cap);
/* wait until `count` requests have completed since the server started: 0, or 1 on timeout */
int cz_server_wait(cz_server *server, long long count, double timeout_s);
int cz_server_stats_get(cz_server *server, cz_server_stats *out);
/* Submit request i at arrival_s[i] seconds after the call (host clock), then wait for all of them: ids[i] gets
 * each request id. 0, or 1 on timeout. */
int cz_server_replay(cz_server *server, int n, const int *kinds, const char *const *texts, const size_t *lens,
                     const int *depths, const double *arrival_s, double timeout_s, int *ids);

/* Convenience for FFI callers that hold the spec as text: parse + search in one call. */
int cz_search_text(cz_engine *engine, const char *spec_text, size_t len, const cz_options *opt, cz_level_fn on_level,
                   void *user, cz_result *out);

/* Lower bounds of `count` residual matrices under the spec's cuts and CX table, computed by the same device code
 * as the search: entries = count x N^2 x (a, b, c, d) limbs (value (a + b w + c w^2 + d w^3) / sqrt2^k), k = their
 * exponents; bounds = count x 4 ints (T bound = PTM sde, CX bound, H structure 0/2, support; the last two are -1
 * when the residual is the identity, where the search stops before the bounds). These are the
 * reference's ptm_wht, cx_bound, h_struct and support (src/cheese.cu:305-338, 585-597, 429-449). A state-target
 * spec is refused with CZ_ERR_USAGE (its search uses the row bounds of src/cheese.cu:451-583 instead). */
int cz_eval_bounds(cz_engine *engine, const cz_spec *spec, int count, const int64_t *entries, const int *k,
                   int *bounds);

/* No counterpart in the reference. The same bounds as cz_eval_bounds for callers that cannot allocate device
 * memory (code running under a custom or fixed-size allocator, inside a memory-capped service, or in a process
 * whose allocator is owned by another runtime): it calls no cudaMalloc / cudaFree and creates no engine. The
 * caller passes device buffers: d_entries (count x N^2 x 4 int64 limbs, 16-byte aligned), d_k (count ints) and
 * d_bounds (count x 4 ints, 16-byte aligned), and the stream to run on (NULL: the legacy default stream). Each
 * call copies the spec's tables from host memory into the array on that stream and waits for the stream
 * (cudaStreamSynchronize) before it queues the kernel, so the host blocks until the work queued earlier on the
 * stream has finished (with NULL: the work of every blocking stream); the results are in d_bounds once the
 * kernel, queued last, completes. The spec's tables (gate matrices, CX table, goal)
 * are staged in a static device array of CZ_NOALLOC_SCRATCH_BYTES that every GPU loading this library keeps
 * until the process exits; a spec whose CX table has more than CZ_NOALLOC_MAX_CXTABLE entries is refused with
 * CZ_ERR_USAGE, and so is a state-target spec (these are bounds of unitary residuals). All calls share that
 * array and each rewrites it in full, so calls that overlap on the GPU race.
 * The first call on a device looks the array up (cudaGetSymbolAddress) with that device current: make it before
 * any stream capture. The address is kept per device index for the life of the process; it assumes the device's
 * primary context (the runtime's) and no cudaDeviceReset in between. */
#define CZ_NOALLOC_SCRATCH_BYTES 86016
#define CZ_NOALLOC_MAX_CXTABLE 4096
int cz_eval_bounds_noalloc(const cz_spec *spec, int count, const int64_t *d_entries, const int *d_k, int *d_bounds,
                           void *stream, char *err, size_t errlen);

/* The CUDA stream (cudaStream_t) the engine launches on, for callers that order their own work or timing
 * events after the engine's kernels. */
void *cz_engine_stream(cz_engine *engine);

/* Sustained int32 multiply-add throughput of the engine's device in ops/s (a multiply-add counts as 2): a
 * register-resident IMAD loop timed with CUDA events. The denominator of the level kernel's roofline. */
int cz_int32_peak(cz_engine *engine, double *ops_per_s);

/* No counterpart in the reference (its dedupe sorts with Thrust, src/cheese.cu:1335-1343). The frontier dedupe's
 * stable LSD radix sort on caller-held device buffers: n (key, value) pairs sorted in place by bits [lo, hi) of the
 * key (hi - lo a multiple of 8, hi <= 64), equal keys in their input order, on the engine's stream (cz_engine_stream:
 * work that fills the buffers on another stream must be finished or ordered before the call); returns once sorted,
 * with the sort's device time in *ms (may be NULL). The engine holds the ping-pong buffers (12 n bytes) and the
 * scratch. For tests and measurement of the dedupe at scale. */
int cz_sort_pairs(cz_engine *engine, uint64_t *d_keys, uint32_t *d_vals, size_t n, int lo, int hi, float *ms);

/* ---------------- T-count (the reference's build/tcount, src/tcount.cu) ---------------- */
/* flags of `tcount TSPEC [--table K] [--max T]` (tcount.cu:452-465) and the table cache directory: the table of
 * (n, K) is cached in <cache_dir>/tcount-table-n<n>-k<K>.cz.bin; a reference-written
 * <cache_dir>/tcount-table-n<n>-k<K>.bin is read too (its tree is used, its keys recomputed). */
typedef struct {
  int table_k;            /* --table K (default 4) */
  int maxt;               /* --max T (default 16) */
  const char *cache_dir;  /* default "build"; NULL: no cache */
} cz_tcount_options;
void cz_tcount_options_default(cz_tcount_options *opt);

/* one JSON line of grow() (tcount.cu:391-392) */
typedef struct {
  int table;              /* 1: "dir": "table" (table build); 0: "dir": "search" */
  int t;
  int64_t parents, children, cosets, fresh;   /* fresh = the "new" field */
  double seconds;
} cz_tcount_level;
typedef void (*cz_tcount_level_fn)(void *user, const cz_tcount_level *level);

#define CZ_TCOUNT_MAXROT 64
typedef struct {
  int rc;                 /* 0 found, 1 none with T-count <= maxt, 2 spec, 3 usage, 4 overflow, 5 CUDA */
  int tcount;             /* rc 0: the optimal T-count (up to global phase) */
  int split_j, split_c;   /* levels from the search and from the table */
  int maxt;
  int nrot;               /* U = X_1 ... X_t C: rotation p = rot_p[i], X = R(P_p) (rot_inv 0) or R(P_p)^-1 (1) */
  int rot_p[CZ_TCOUNT_MAXROT], rot_inv[CZ_TCOUNT_MAXROT];
  int64_t table_cosets;   /* cosets in the table (all levels) */
  int table_levels;
  int table_loaded, table_built, table_resident;   /* where the table came from this call */
  double table_seconds, total_seconds;
  int64_t kernel_launches;
  char table_path[256];
  char error[256];
} cz_tcount_result;

/* Parse a tcount-spec without touching the device: 0 and the qubit count in *n, or 2 (not a tcount spec, unknown
 * field, short matrix: the exits of tcount.cu's read_spec, :434-450) / 3 (n outside 1..3) with the message. */
int cz_tspec_check(const char *tspec, size_t len, int *n, char *err, size_t errlen);

/* Optimal T-count of the unitary whose tcount-spec (the grammar of tcount.cu:434-450, written by
 * python/cheese/tcount.py:157-168) is given (replaces tcount.cu's main, :452-532). The engine keeps each (n, K)
 * table resident in device memory after its first use. */
int cz_tcount(cz_engine *engine, const char *tspec, size_t len, const cz_tcount_options *opt,
              cz_tcount_level_fn on_level, void *user, cz_tcount_result *out);

/* ---------------- RUS T-count (the reference's build/rus, src/rus.cu) ---------------- */
/* flags of `rus SPEC [--table K] [--max T]` (rus.cu:512-523) and the table cache directory: the table of K is cached
 * in <cache_dir>/rus-table-k<K>.cz.bin (this build's coset keys; the reference's rus-table-k<K>.bin is not read). */
typedef struct {
  int table_k;            /* --table K (default 8) */
  int maxt;               /* --max T (default 16) */
  const char *cache_dir;  /* default "build"; NULL: no cache */
} cz_rus_options;
void cz_rus_options_default(cz_rus_options *opt);

#define CZ_RUS_MAXPEEL 32
typedef struct {
  int rc;                 /* 0 found, 1 none with T-count <= maxt, 2 spec, 3 usage, 4 overflow, 5 CUDA */
  int tcount;             /* rc 0: the optimal RUS T-count */
  int split_j, split_c;   /* peels of the search node and of the table entry */
  int maxt;
  uint32_t root;          /* the root the search node descends from */
  int cliff;              /* the Clifford C (node = C x table entry): index into the spec's Clifford list */
  int fw[CZ_RUS_MAXPEEL], tb[CZ_RUS_MAXPEEL];   /* rotation indices 1..15 of the two peel sequences */
  int64_t table_cosets;   /* cosets in the table (all levels) */
  int table_levels;
  int table_loaded, table_built, table_resident;
  double table_seconds, total_seconds;
  int64_t kernel_launches;
  char table_path[256];
  char error[256];
} cz_rus_result;

/* Parse a rus-spec without touching the device: 0 and the number of roots in *nroot, or 2 (not a rus spec, unknown
 * field, incomplete spec, Clifford list not 11520 long or its generator images not unique: the exits of rus.cu's
 * read_spec and main, :486-510, 528-533) with the message. */
int cz_rspec_check(const char *rspec, size_t len, int *nroot, char *err, size_t errlen);

/* Optimal T-count of a two-qubit repeat-until-success circuit with measurement, from its rus-spec (written by
 * python/cheese/rus.py; replaces rus.cu's main, :512-587). Level lines go to on_level as cz_tcount_level (the same
 * fields). The engine keeps each table resident in device memory after its first use. */
int cz_rus(cz_engine *engine, const char *rspec, size_t len, const cz_rus_options *opt, cz_tcount_level_fn on_level,
           void *user, cz_rus_result *out);

/* ---------------- Clifford table (the reference's build/cliffopt, src/clifford.cu) ---------------- */
/* Tableau of an n <= 3 qubit Clifford up to phase, as the reference packs it (clifford.cu:16-19, 46-58): row
 * i < n is the image of X_i, row n + i the image of Z_i, each row (x bits | z bits << n | sign << 2n) of 2n + 1
 * bits, row i at bit i * (2n + 1). */
typedef struct {
  int n;
  int64_t order, elements;          /* group order up to phase; elements reached by the BFS (equal when correct) */
  int max_distance;
  int64_t per_distance[32];         /* elements at each minimal gate count (the "clifford gates d" lines) */
  int built;                        /* 1: built by this call; 0: resident from an earlier call */
  double seconds;
} cz_clifford_table_info;

/* The BFS distance table of the n-qubit Clifford group over H, S, Sdg, X, Z and CX (clifford.cu:247-276), built
 * once per engine and kept resident: 0, 3 (n not 1..3), 4 (group order mismatch), 5 (CUDA). */
int cz_clifford_table(cz_engine *engine, int n, cz_clifford_table_info *out, char *err, size_t errlen);
/* Minimal gate counts of tableaux (-1 for a word that is not a valid tableau). */
int cz_clifford_dist(cz_engine *engine, int n, const uint64_t *tableaux, size_t count, int *out);
/* An optimal word of each tableau (the read-back of clifford.cu:352-371): words = count x CZ_CLIFFORD_WORDMAX x
 * (kind, a, b), kinds 0..6 = h s sdg x z cx y, lens = gates per word. */
#define CZ_CLIFFORD_WORDMAX 32
int cz_clifford_words(cz_engine *engine, int n, const uint64_t *tableaux, size_t count, int *words, int *lens);
/* The group element of each index in [0, order): index -> element is a fixed bijection (uniform draws). */
int cz_clifford_element(cz_engine *engine, int n, const uint64_t *index, size_t count, uint64_t *tableaux);

/* Parse a cliffopt job (clifford.cu:213-238) on the host: 0, or 2 ("bad job file", "unknown Clifford gate X"). */
int cz_cliffjob_check(const char *job, size_t len, int *n, int *t_gates, char *err, size_t errlen);

/* one "T gate j: P placements x beam, best partial C" line (clifford.cu:330) */
typedef void (*cz_cliffopt_step_fn)(void *user, int tgate, int64_t placements, int best_partial);
typedef struct {
  int rc;                           /* 0, 2 job, 3 usage, 4 table / reconstruction, 5 CUDA */
  int clifford_gates, clifford_gates_before, t_gates;
  double seconds;
  cz_clifford_table_info table;
  int64_t kernel_launches;
  size_t text_len;                  /* length of the gate lines (text is truncated to text_cap - 1) */
  char error[256];
} cz_cliffopt_result;
/* `cliffopt JOB --beam B` (replaces clifford.cu's main, :240-384): fewer Clifford gates around the job's T gates.
 * text receives the output lines after the JSON line: one gate per line, T gates as "t q" / "tdg q". */
int cz_cliffopt(cz_engine *engine, const char *job, size_t len, int beam, cz_cliffopt_step_fn on_step, void *user,
                char *text, size_t text_cap, cz_cliffopt_result *out);

/* ---------------- spec generation (the reference's python/cheese/spec.py and tcount.py writers) ---------------- */
typedef struct {
  int n;                 /* qubits */
  int gates;             /* gates of the target circuit */
  int candidates;        /* candidate gates of the spec */
  int w2_pairs, w3_triples;
} cz_specgen_info;
/* The gate-count spec of a target circuit with budget `depth`, as `python -m cheese.spec TARGET.qasm DEPTH
 * [--no-w3]` writes it (spec.py:127-350, unitary targets): Clifford+T plus the circuit's own gates as candidates,
 * the W2/W3 window rules, the target unitary, the cuts and the CX table. The W3 triples are listed by (first,
 * second) gate and then by third gate (the reference lists the third gates of one (first, second) in Python set
 * order); the set of triples is the same. The per-gate-set parts are cached across calls (thread safe).
 * The circuit is either QASM text (the reference's parse_qasm subset, spec.py:113-123: qreg/qubit declaration,
 * one known gate per statement) or, with qasm NULL, n qubits and ngates gates: names[i] with qubits
 * qubits[3 i .. 3 i + arity). The text goes to out (cap bytes, NUL-terminated); out_len receives the length it
 * needs without the NUL. Returns 0, 2 (bad circuit: err), or 3 (cap too small: nothing written).
 * No compiled counterpart in the reference (its generator is Python). */
int cz_spec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                     const int *qubits, int depth, int no_w3, char *out, size_t cap, size_t *out_len,
                     cz_specgen_info *info, char *err, size_t errlen);
/* The state-target spec of a target circuit, as `python -m cheese.spec TARGET.qasm DEPTH --inputs a,b,..` (or
 * `--ancilla q ..`: every basis state with those qubits 0) writes it (spec.py:229-325, 356-424): "mode states", the
 * start rows e_x and the goal rows U e_x of the ninputs input basis states (bit q of x = qubit q), and per goal row
 * its sde, stabilizer nullity and Schmidt ranks across the cuts. Other arguments and returns as cz_spec_generate;
 * 2 also for an input out of range or more inputs than basis states. */
int cz_spec_generate_states(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                            const int *qubits, int depth, int no_w3, const int *inputs, int ninputs, char *out,
                            size_t cap, size_t *out_len, cz_specgen_info *info, char *err, size_t errlen);
/* The T-count spec of a target circuit, as `python -m cheese.tcount spec TARGET.qasm` writes it (tcount.py:79-168):
 * the channel representation and the Pauli rotation tables. Arguments and returns as cz_spec_generate. */
int cz_tspec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                      const int *qubits, char *out, size_t cap, size_t *out_len, char *err, size_t errlen);

/* The rus-spec of a two-qubit repeat-until-success circuit (q0 ancilla, measured; q1 data), as `python -m cheese.rus
 * spec TARGET.qasm [--outcome K]` writes it (rus.py:214-303): the table root, the roots (every valid isometry for
 * the success branch up to left Cliffords), the rotation tables and the 11520 Cliffords. outcome: the success
 * outcome, or -1 for the QASM text's "success outcome K" comment, else the branch not proportional to a Clifford.
 * info (may be NULL): outcome, roots, p = (A, B, m) with Pr[success] = (A + B sqrt2) / 2^m, rescalings, failure
 * amplitudes. Circuit input, out, out_len and returns as cz_spec_generate. */
typedef struct {
  int outcome, roots, rescalings, failure_amplitudes;
  int64_t p[3];
} cz_rspec_info;
int cz_rspec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                      const int *qubits, int outcome, char *out, size_t cap, size_t *out_len, cz_rspec_info *info,
                      char *err, size_t errlen);

/* The library version string and the CUDA architecture it was compiled for ("sm_100a"). */
const char *cz_version(void);

#ifdef __cplusplus
}
#endif
#endif
