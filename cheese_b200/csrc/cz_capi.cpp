// C ABI over the C++ engine: no exception crosses it, every call returns 0 or a reference exit code.
#include <cuda_runtime.h>

#include <cstdio>
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cz_capi_internal.h"
#include "cz_specgen.h"

namespace {
void put_err(char *err, size_t n, const std::string &m) {
  if (err && n) { std::snprintf(err, n, "%s", m.c_str()); }
}
}  // namespace

extern "C" {

int cz_spec_parse(const char *text, size_t len, cz_spec **out, char *err, size_t errlen) {
  if (!out) return CZ_ERR_USAGE;
  *out = nullptr;
  try {
    cz_spec *s = new cz_spec;
    std::string e;
    const int rc = cz::parse_spec(text ? text : "", text ? len : 0, s->hs, e);
    if (rc) { put_err(err, errlen, e); delete s; return rc; }
    *out = s;
    return 0;
  } catch (const std::exception &ex) {
    put_err(err, errlen, ex.what());
    return CZ_ERR_SPEC;
  }
}

void cz_spec_free(cz_spec *spec) { delete spec; }

int cz_spec_info(const cz_spec *spec, int *n, int *gates, int *depth) {
  if (!spec) return CZ_ERR_USAGE;
  if (n) *n = spec->hs.n;
  if (gates) *gates = spec->hs.G;
  if (depth) *depth = spec->hs.depth;
  return 0;
}

const char *cz_spec_gate_name(const cz_spec *spec, int g) {
  if (!spec || g < 0 || g >= spec->hs.G) return nullptr;
  return spec->hs.names[g].c_str();
}

int cz_spec_is_states(const cz_spec *spec) { return spec && spec->hs.states; }

int cz_engine_create(int device, cz_engine **out, char *err, size_t errlen) {
  if (!out) return CZ_ERR_USAGE;
  *out = nullptr;
  int ndev = 0;
  const cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || device < 0 || device >= ndev) {
    put_err(err, errlen, std::string("no CUDA device ") + std::to_string(device) + ": " +
                             (ce != cudaSuccess ? cudaGetErrorString(ce) : "out of range"));
    return CZ_ERR_CUDA;
  }
  try {
    cz_engine *e = new cz_engine{new cz::Engine(device), nullptr, nullptr, nullptr};
    *out = e;
    return 0;
  } catch (const std::exception &ex) {
    put_err(err, errlen, ex.what());
    return CZ_ERR_CUDA;
  }
}

int64_t cz_engine_trim(cz_engine *engine) {
  if (!engine) return 0;
  size_t n = engine->e->trim();
  if (engine->tc) n += cz::tcount_context_trim(engine->tc);
  if (engine->cl) n += cz::clifford_context_trim(engine->cl);
  if (engine->ru) n += cz::rus_context_trim(engine->ru);
  return (int64_t)n;
}

void cz_engine_destroy(cz_engine *engine) {
  if (!engine) return;
  if (engine->tc) cz::tcount_context_destroy(engine->tc);
  if (engine->cl) cz::clifford_context_destroy(engine->cl);
  if (engine->ru) cz::rus_context_destroy(engine->ru);
  delete engine->e;
  delete engine;
}

void cz_options_default(cz_options *opt) {
  if (!opt) return;
  opt->depth = -1; opt->dedupe = 1; opt->sym = 1; opt->store64 = 0; opt->profile = 0; opt->table_k = 0;
  opt->cache_dir = "build"; opt->mitm = 0;
}

namespace {
void fill_result(const cz::SearchResult &r, cz_result *out) {
  out->rc = r.rc;
  out->depth0 = r.depth0;
  out->found_len = (int)r.circuit.size();
  for (size_t i = 0; i < r.circuit.size() && i < CZ_MAX_DEPTH; i++) out->found[i] = r.circuit[i];
  out->n_found = r.n_found;
  out->nsym = r.nsym;
  out->store64 = r.store64;
  out->levels = r.levels;
  out->prefixes = r.prefixes;
  out->kernel_launches = r.launches;
  out->t_evals = r.t_evals;
  out->children = r.children;
  out->expand_ms = r.expand_ms;
  out->dedupe_ms = r.dedupe_ms;
  out->total_ms = r.total_ms;
  out->expand_launches = r.expand_launches;
  out->h2d_bytes = r.h2d_bytes;
  out->d2h_bytes = r.d2h_bytes;
  out->children_full = r.children_full;
  out->table_k = r.table_k;
  out->table_split[0] = r.table_split[0];
  out->table_split[1] = r.table_split[1];
  out->table_proof = r.table_proof;
  out->table_classes = r.table_classes;
  out->table_levels = r.table_levels;
  out->table_loaded = r.table_loaded;
  out->table_built = r.table_built;
  out->table_seconds = r.table_seconds;
  put_err(out->table_path, sizeof out->table_path, r.table_path);
  out->mitm_join = r.mitm_join;
  out->mitm_forward = r.mitm_forward;
  out->mitm_backward = r.mitm_backward;
  out->mitm_hash_matches = r.mitm_hash_matches;
  out->mitm_seconds = r.mitm_seconds;
  out->mitm_split[0] = r.mitm_split[0];
  out->mitm_split[1] = r.mitm_split[1];
  out->mitm_found = r.mitm_found;
  out->mitm_proof = r.mitm_proof;
  put_err(out->error, sizeof out->error, r.error);
}

cz_level_stats level_stats(const cz::LevelStats &L) {
  cz_level_stats s;
  s.t = L.t; s.parents = L.parents; s.prefixes = L.prefixes; s.cut_w3 = L.cut_w3; s.cut_lb = L.cut_lb;
  s.survivors = L.survivors; s.distinct = L.distinct; s.proved_unsat = L.proved_unsat; s.seconds = L.seconds;
  s.dir = L.dir;
  return s;
}
}  // namespace

int cz_search(cz_engine *engine, const cz_spec *spec, const cz_options *opt, cz_level_fn on_level, void *user,
              cz_result *out) {
  if (!engine || !spec || !out) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  cz_options o;
  cz_options_default(&o);
  if (opt) o = *opt;
  const cz::HostSpec &hs = spec->hs;
  const int depth = o.depth >= 0 ? o.depth : hs.depth;
  if (depth > CZ_MAX_DEPTH) {
    put_err(out->error, sizeof out->error, "depth > " + std::to_string(CZ_MAX_DEPTH));
    out->rc = CZ_ERR_USAGE;
    return CZ_ERR_USAGE;
  }
  cz::Options eo;
  eo.depth = depth; eo.dedupe = o.dedupe != 0; eo.sym = o.sym != 0; eo.store64 = o.store64; eo.profile = o.profile < 0 ? 0 : o.profile;
  if (o.table_k < 0 || o.table_k > CZ_MAX_DEPTH) {
    put_err(out->error, sizeof out->error, "table depth out of range");
    out->rc = CZ_ERR_USAGE;
    return CZ_ERR_USAGE;
  }
  eo.table_k = o.table_k;
  eo.cache_dir = o.cache_dir ? o.cache_dir : "";
  eo.mitm = o.mitm != 0;
  cz::SearchResult r;
  int rc;
  try {
    rc = engine->e->search(hs, eo, [&](const cz::LevelStats &L) {
      if (!on_level) return;
      const cz_level_stats s = level_stats(L);
      on_level(user, &s);
    }, r);
  } catch (const std::bad_alloc &) {
    r.error = "host out of memory";
    rc = CZ_ERR_CUDA;
  } catch (const std::exception &ex) {
    r.error = ex.what();
    rc = CZ_ERR_CUDA;
  }
  r.rc = rc;
  fill_result(r, out);
  return rc;
}


int cz_batch_create(cz_engine *engine, int nq, cz_batch **out) {
  if (!engine || !out || nq < 1 || nq > 3) return CZ_ERR_USAGE;
  *out = nullptr;
  try {
    *out = new cz_batch{new cz::BatchSession(*engine->e, nq), std::string()};
    return 0;
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

void cz_batch_destroy(cz_batch *batch) {
  if (!batch) return;
  delete batch->b;
  delete batch;
}

int cz_batch_set_memory(cz_batch *batch, double gb) {
  if (!batch || !(gb > 0)) return CZ_ERR_USAGE;
  batch->b->set_memory_budget((size_t)(gb * 1e9));
  return 0;
}

int cz_batch_submit(cz_batch *batch, const cz_spec *spec, const cz_options *opt) {
  if (!batch || !spec) return -CZ_ERR_USAGE;
  const cz::HostSpec &hs = spec->hs;
  if (hs.states || hs.n != batch->b->nq()) return -CZ_ERR_USAGE;
  cz_options o;
  cz_options_default(&o);
  if (opt) o = *opt;
  const int depth = o.depth >= 0 ? o.depth : hs.depth;
  if (depth > CZ_MAX_DEPTH) return -CZ_ERR_USAGE;
  cz::Options eo;
  eo.depth = depth; eo.dedupe = o.dedupe != 0; eo.sym = o.sym != 0; eo.store64 = o.store64; eo.profile = false;
  try {
    return batch->b->submit(hs, eo);
  } catch (const std::exception &) {
    return -CZ_ERR_CUDA;
  }
}

int cz_batch_step(cz_batch *batch, int *running) {
  if (!batch) return CZ_ERR_USAGE;
  try {
    const int r = batch->b->step();
    if (running) *running = r;
    return 0;
  } catch (const std::exception &ex) {
    batch->err = ex.what();
    return CZ_ERR_CUDA;
  }
}

const char *cz_batch_error(const cz_batch *batch) { return batch ? batch->err.c_str() : "";
}

int cz_batch_set_tuning(cz_batch *batch, const cz_batch_tuning *t) {
  if (!batch || !t || t->chunk_bytes <= 0 || t->expand_blocks_per_sm < 1 || t->tbound_blocks_per_sm < 1 ||
      t->expand_blocks_per_sm > 64 || t->tbound_blocks_per_sm > 64)
    return CZ_ERR_USAGE;
  cz::BatchTuning bt;
  bt.chunk_bytes = (size_t)t->chunk_bytes;
  bt.expand_blocks_per_sm = t->expand_blocks_per_sm;
  bt.tbound_blocks_per_sm = t->tbound_blocks_per_sm;
  batch->b->set_tuning(bt);
  return 0;
}

int cz_batch_autotune(cz_engine *engine, int nq, const cz_spec *const *probe, int nprobe, const cz_options *opt,
                      cz_batch_tuning *out) {
  if (!engine || !out || nq < 1 || nq > 3 || nprobe < 1 || !probe) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  cz_options o;
  cz_options_default(&o);
  if (opt) o = *opt;
  cz::Options eo;
  eo.depth = o.depth; eo.dedupe = o.dedupe != 0; eo.sym = o.sym != 0; eo.store64 = o.store64; eo.profile = false;
  std::vector<const cz::HostSpec *> hs;
  for (int i = 0; i < nprobe; i++) {
    if (!probe[i] || probe[i]->hs.n != nq || probe[i]->hs.states) return CZ_ERR_USAGE;
    hs.push_back(&probe[i]->hs);
  }
  try {
    std::vector<cz::TuneTrial> trials;
    const cz::BatchTuning best = cz::autotune_batch(*engine->e, nq, hs, eo, &trials);
    out->chunk_bytes = (int64_t)best.chunk_bytes;
    out->expand_blocks_per_sm = best.expand_blocks_per_sm;
    out->tbound_blocks_per_sm = best.tbound_blocks_per_sm;
    out->trials = (int)std::min<size_t>(trials.size(), 16);
    out->best_seconds = 1e30;
    for (size_t i = 0; i < trials.size(); i++) {
      if (i < 16) out->trial_seconds[i] = trials[i].seconds;
      const cz::BatchTuning &t = trials[i].t;
      if (t.chunk_bytes == best.chunk_bytes && t.expand_blocks_per_sm == best.expand_blocks_per_sm &&
          t.tbound_blocks_per_sm == best.tbound_blocks_per_sm)
        out->best_seconds = std::min(out->best_seconds, trials[i].seconds);
    }
    return 0;
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

int cz_batch_info_get(const cz_batch *batch, cz_batch_info *out) {
  if (!batch || !out) return CZ_ERR_USAGE;
  out->nq = batch->b->nq();
  out->jobs = batch->b->jobs();
  out->running = batch->b->running();
  out->frontier = batch->b->frontier();
  out->steps = batch->b->steps();
  out->kernel_launches = batch->b->launches();
  out->device_bytes = (int64_t)batch->b->device_bytes();
  out->waits = batch->b->waits();
  return 0;
}

int cz_batch_done(const cz_batch *batch, int job) {
  if (!batch || job < 0 || job >= batch->b->jobs()) return 0;
  return batch->b->job(job).done ? 1 : 0;
}

int cz_batch_result(const cz_batch *batch, int job, cz_level_fn on_level, void *user, cz_result *out) {
  if (!batch || !out || job < 0 || job >= batch->b->jobs()) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  const cz::BatchJob &j = batch->b->job(job);
  if (!j.done) return CZ_ERR_USAGE;
  for (const cz::LevelStats &L : j.levels) {
    if (!on_level) break;
    const cz_level_stats s = level_stats(L);
    on_level(user, &s);
  }
  fill_result(j.res, out);
  return 0;
}

int cz_search_text(cz_engine *engine, const char *spec_text, size_t len, const cz_options *opt, cz_level_fn on_level,
                   void *user, cz_result *out) {
  if (!out) return CZ_ERR_USAGE;
  cz_spec *s = nullptr;
  char err[256] = {0};
  const int prc = cz_spec_parse(spec_text, len, &s, err, sizeof err);
  if (prc) {
    std::memset(out, 0, sizeof *out);
    out->rc = prc;
    std::snprintf(out->error, sizeof out->error, "%s", err);
    return prc;
  }
  const int rc = cz_search(engine, s, opt, on_level, user, out);
  cz_spec_free(s);
  return rc;
}

int cz_eval_bounds(cz_engine *engine, const cz_spec *spec, int count, const int64_t *entries, const int *k,
                   int *bounds) {
  if (!engine || !spec || count < 0 || (count && (!entries || !k || !bounds))) return CZ_ERR_USAGE;
  if (spec->hs.states) return CZ_ERR_USAGE;   // the bounds are those of unitary residuals (like --mitm)
  if (!count) return 0;
  std::string err;
  try {
    return engine->e->eval_bounds(spec->hs, count, entries, k, bounds, err);
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

int cz_eval_bounds_noalloc(const cz_spec *spec, int count, const int64_t *d_entries, const int *d_k, int *d_bounds,
                           void *stream, char *err, size_t errlen) {
  static_assert(CZ_NOALLOC_SCRATCH_BYTES == cz::NOALLOC_SCRATCH_BYTES, "header and library disagree");
  static_assert(CZ_NOALLOC_MAX_CXTABLE == cz::NOALLOC_MAX_CXTABLE, "header and library disagree");
  if (!spec) { put_err(err, errlen, "null spec"); return CZ_ERR_USAGE; }
  if (spec->hs.states) {
    put_err(err, errlen, "state-target spec: these bounds are defined for unitary residuals only");
    return CZ_ERR_USAGE;
  }
  std::string e;
  int rc;
  try {
    rc = cz::eval_bounds_noalloc(spec->hs, count, d_entries, d_k, d_bounds, stream, e);
  } catch (const std::exception &ex) {
    e = ex.what();
    rc = CZ_ERR_CUDA;
  }
  put_err(err, errlen, e);
  return rc;
}

void *cz_engine_stream(cz_engine *engine) { return engine ? engine->e->stream() : nullptr; }

int cz_sort_pairs(cz_engine *engine, uint64_t *d_keys, uint32_t *d_vals, size_t n, int lo, int hi, float *ms) {
  if (!engine || (n && (!d_keys || !d_vals))) return CZ_ERR_USAGE;
  if (n < 2) { if (ms) *ms = 0; return 0; }
  std::string err;
  try {
    return engine->e->sort_pairs(d_keys, d_vals, n, lo, hi, ms, err);
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

int cz_int32_peak(cz_engine *engine, double *ops_per_s) {
  if (!engine || !ops_per_s) return CZ_ERR_USAGE;
  try {
    *ops_per_s = engine->e->int32_peak();
    return 0;
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

void cz_tcount_options_default(cz_tcount_options *opt) {
  if (!opt) return;
  opt->table_k = 4; opt->maxt = 16; opt->cache_dir = "build";
}

int cz_tspec_check(const char *tspec, size_t len, int *n, char *err, size_t errlen) {
  cz::TSpec sp;
  std::string msg;
  const int rc = cz::parse_tspec(tspec ? tspec : "", tspec ? len : 0, sp, msg);
  if (n) *n = rc ? 0 : sp.n;
  if (err && errlen) put_err(err, errlen, msg);
  return rc;
}

int cz_tcount(cz_engine *engine, const char *tspec, size_t len, const cz_tcount_options *opt,
              cz_tcount_level_fn on_level, void *user, cz_tcount_result *out) {
  if (!engine || !out) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  cz_tcount_options o;
  cz_tcount_options_default(&o);
  if (opt) o = *opt;
  cz::TSpec sp;
  std::string err;
  int rc = cz::parse_tspec(tspec ? tspec : "", tspec ? len : 0, sp, err);
  if (rc) { out->rc = rc; put_err(out->error, sizeof out->error, err); return rc; }
  if (o.table_k < 0 || o.table_k > 32 || o.maxt < 0 || o.maxt > 63) {
    out->rc = CZ_ERR_USAGE;
    put_err(out->error, sizeof out->error, "table depth or max T-count out of range");
    return CZ_ERR_USAGE;
  }
  cz::TcOptions to;
  to.table_k = o.table_k; to.maxt = o.maxt;
  to.use_cache = o.cache_dir != nullptr;
  if (o.cache_dir) to.cache_dir = o.cache_dir;
  cz::TcResult r;
  try {
    if (!engine->tc) engine->tc = cz::tcount_context_create(engine->e->device(), engine->e->stream());
    rc = cz::tcount_run(engine->tc, sp, to, [&](const cz::TcLevel &L) {
      if (!on_level) return;
      cz_tcount_level l;
      l.table = L.table; l.t = L.t; l.parents = L.parents; l.children = L.children; l.cosets = L.cosets;
      l.fresh = L.fresh; l.seconds = L.seconds;
      on_level(user, &l);
    }, r);
  } catch (const std::exception &ex) {
    r.error = ex.what();
    rc = CZ_ERR_CUDA;
  }
  out->rc = rc;
  out->tcount = r.tcount; out->split_j = r.split_j; out->split_c = r.split_c; out->maxt = r.maxt;
  out->nrot = (int)std::min<size_t>(r.rotations.size(), CZ_TCOUNT_MAXROT);
  for (int i = 0; i < out->nrot; i++) { out->rot_p[i] = r.rotations[i].first; out->rot_inv[i] = r.rotations[i].second; }
  out->table_cosets = r.table_cosets; out->table_levels = r.table_levels;
  out->table_loaded = r.table_loaded; out->table_built = r.table_built; out->table_resident = r.table_resident;
  out->table_seconds = r.table_seconds; out->total_seconds = r.total_seconds; out->kernel_launches = r.launches;
  put_err(out->table_path, sizeof out->table_path, r.table_path);
  put_err(out->error, sizeof out->error, r.error);
  return rc;
}

void cz_rus_options_default(cz_rus_options *opt) {
  if (!opt) return;
  opt->table_k = 8; opt->maxt = 16; opt->cache_dir = "build";
}

int cz_rspec_check(const char *rspec, size_t len, int *nroot, char *err, size_t errlen) {
  cz::RSpec sp;
  std::string msg;
  const int rc = cz::parse_rspec(rspec ? rspec : "", rspec ? len : 0, sp, msg);
  if (nroot) *nroot = rc ? 0 : sp.nroot;
  if (err && errlen) put_err(err, errlen, msg);
  return rc;
}

int cz_rus(cz_engine *engine, const char *rspec, size_t len, const cz_rus_options *opt, cz_tcount_level_fn on_level,
           void *user, cz_rus_result *out) {
  if (!engine || !out) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  cz_rus_options o;
  cz_rus_options_default(&o);
  if (opt) o = *opt;
  cz::RSpec sp;
  std::string err;
  int rc = cz::parse_rspec(rspec ? rspec : "", rspec ? len : 0, sp, err);
  if (rc) { out->rc = rc; put_err(out->error, sizeof out->error, err); return rc; }
  if (o.table_k < 0 || o.table_k > CZ_RUS_MAXPEEL || o.maxt > 63) {
    out->rc = CZ_ERR_USAGE;
    put_err(out->error, sizeof out->error, "table depth or max T-count out of range");
    return CZ_ERR_USAGE;
  }
  cz::RusOptions ro;
  ro.table_k = o.table_k; ro.maxt = o.maxt;
  ro.use_cache = o.cache_dir != nullptr;
  if (o.cache_dir) ro.cache_dir = o.cache_dir;
  cz::RusResult r;
  try {
    if (!engine->ru) engine->ru = cz::rus_context_create(engine->e->device(), engine->e->stream());
    rc = cz::rus_run(engine->ru, sp, ro, [&](const cz::RusLevel &L) {
      if (!on_level) return;
      cz_tcount_level l;
      l.table = L.table; l.t = L.t; l.parents = L.parents; l.children = L.children; l.cosets = L.cosets;
      l.fresh = L.fresh; l.seconds = L.seconds;
      on_level(user, &l);
    }, r);
  } catch (const std::exception &ex) {
    r.error = ex.what();
    rc = CZ_ERR_CUDA;
  }
  out->rc = rc;
  out->tcount = r.tcount; out->split_j = r.split_j; out->split_c = r.split_c; out->maxt = r.maxt;
  out->root = r.root; out->cliff = r.cliff;
  for (size_t i = 0; i < r.fw.size() && i < CZ_RUS_MAXPEEL; i++) out->fw[i] = r.fw[i];
  for (size_t i = 0; i < r.tb.size() && i < CZ_RUS_MAXPEEL; i++) out->tb[i] = r.tb[i];
  out->table_cosets = r.table_cosets; out->table_levels = r.table_levels;
  out->table_loaded = r.table_loaded; out->table_built = r.table_built; out->table_resident = r.table_resident;
  out->table_seconds = r.table_seconds; out->total_seconds = r.total_seconds; out->kernel_launches = r.launches;
  put_err(out->table_path, sizeof out->table_path, r.table_path);
  put_err(out->error, sizeof out->error, r.error);
  return rc;
}

int cz_cliffjob_check(const char *job, size_t len, int *n, int *t_gates, char *err, size_t errlen) {
  cz::CliffJob J;
  std::string msg;
  const int rc = cz::parse_cliff_job(job ? job : "", job ? len : 0, J, msg);
  if (n) *n = rc ? 0 : J.n;
  if (t_gates) *t_gates = rc ? 0 : (int)J.tq.size();
  if (err && errlen) put_err(err, errlen, msg);
  return rc;
}

namespace {
void fill_table_info(const cz::CliffTableInfo &i, cz_clifford_table_info *o) {
  std::memset(o, 0, sizeof *o);
  o->n = i.n; o->order = i.order; o->elements = i.elements; o->max_distance = i.max_distance;
  for (int d = 0; d < 32; d++) o->per_distance[d] = i.per_distance[d];
  o->built = i.built; o->seconds = i.seconds;
}
cz::CliffordContext *cliff_ctx(cz_engine *engine) {
  if (!engine->cl) engine->cl = cz::clifford_context_create(engine->e->device(), engine->e->stream());
  return engine->cl;
}
}  // namespace

int cz_clifford_table(cz_engine *engine, int n, cz_clifford_table_info *out, char *err, size_t errlen) {
  if (!engine) return CZ_ERR_USAGE;
  try {
    cz::CliffTableInfo info;
    std::string e;
    const int rc = cz::clifford_table(cliff_ctx(engine), n, info, e);
    if (rc) { put_err(err, errlen, e); return rc; }
    if (out) fill_table_info(info, out);
    return 0;
  } catch (const std::exception &ex) {
    put_err(err, errlen, ex.what());
    return CZ_ERR_CUDA;
  }
}

int cz_cliffopt(cz_engine *engine, const char *job, size_t len, int beam, cz_cliffopt_step_fn on_step, void *user,
                char *text, size_t text_cap, cz_cliffopt_result *out) {
  if (!engine || !out) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  cz::CliffJob J;
  std::string err;
  int rc = cz::parse_cliff_job(job ? job : "", job ? len : 0, J, err);
  if (rc) { out->rc = rc; put_err(out->error, sizeof out->error, err); return rc; }
  cz::CliffOptResult r;
  try {
    rc = cz::cliffopt_run(cliff_ctx(engine), J, beam, [&](int j, const cz::CliffStep &st) {
      if (on_step) on_step(user, j, st.placements, st.best_partial);
    }, r);
  } catch (const std::exception &ex) {
    r.error = ex.what();
    rc = CZ_ERR_CUDA;
  }
  out->rc = rc;
  out->clifford_gates = r.clifford_gates; out->clifford_gates_before = r.before; out->t_gates = r.t_gates;
  out->seconds = r.seconds;
  fill_table_info(r.table, &out->table);
  out->kernel_launches = r.launches;
  out->text_len = r.text.size();
  if (text && text_cap) {
    const size_t m = std::min(text_cap - 1, r.text.size());
    std::memcpy(text, r.text.data(), m);
    text[m] = 0;
  }
  put_err(out->error, sizeof out->error, r.error);
  return rc;
}

int cz_clifford_dist(cz_engine *engine, int n, const uint64_t *tableaux, size_t count, int *out) {
  if (!engine || (count && (!tableaux || !out))) return CZ_ERR_USAGE;
  try {
    std::string e;
    return cz::clifford_dist(cliff_ctx(engine), n, tableaux, count, out, e);
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

int cz_clifford_words(cz_engine *engine, int n, const uint64_t *tableaux, size_t count, int *words, int *lens) {
  if (!engine || (count && (!tableaux || !words || !lens))) return CZ_ERR_USAGE;
  try {
    std::string e;
    std::vector<std::vector<int>> w;
    const int rc = cz::clifford_words(cliff_ctx(engine), n, tableaux, count, w, e);
    if (rc) return rc;
    for (size_t i = 0; i < count; i++) {
      lens[i] = (int)(w[i].size() / 3);
      for (size_t j = 0; j < w[i].size() && j < (size_t)CZ_CLIFFORD_WORDMAX * 3; j++) words[i * CZ_CLIFFORD_WORDMAX * 3 + j] = w[i][j];
    }
    return 0;
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

int cz_clifford_element(cz_engine *engine, int n, const uint64_t *index, size_t count, uint64_t *tableaux) {
  if (!engine || (count && (!index || !tableaux))) return CZ_ERR_USAGE;
  try {
    std::string e;
    return cz::clifford_element(cliff_ctx(engine), n, index, count, tableaux, e);
  } catch (const std::exception &) {
    return CZ_ERR_CUDA;
  }
}

const char *cz_version(void) { return "cheese_b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace {
int specgen_input(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names, const int *qubits,
                  int &nq, std::vector<cz::CircGate> &circ, std::string &err) {
  if (qasm) return cz::parse_qasm(qasm, qasm_len, nq, circ, err);
  if (ngates < 0 || (ngates > 0 && (!names || !qubits))) { err = "bad gate list"; return CZ_ERR_SPEC; }
  nq = n;
  circ.clear();
  for (int i = 0; i < ngates; i++) {
    cz::CircGate g;
    g.g = names[i] ? names[i] : "";
    for (int j = 0; j < 3 && qubits[3 * i + j] >= 0; j++) g.q[g.nq++] = qubits[3 * i + j];
    circ.push_back(g);
  }
  return 0;
}
int specgen_out(const std::string &text, char *out, size_t cap, size_t *out_len) {
  if (out_len) *out_len = text.size();
  if (!out || cap < text.size() + 1) return CZ_ERR_USAGE;
  std::memcpy(out, text.c_str(), text.size() + 1);
  return 0;
}
}  // namespace

int cz_spec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                     const int *qubits, int depth, int no_w3, char *out, size_t cap, size_t *out_len,
                     cz_specgen_info *info, char *err, size_t errlen) {
  return cz_spec_generate_states(qasm, qasm_len, n, ngates, names, qubits, depth, no_w3, nullptr, 0, out, cap,
                                 out_len, info, err, errlen);
}

int cz_spec_generate_states(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                            const int *qubits, int depth, int no_w3, const int *inputs, int ninputs, char *out,
                            size_t cap, size_t *out_len, cz_specgen_info *info, char *err, size_t errlen) {
  std::string e, text;
  std::vector<cz::CircGate> circ;
  int nq = 0;
  if (ninputs < 0 || (ninputs > 0 && !inputs)) {
    put_err(err, errlen, "bad input list");
    return 2;
  }
  int rc = specgen_input(qasm, qasm_len, n, ngates, names, qubits, nq, circ, e);
  cz::SpecGenInfo gi;
  const std::vector<int> in(inputs, inputs + ninputs);
  if (!rc) rc = cz::spec_generate(nq, circ, depth, no_w3 == 0, in, text, gi, e);
  if (rc) {
    put_err(err, errlen, e);
    return rc;
  }
  if (info) {
    info->n = nq; info->gates = (int)circ.size(); info->candidates = gi.candidates;
    info->w2_pairs = gi.bad2; info->w3_triples = gi.bad3;
  }
  return specgen_out(text, out, cap, out_len);
}

int cz_rspec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                      const int *qubits, int outcome, char *out, size_t cap, size_t *out_len, cz_rspec_info *info,
                      char *err, size_t errlen) {
  std::string e, text;
  std::vector<cz::CircGate> circ;
  int nq = 0;
  int rc = specgen_input(qasm, qasm_len, n, ngates, names, qubits, nq, circ, e);
  cz::RusSpecInfo ri;
  if (!rc) rc = cz::rspec_generate(nq, circ, qasm ? std::string(qasm, qasm_len) : std::string(), outcome, text, ri, e);
  if (rc) {
    put_err(err, errlen, e);
    return rc;
  }
  if (info) {
    info->outcome = ri.outcome; info->roots = ri.roots; info->rescalings = ri.rescalings;
    info->failure_amplitudes = ri.failure_amplitudes;
    for (int i = 0; i < 3; i++) info->p[i] = ri.p[i];
  }
  return specgen_out(text, out, cap, out_len);
}

int cz_tspec_generate(const char *qasm, size_t qasm_len, int n, int ngates, const char *const *names,
                      const int *qubits, char *out, size_t cap, size_t *out_len, char *err, size_t errlen) {
  std::string e, text;
  std::vector<cz::CircGate> circ;
  int nq = 0;
  int rc = specgen_input(qasm, qasm_len, n, ngates, names, qubits, nq, circ, e);
  if (!rc) rc = cz::tspec_generate(nq, circ, text, e);
  if (rc) {
    put_err(err, errlen, e);
    return rc;
  }
  return specgen_out(text, out, cap, out_len);
}
