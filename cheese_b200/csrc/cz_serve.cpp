// Serving loop: a persistent request server over one GPU (no counterpart in the reference, which runs one search
// per process). Three kinds of requests arrive at any time:
//   gate-count searches (spec text + budget)   -> continuous batching in one BatchSession per qubit count
//   T-count queries (tcount-spec text)          -> the T-count path, coset tables resident
//   Clifford-segment jobs (cliffopt job text)   -> the Clifford-table path, group tables resident
// Each kind has its own worker thread, engine and CUDA stream, so their device work overlaps. Gate-count requests
// join the running batch at its next level step when the batch's frontier-memory estimate (its survivor capacity
// for the next level, every running job's frontier x candidates x record size, plus the frontier itself) leaves
// room for the newcomer's first level under the memory budget, and while a slot is free. Results are the same as
// the plain entry points give for each request on its own.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cz_capi_internal.h"
#include "cz_specgen.h"

namespace {

double wall() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

struct Req {
  int id = 0, kind = 0, depth = -1;
  bool qasm = false;               // text is an OpenQASM target: the spec is generated here
  std::string text;
  double t_submit = 0, t_start = 0, t_done = 0;
  bool done = false;
  int rc = -1;
  std::string out;                 // the stdout of the reference program for this request
  std::string error;
  long long gpu_work = 0;          // prefixes (gate count), children (T count), placements (Clifford)
};

std::string level_line(const cz::LevelStats &L) {
  char b[320];
  std::snprintf(b, sizeof b,
                "{\"t\": %d, \"parents\": %lld, \"prefixes\": %lld, \"cut_w3\": %lld, \"cut_lb\": %lld, \"survivors\": %lld, "
                "\"distinct\": %lld, \"proved_unsat\": %s, \"seconds\": 0.00}\n",
                L.t, L.parents, L.prefixes, L.cut_w3, L.cut_lb, L.survivors, L.distinct, L.distinct == 0 ? "true" : "false");
  return b;
}

}  // namespace

struct cz_server {
  cz_server_options opt;
  std::mutex mu;
  std::condition_variable cv_work[3], cv_done;
  std::map<int, Req *> reqs;
  std::deque<Req *> queue[3];
  std::atomic<bool> stop{false};
  std::thread workers[3];
  int next_id = 0;
  std::atomic<long long> done_count{0};
  std::string start_error;
  std::atomic<int> started{0};
  // gate-count worker state (read by stats)
  std::atomic<long long> batch_steps{0}, batch_admitted{0}, batch_peak_running{0}, batch_deferred{0};
  std::atomic<long long> batch_peak_bytes{0};

  void finish(Req *r) {
    std::lock_guard<std::mutex> lk(mu);
    r->t_done = wall();
    r->done = true;
    done_count++;
    cv_done.notify_all();
  }
  Req *pop(int kind, bool wait) {
    std::unique_lock<std::mutex> lk(mu);
    if (wait) cv_work[kind].wait_for(lk, std::chrono::milliseconds(50), [&] { return stop || !queue[kind].empty(); });
    if (queue[kind].empty()) return nullptr;
    Req *r = queue[kind].front();
    queue[kind].pop_front();
    return r;
  }

  // ---- gate-count searches: continuous batching ----
  void gate_worker() {
    cz_engine *eng = nullptr;
    char err[256] = {0};
    if (cz_engine_create(opt.device, &eng, err, sizeof err)) { start_error = err; started++; return; }
    started++;
    struct Live { Req *r; cz_spec *spec; int nq, jid; };
    std::vector<cz::BatchSession *> sess(4, nullptr);
    std::vector<Live> live;
    std::deque<std::pair<Req *, cz_spec *>> waiting;
    const double budget = opt.memory_gb * 1e9;
    while (!stop) {
      for (Req *r; (r = pop(0, live.empty() && waiting.empty())) != nullptr;) {
        cz_spec *sp = nullptr;
        char e2[256] = {0};
        r->t_start = wall();
        if (r->qasm) {                       // an OpenQASM target: its spec, budget = its gate count by default
          int nq = 0;
          std::vector<cz::CircGate> circ;
          std::string ge, text;
          cz::SpecGenInfo gi;
          int grc = cz::parse_qasm(r->text.data(), r->text.size(), nq, circ, ge);
          if (!grc) grc = cz::spec_generate(nq, circ, r->depth >= 0 ? r->depth : (int)circ.size(), true, {}, text, gi, ge);
          if (grc) {
            r->rc = grc;
            r->error = ge;
            finish(r);
            continue;
          }
          r->text.swap(text);
        }
        const int prc = cz_spec_parse(r->text.data(), r->text.size(), &sp, e2, sizeof e2);
        if (prc || sp->hs.states || (r->depth >= 0 ? r->depth : sp->hs.depth) > CZ_MAX_DEPTH) {
          r->rc = prc ? prc : CZ_ERR_USAGE;
          r->error = prc ? e2 : "unsupported request";
          if (sp) cz_spec_free(sp);
          finish(r);
          continue;
        }
        waiting.emplace_back(r, sp);
      }
      // admission: the batch's next-level survivor capacity plus the newcomer's first level under the budget
      double projected = 0;
      int running = 0;
      for (int q = 1; q <= 3; q++)
        if (sess[q]) { projected += (double)sess[q]->projected_bytes(); running += sess[q]->running(); }
      while (!waiting.empty() && running < opt.max_jobs) {
        Req *r = waiting.front().first;
        cz_spec *sp = waiting.front().second;
        const int nq = sp->hs.n;
        const double need = (double)sp->hs.G * ((double)(1 << (2 * nq)) * 16.0 + 40.0);
        if (running > 0 && projected + need > budget) { batch_deferred++; break; }
        if (!sess[nq]) {
          sess[nq] = new cz::BatchSession(*eng->e, nq);
          sess[nq]->set_memory_budget((size_t)budget);
        }
        cz::Options o;
        o.depth = r->depth >= 0 ? r->depth : sp->hs.depth;
        const int jid = sess[nq]->submit(sp->hs, o);
        live.push_back(Live{r, sp, nq, jid});
        waiting.pop_front();
        projected += need;
        running++;
        batch_admitted++;
      }
      if ((long long)running > batch_peak_running) batch_peak_running = running;
      bool any = false;
      for (int q = 1; q <= 3; q++) {
        if (!sess[q] || !sess[q]->running()) continue;
        any = true;
        try {
          sess[q]->step();
          batch_steps++;
        } catch (const std::exception &ex) {
          for (auto &l : live)
            if (l.nq == q) { l.r->rc = CZ_ERR_CUDA; l.r->error = ex.what(); }
          delete sess[q];
          sess[q] = nullptr;
        }
        if (sess[q] && (long long)sess[q]->device_bytes() > batch_peak_bytes) batch_peak_bytes = (long long)sess[q]->device_bytes();
      }
      (void)any;
      for (size_t i = 0; i < live.size();) {
        Live &l = live[i];
        bool fin = false;
        if (l.r->rc == CZ_ERR_CUDA) fin = true;
        else if (sess[l.nq] && sess[l.nq]->job(l.jid).done) {
          const cz::BatchJob &j = sess[l.nq]->job(l.jid);
          std::string out;
          for (const cz::LevelStats &L : j.levels) out += level_line(L);
          const cz::SearchResult &res = j.res;
          if (res.rc == 0) {
            if (res.depth0) out += "{\"found\": 0, \"circuit\": []}\n";
            else {
              out += "{\"t\": " + std::to_string(res.circuit.size()) + ", \"found\": " +
                     std::to_string(res.n_found ? res.n_found : 1) + ", \"circuit\": [";
              for (size_t g = 0; g < res.circuit.size(); g++)
                out += (g ? ", \"" : "\"") + l.spec->hs.names[res.circuit[g]] + "\"";
              out += "], \"seconds\": 0.00}\n";
            }
          }
          l.r->out = out;
          l.r->rc = res.rc;
          l.r->error = res.error;
          l.r->gpu_work = res.prefixes;
          fin = true;
        }
        if (fin) {
          cz_spec_free(l.spec);
          finish(l.r);
          live[i] = live.back();
          live.pop_back();
        } else {
          i++;
        }
      }
      // a session stays (its buffers are reused by the next jobs) until it has held many jobs and none runs
      for (int q = 1; q <= 3; q++)
        if (sess[q] && !sess[q]->running() && sess[q]->jobs() > 4096) {
          bool used = false;
          for (auto &l : live) used |= l.nq == q;
          if (!used) { delete sess[q]; sess[q] = nullptr; }
        }
    }
    for (auto &l : live) { cz_spec_free(l.spec); l.r->rc = CZ_ERR_USAGE; l.r->error = "server stopped"; finish(l.r); }
    for (auto &w : waiting) { cz_spec_free(w.second); w.first->rc = CZ_ERR_USAGE; w.first->error = "server stopped"; finish(w.first); }
    for (auto *s : sess) delete s;
    cz_engine_destroy(eng);
  }

  // ---- T-count queries ----
  void tcount_worker() {
    cz_engine *eng = nullptr;
    char err[256] = {0};
    if (cz_engine_create(opt.device, &eng, err, sizeof err)) { start_error = err; started++; return; }
    started++;
    cz_tcount_options to;
    cz_tcount_options_default(&to);
    to.table_k = opt.tcount_table_k;
    to.cache_dir = opt.cache_dir;
    while (!stop) {
      Req *r = pop(1, true);
      if (!r) continue;
      r->t_start = wall();
      if (r->qasm) {                         // an OpenQASM target: its T-count spec
        int nq = 0;
        std::vector<cz::CircGate> circ;
        std::string ge, text;
        int grc = cz::parse_qasm(r->text.data(), r->text.size(), nq, circ, ge);
        if (!grc) grc = cz::tspec_generate(nq, circ, text, ge);
        if (grc) {
          r->rc = grc;
          r->error = ge;
          finish(r);
          continue;
        }
        r->text.swap(text);
      }
      std::string out;
      long long children = 0;
      auto on_level = [](void *u, const cz_tcount_level *l) {
        auto *p = (std::pair<std::string *, long long *> *)u;
        char b[256];
        std::snprintf(b, sizeof b,
                      "{\"dir\": \"%s\", \"t\": %d, \"parents\": %lld, \"children\": %lld, \"cosets\": %lld, \"new\": %lld, "
                      "\"seconds\": 0.00}\n",
                      l->table ? "table" : "search", l->t, (long long)l->parents, (long long)l->children,
                      (long long)l->cosets, (long long)l->fresh);
        *p->first += b;
        *p->second += l->children;
      };
      std::pair<std::string *, long long *> u(&out, &children);
      cz_tcount_result res;
      const int rc = cz_tcount(eng, r->text.data(), r->text.size(), &to, on_level, &u, &res);
      if (rc == 0) {
        out += "{\"tcount\": " + std::to_string(res.tcount) + ", \"rotations\": [";
        for (int i = 0; i < res.nrot; i++)
          out += (i ? ", [" : "[") + std::to_string(res.rot_p[i]) + ", " + std::to_string(res.rot_inv[i]) + "]";
        out += "], \"split\": [" + std::to_string(res.split_j) + ", " + std::to_string(res.split_c) + "], \"seconds\": 0.00}\n";
      } else if (rc == 1) {
        out += "{\"tcount_above\": " + std::to_string(res.maxt) + ", \"seconds\": 0.00}\n";
      }
      r->out = out;
      r->rc = rc;
      r->error = res.error;
      r->gpu_work = children;
      finish(r);
    }
    cz_engine_destroy(eng);
  }

  // ---- Clifford-segment jobs ----
  void cliff_worker() {
    cz_engine *eng = nullptr;
    char err[256] = {0};
    if (cz_engine_create(opt.device, &eng, err, sizeof err)) { start_error = err; started++; return; }
    started++;
    std::vector<char> text(1 << 16);
    while (!stop) {
      Req *r = pop(2, true);
      if (!r) continue;
      r->t_start = wall();
      cz_cliffopt_result res;
      long long placements = 0;
      auto on_step = [](void *u, int, int64_t p, int) { *(long long *)u += p; };
      int rc = cz_cliffopt(eng, r->text.data(), r->text.size(), opt.beam, on_step, &placements, text.data(),
                           text.size(), &res);
      if (rc == 0 && res.text_len >= text.size()) {
        text.resize(res.text_len + 1);
        rc = cz_cliffopt(eng, r->text.data(), r->text.size(), opt.beam, nullptr, nullptr, text.data(), text.size(), &res);
      }
      if (rc == 0) {
        char b[200];
        std::snprintf(b, sizeof b,
                      "{\"clifford_gates\": %d, \"clifford_gates_before\": %d, \"t_gates\": %d, \"seconds\": 0.00}\n",
                      res.clifford_gates, res.clifford_gates_before, res.t_gates);
        r->out = std::string(b) + text.data();
      }
      r->rc = rc;
      r->error = res.error;
      r->gpu_work = placements;
      finish(r);
    }
    cz_engine_destroy(eng);
  }
};

extern "C" {

void cz_server_options_default(cz_server_options *o) {
  if (!o) return;
  o->device = 0;
  o->memory_gb = 150.0;
  o->max_jobs = 4096;
  o->tcount_table_k = 4;
  o->beam = 16;
  o->cache_dir = nullptr;
}

int cz_server_create(const cz_server_options *opt, cz_server **out, char *err, size_t errlen) {
  if (!out) return CZ_ERR_USAGE;
  *out = nullptr;
  cz_server *s = new cz_server;
  cz_server_options_default(&s->opt);
  if (opt) s->opt = *opt;
  s->workers[0] = std::thread([s] { s->gate_worker(); });
  s->workers[1] = std::thread([s] { s->tcount_worker(); });
  s->workers[2] = std::thread([s] { s->cliff_worker(); });
  while (s->started < 3) std::this_thread::sleep_for(std::chrono::milliseconds(1));
  if (!s->start_error.empty()) {
    if (err && errlen) std::snprintf(err, errlen, "%s", s->start_error.c_str());
    cz_server_destroy(s);
    return CZ_ERR_CUDA;
  }
  *out = s;
  return 0;
}

void cz_server_destroy(cz_server *s) {
  if (!s) return;
  s->stop = true;
  for (auto &cv : s->cv_work) cv.notify_all();
  for (auto &w : s->workers) if (w.joinable()) w.join();
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
}

int cz_server_submit(cz_server *s, int kind, const char *text, size_t len, int depth) {
  if (!s || kind < 0 || kind > 4 || (!text && len)) return -CZ_ERR_USAGE;
  Req *r = new Req;
  r->kind = kind;
  r->depth = depth;
  r->qasm = kind >= CZ_REQ_GATES_QASM;
  const int q = kind == CZ_REQ_GATES_QASM ? 0 : kind == CZ_REQ_TCOUNT_QASM ? 1 : kind;
  r->text.assign(text ? text : "", len);
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  r->t_submit = wall();
  s->reqs[r->id] = r;
  s->queue[q].push_back(r);
  s->cv_work[q].notify_one();
  return r->id;
}

int cz_server_poll(cz_server *s, int id, cz_server_result *out, char *text, size_t cap) {
  if (!s || !out) return -CZ_ERR_USAGE;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return -CZ_ERR_USAGE;
  const Req *r = it->second;
  std::memset(out, 0, sizeof *out);
  if (!r->done) return 0;
  out->rc = r->rc;
  out->kind = r->kind;
  out->latency_s = r->t_done - r->t_submit;
  out->queued_s = r->t_start - r->t_submit;
  out->gpu_work = r->gpu_work;
  out->text_len = r->out.size();
  std::snprintf(out->error, sizeof out->error, "%s", r->error.c_str());
  if (text && cap) {
    const size_t m = std::min(cap - 1, r->out.size());
    std::memcpy(text, r->out.data(), m);
    text[m] = 0;
  }
  return 1;
}

int cz_server_wait(cz_server *s, long long count, double timeout_s) {
  if (!s) return CZ_ERR_USAGE;
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return s->done_count >= count; });
  return ok ? 0 : 1;
}

int cz_server_stats_get(cz_server *s, cz_server_stats *out) {
  if (!s || !out) return CZ_ERR_USAGE;
  std::memset(out, 0, sizeof *out);
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = (int64_t)s->reqs.size();
  out->completed = s->done_count;
  out->batch_steps = s->batch_steps;
  out->batch_admitted = s->batch_admitted;
  out->batch_deferred = s->batch_deferred;
  out->batch_peak_running = s->batch_peak_running;
  out->batch_peak_bytes = s->batch_peak_bytes;
  for (int k = 0; k < 3; k++) out->queued[k] = (int64_t)s->queue[k].size();
  return 0;
}

int cz_server_replay(cz_server *s, int n, const int *kinds, const char *const *texts, const size_t *lens,
                     const int *depths, const double *arrival_s, double timeout_s, int *ids) {
  if (!s || n < 0 || (n && (!kinds || !texts || !lens || !arrival_s || !ids))) return CZ_ERR_USAGE;
  const long long base = s->done_count;
  const double t0 = wall();
  for (int i = 0; i < n; i++) {
    const double wait_s = t0 + arrival_s[i] - wall();
    if (wait_s > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait_s));
    ids[i] = cz_server_submit(s, kinds[i], texts[i], lens[i], depths ? depths[i] : -1);
  }
  return cz_server_wait(s, base + n, timeout_s);
}

}  // extern "C"
