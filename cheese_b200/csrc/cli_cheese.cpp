// cheese: drop-in for the reference's build/cheese (src/cheese.cu:1851-1895). Same arguments, stdout lines, stderr
// banner and exit codes; the search runs on the B200 through the C ABI.
//   cheese SPEC [--depth D] [--no-dedupe] [--chunk PARENTS] [--mitm] [--no-sym] [--table K] [--profile]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/cheese_b200.h"

static double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

static void print_level(void *, const cz_level_stats *s) {
  std::printf("{%s\"t\": %d, \"parents\": %lld, \"prefixes\": %lld, \"cut_w3\": %lld, \"cut_lb\": %lld, \"survivors\": %lld, "
              "\"distinct\": %lld, \"proved_unsat\": %s, \"seconds\": %.2f}\n",
              s->dir == 1 ? "\"dir\": \"table\", " : s->dir == 2 ? "\"dir\": \"fwd\", " : s->dir == 3 ? "\"dir\": \"bwd\", " : "",
              s->t, (long long)s->parents, (long long)s->prefixes, (long long)s->cut_w3, (long long)s->cut_lb,
              (long long)s->survivors, (long long)s->distinct, s->distinct ? "false" : "true", s->seconds);
  std::fflush(stdout);
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: cheese SPEC [--depth D] [--no-dedupe] [--chunk PARENTS] [--mitm] [--no-sym] [--table K] [--profile]\n"
                         "exit 0: circuit found, 1: no circuit of <= depth gates (proof)\n");
    return 3;
  }
  std::ifstream f(argv[1], std::ios::binary);
  std::stringstream ss;
  if (f) ss << f.rdbuf();
  const std::string text = ss.str();
  cz_spec *spec = nullptr;
  char err[256] = {0};
  const int prc = cz_spec_parse(text.data(), text.size(), &spec, err, sizeof err);
  if (prc == CZ_ERR_SPEC) { std::fprintf(stderr, "%s\n", err); return 2; }
  int n = 0, G = 0, sdepth = 0;
  if (spec) cz_spec_info(spec, &n, &G, &sdepth);
  cz_options opt;
  cz_options_default(&opt);
  int depth = sdepth, mitm = 0, tablek = 0, profile = 0;
  for (int i = 2; i < argc; i++) {
    if (!std::strcmp(argv[i], "--depth") && i + 1 < argc) depth = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--no-dedupe")) opt.dedupe = 0;
    else if (!std::strcmp(argv[i], "--chunk") && i + 1 < argc) ++i;      // the whole level runs in one launch
    else if (!std::strcmp(argv[i], "--profile")) profile = 2;   // both phases timed
    else if (!std::strcmp(argv[i], "--mitm")) mitm = 1;
    else if (!std::strcmp(argv[i], "--no-sym")) opt.sym = 0;
    else if (!std::strcmp(argv[i], "--table") && i + 1 < argc) tablek = std::atoi(argv[++i]);
  }
  if (depth > CZ_MAX_DEPTH) { std::fprintf(stderr, "depth > %d\n", CZ_MAX_DEPTH); return 3; }
  std::fprintf(stderr, "cheese: n %d, %d candidates, depth %d, dedupe %d\n", n, G, depth, opt.dedupe);
  if (prc == CZ_ERR_USAGE || !spec) { std::fprintf(stderr, "n = %d not built (NQ_MIN..NQ_MAX)\n", n); return 3; }
  opt.depth = depth;
  opt.mitm = mitm;
  opt.table_k = tablek > 0 ? tablek : 0;
  opt.profile = profile;
  cz_engine *eng = nullptr;
  if (cz_engine_create(0, &eng, err, sizeof err)) { std::fprintf(stderr, "CUDA error after engine: %s\n", err); return 5; }
  cz_result res;
  const double t0 = now();
  const int rc = cz_search(eng, spec, &opt, print_level, nullptr, &res);
  std::fprintf(stderr, "symmetry classes: %d group elements\n", res.nsym);
  if (res.table_loaded)
    std::fprintf(stderr, "table %s: %lld classes (loaded, %.1f s)\n", res.table_path, (long long)res.table_classes,
                 res.table_seconds);
  else if (res.table_built)
    std::fprintf(stderr, "table: %lld classes within %d gates (%.1f s), cached in %s\n", (long long)res.table_classes,
                 res.table_levels, res.table_seconds, res.table_path);
  int code = rc;
  if (res.mitm_join)
    std::printf("{\"dir\": \"join\", \"forward\": %lld, \"backward\": %lld, \"hash_matches\": %lld, \"seconds\": %.2f}\n",
                (long long)res.mitm_forward, (long long)res.mitm_backward, (long long)res.mitm_hash_matches,
                res.mitm_seconds);
  if (rc == CZ_CIRCUIT) {
    if (res.depth0) std::printf("{\"found\": 0, \"circuit\": []}\n");
    else {
      std::printf("{\"t\": %d, \"found\": %lld, \"circuit\": [", res.found_len, (long long)(res.n_found ? res.n_found : 1));
      for (int i = 0; i < res.found_len; i++) std::printf("%s\"%s\"", i ? ", " : "", cz_spec_gate_name(spec, res.found[i]));
      if (res.mitm_found)
        std::printf("], \"mitm\": [%d, %d], \"seconds\": %.2f}\n", res.mitm_split[0], res.mitm_split[1], now() - t0);
      else if (res.table_split[0] + res.table_split[1] > 0)
        std::printf("], \"table\": [%d, %d], \"seconds\": %.2f}\n", res.table_split[0], res.table_split[1], now() - t0);
      else
        std::printf("], \"seconds\": %.2f}\n", now() - t0);
    }
  } else if (rc == CZ_PROOF && res.mitm_proof) {
    std::printf("{\"depth\": %d, \"proved_unsat\": true, \"mitm\": [%d, %d]}\n", depth, res.mitm_split[0],
                res.mitm_split[1]);
  } else if (rc == CZ_PROOF && res.table_proof) {
    std::printf("{\"depth\": %d, \"proved_unsat\": true, \"table\": %d}\n", depth, res.table_k);
  } else if (rc == CZ_ERR_CUDA) {
    std::fprintf(stderr, "%s\n", res.error);
  } else if (rc != CZ_PROOF) {
    if (res.error[0]) std::fprintf(stderr, "%s\n", res.error);
  }
  if (profile) {
    std::fprintf(stderr, "  %-9s %.3f s\n", "expand", res.expand_ms / 1e3);
    std::fprintf(stderr, "  %-9s %.3f s\n", "dedupe", res.dedupe_ms / 1e3);
    std::fprintf(stderr, "  kernels   %lld, T-bound evaluations %lld, int64 limbs %d\n", (long long)res.kernel_launches,
                 (long long)res.t_evals, res.store64);
  }
  cz_engine_destroy(eng);
  cz_spec_free(spec);
  std::fflush(stdout);
  return code;
}
