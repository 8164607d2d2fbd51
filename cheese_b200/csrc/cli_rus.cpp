// rus: drop-in for the reference's build/rus (src/rus.cu:512-587). Same arguments, stdout lines, stderr messages and
// exit codes; runs on the B200 through the C ABI.
//   rus SPEC [--table K] [--max T]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/cheese_b200.h"

static void print_level(void *, const cz_tcount_level *l) {
  std::printf("{\"dir\": \"%s\", \"t\": %d, \"parents\": %lld, \"children\": %lld, \"cosets\": %lld, \"new\": %lld, "
              "\"seconds\": %.2f}\n",
              l->table ? "table" : "search", l->t, (long long)l->parents, (long long)l->children, (long long)l->cosets,
              (long long)l->fresh, l->seconds);
  std::fflush(stdout);
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: rus SPEC [--table K] [--max T]\n"
                         "optimal RUS T-count (success branch and Pr[success] fixed, failure a Clifford);\n"
                         "exit 0 found, 1 none with T-count <= T\n");
    return 3;
  }
  std::ifstream f(argv[1], std::ios::binary);
  std::stringstream ss;
  if (f) ss << f.rdbuf();
  const std::string text = ss.str();
  cz_rus_options opt;
  cz_rus_options_default(&opt);
  for (int i = 2; i < argc; i++) {
    if (!std::strcmp(argv[i], "--table") && i + 1 < argc) opt.table_k = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--max") && i + 1 < argc) opt.maxt = std::atoi(argv[++i]);
  }
  char err[256] = {0};
  // spec errors are reported before any device work, like the reference (read_spec runs before CUDA setup)
  if (const int prc = cz_rspec_check(text.data(), text.size(), nullptr, err, sizeof err)) {
    std::fprintf(stderr, "%s\n", err);
    return prc;
  }
  cz_engine *eng = nullptr;
  if (cz_engine_create(0, &eng, err, sizeof err)) {
    std::fprintf(stderr, "CUDA error: %s\n", err);
    return 5;
  }
  cz_rus_result res;
  const int rc = cz_rus(eng, text.data(), text.size(), &opt, print_level, nullptr, &res);
  if (rc == 2 || rc == 3) {
    std::fprintf(stderr, "%s\n", res.error);
  } else {
    if (res.table_loaded)
      std::fprintf(stderr, "table %s: %lld cosets (loaded, %.1f s)\n", res.table_path, (long long)res.table_cosets,
                   res.table_seconds);
    else if (res.table_built)
      std::fprintf(stderr, "table: %lld cosets with T-count <= %d (%.1f s), cached in %s\n",
                   (long long)res.table_cosets, res.table_levels, res.table_seconds, res.table_path);
    if (rc == 0) {
      std::printf("{\"tcount\": %d, \"root\": %u, \"fw\": [", res.tcount, res.root);
      for (int i = 0; i < res.split_j; i++) std::printf("%s%d", i ? ", " : "", res.fw[i]);
      std::printf("], \"cliff\": %d, \"tb\": [", res.cliff);
      for (int i = 0; i < res.split_c; i++) std::printf("%s%d", i ? ", " : "", res.tb[i]);
      std::printf("], \"split\": [%d, %d], \"seconds\": %.2f}\n", res.split_j, res.split_c, res.total_seconds);
    } else if (rc == 1) {
      std::printf("{\"tcount_above\": %d, \"seconds\": %.2f}\n", res.maxt, res.total_seconds);
    } else {
      std::fprintf(stderr, "%s\n", res.error);
    }
  }
  cz_engine_destroy(eng);
  std::fflush(stdout);
  return rc;
}
