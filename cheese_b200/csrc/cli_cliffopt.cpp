// cliffopt: drop-in for the reference's build/cliffopt (src/clifford.cu:240-384). Same arguments, stdout, stderr
// lines and exit codes; runs on the B200 through the C ABI.
//   cliffopt JOB [--beam B]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cheese_b200.h"

static void print_step(void *, int j, int64_t placements, int best) {
  std::fprintf(stderr, "  T gate %d: %lld placements x beam, best partial %d\n", j + 1, (long long)placements, best);
}

int main(int argc, char **argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: cliffopt JOB [--beam B]\n"); return 3; }
  std::ifstream f(argv[1], std::ios::binary);
  std::stringstream ss;
  if (f) ss << f.rdbuf();
  const std::string job = ss.str();
  int beam = 16;
  for (int i = 2; i < argc; i++)
    if (!std::strcmp(argv[i], "--beam") && i + 1 < argc) beam = std::max(1, std::min(255, std::atoi(argv[++i])));
  char err[256] = {0};
  int n = 0, t = 0;
  if (const int prc = cz_cliffjob_check(job.data(), job.size(), &n, &t, err, sizeof err)) {
    std::fprintf(stderr, "%s\n", err);
    return prc;
  }
  cz_engine *eng = nullptr;
  if (cz_engine_create(0, &eng, err, sizeof err)) {
    std::fprintf(stderr, "CUDA error: %s\n", err);
    return 5;
  }
  cz_clifford_table_info ti;
  int rc = cz_clifford_table(eng, n, &ti, err, sizeof err);
  if (rc) {
    std::fprintf(stderr, "%s\n", err);
    cz_engine_destroy(eng);
    return rc;
  }
  for (int d = 1; d <= ti.max_distance && d < 32; d++)
    std::fprintf(stderr, "  clifford gates %d: %lld\n", d, (long long)ti.per_distance[d]);
  std::fprintf(stderr, "clifford table: %lld elements (group order %lld), %.1f s\n", (long long)ti.elements,
               (long long)ti.order, ti.seconds);
  std::vector<char> text((size_t)(t + 1) * 16 * 14 + 4096);
  cz_cliffopt_result res;
  rc = cz_cliffopt(eng, job.data(), job.size(), beam, print_step, nullptr, text.data(), text.size(), &res);
  if (rc == 0 && res.text_len >= text.size()) {   // longer than the estimate: run again into a big enough buffer
    text.resize(res.text_len + 1);
    rc = cz_cliffopt(eng, job.data(), job.size(), beam, nullptr, nullptr, text.data(), text.size(), &res);
  }
  if (rc) {
    std::fprintf(stderr, "%s\n", res.error);
  } else {
    std::printf("{\"clifford_gates\": %d, \"clifford_gates_before\": %d, \"t_gates\": %d, \"seconds\": %.2f}\n",
                res.clifford_gates, res.clifford_gates_before, res.t_gates, res.seconds + ti.seconds);
    std::fputs(text.data(), stdout);
  }
  cz_engine_destroy(eng);
  std::fflush(stdout);
  return rc;
}
