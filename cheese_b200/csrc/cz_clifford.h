// Clifford-table path (the reference's src/clifford.cu, "cliffopt"): BFS distance table of the n-qubit Clifford
// group, beam search over T-gate placements, optimal read-back of every Clifford segment.
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace cz {

struct CliffJob {                  // clifford.cu:213-238
  int n = 0;
  std::vector<int> tq, td;         // T gates in time order: qubit, dagger
  std::vector<std::vector<int>> seg;   // t + 1 segments, 3 ints per gate (kind, a, b)
};
// 0, or 2 with the reference's message ("bad job file", "unknown Clifford gate X")
int parse_cliff_job(const char *text, size_t len, CliffJob &job, std::string &err);

struct CliffTableInfo {
  int n = 0;
  long long order = 0, elements = 0;
  int max_distance = 0;
  long long per_distance[32] = {0};
  bool built = false;              // built by this call (else resident)
  double seconds = 0;
};

struct CliffStep { long long placements; int best_partial; };
struct CliffOptResult {
  int rc = 0;
  int clifford_gates = 0, before = 0, t_gates = 0;
  double seconds = 0;
  CliffTableInfo table;
  std::string text;                // the gate lines after the JSON line
  std::string error;
  long long launches = 0;
};

class CliffordContext;
CliffordContext *clifford_context_create(int device, void *stream);
void clifford_context_destroy(CliffordContext *c);
// release the work buffers (kept at peak size between calls); resident tables stay; returns the bytes released
size_t clifford_context_trim(CliffordContext *c);
// the table of n qubits, resident after the first call: 0 or 5 (CUDA error) / 4 (group order mismatch)
int clifford_table(CliffordContext *c, int n, CliffTableInfo &info, std::string &err);
int cliffopt_run(CliffordContext *c, const CliffJob &job, int beam,
                 const std::function<void(int, const CliffStep &)> &on_step, CliffOptResult &res);
// minimal gate counts of tableaux (-1: not a valid tableau)
int clifford_dist(CliffordContext *c, int n, const uint64_t *tab, size_t count, int *out, std::string &err);
// an optimal word of each tableau: (kind, a, b) triples, kinds as in the job grammar (h s sdg x z cx y = 0..6)
int clifford_words(CliffordContext *c, int n, const uint64_t *tab, size_t count,
                   std::vector<std::vector<int>> &words, std::string &err);
// the group element of each rank (index in [0, order))
int clifford_element(CliffordContext *c, int n, const uint64_t *index, size_t count, uint64_t *tab, std::string &err);

}  // namespace cz
