// RUS T-count with measurement (the reference's build/rus, src/rus.cu), host side.
//
// Only J = W(|0> x I) of a two-qubit circuit W (ancilla q0, data q1) matters. The search works on J's Pauli
// transfer matrix Jc[a][b] = Tr(P_a J P_b J^dag) / 2 (16 rows: two-qubit Paulis, 4 columns: one-qubit Paulis), entries
// (x + y sqrt2) / sqrt2^e, modulo left Cliffords (signed row permutations). A table holds the cosets reachable from
// J00 = |0> x I with <= K peels R(P)^-1; the search peels the spec's roots level by level and looks every node up in
// the table: a node equal to C times a table entry of level c gives a circuit with j + c T gates, and the first level
// with a hit is optimal (rus.cu:1-24, 512-587).
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace cz {

struct RSpec {                      // a rus-spec (rus.cu:470-510; writer python/cheese/rus.py)
  int nroot = 0, te = 0;
  std::vector<int> rx, ry, re;      // roots: nroot x 16 x 4 entries (x, y) and exponents
  std::vector<int> tx, ty;          // table root J00
  std::vector<int> tr, ts;          // 15 x 16: partner row and sign per rotation and row (partner < 0: commutes)
  std::vector<uint8_t> perm;        // 11520 x 16: the row permutation of each left Clifford
  std::vector<int8_t> sign;         // 11520 x 16: its signs
};
// the grammar of rus.cu:486-510; returns 0 or 2 (with err: the reference's message where it has one)
int parse_rspec(const char *text, size_t len, RSpec &out, std::string &err);

struct RusLevel {                   // one JSON line of grow() (rus.cu:430-432)
  bool table = false;               // "dir": "table" (table build) or "search"
  int t = 0;
  long long parents = 0, children = 0, cosets = 0, fresh = 0;
  double seconds = 0;
};

struct RusResult {
  int rc = 1;                       // 0 found, 1 none with T-count <= maxt, 4 coefficient overflow, 5 CUDA error
  int tcount = -1, split_j = 0, split_c = 0, maxt = 16;
  uint32_t root = 0;                // the root the found node descends from
  int cliff = -1;                   // index of the Clifford C (node = C x table entry) in the spec's list
  std::vector<int> fw, tb;          // peels of the search node and of the table entry
  long long table_cosets = 0;       // table size (all levels)
  int table_levels = 0;
  bool table_loaded = false, table_built = false, table_resident = false;
  std::string table_path;
  double table_seconds = 0, total_seconds = 0;
  long long launches = 0;
  std::string error;
};

struct RusOptions {
  int table_k = 8, maxt = 16;
  std::string cache_dir = "build";  // table cache: <dir>/rus-table-k<K>.cz.bin
  bool use_cache = true;
};

class RusContext;                   // device state of one engine: resident tables per (K, fixed tables)
RusContext *rus_context_create(int device, void *stream);
void rus_context_destroy(RusContext *);
size_t rus_context_trim(RusContext *);   // work buffers back to the device; resident tables stay
int rus_run(RusContext *ctx, const RSpec &sp, const RusOptions &opt,
            const std::function<void(const RusLevel &)> &on_level, RusResult &res);

}  // namespace cz
