// T-count search with a coset table (the reference's build/tcount, src/tcount.cu), host side.
//
// U = R(P_1) ... R(P_t) C with R(P) = ((1 + w) I + (1 - w) P) / 2 and C a Clifford (global phase ignored). The
// search works on channel matrices Uc[a][b] = Tr(P_a U P_b U^dag) / 2^n, 4^n x 4^n with entries
// (x + y sqrt2) / sqrt2^e and one exponent e per matrix. Peeling R(P_p)^-1 off the left keeps the rows that commute
// with P_p (times sqrt2 in the common exponent) and replaces an anticommuting row a by row a - s row r, where
// i P_p P_a = s P_r (tcount.cu:80-113). A right coset S C is labelled by e and the multiset of sign-normalised
// columns; equality of cosets is always decided exactly.
#pragma once
#include <functional>
#include <string>
#include <vector>

namespace cz {

struct TSpec {
  int n = 0, P = 0, e = 0;
  std::vector<int> x, y, tr, ts;   // channel P x P; rotation tables (P - 1) x P
};
// the grammar of tcount.cu:434-450; returns 0, 2 (bad spec) or 3 (n outside 1..3)
int parse_tspec(const char *text, size_t len, TSpec &out, std::string &err);

struct TcLevel {                    // one JSON line of grow() (tcount.cu:391-392)
  bool table = false;               // "dir": "table" (table build) or "search"
  int t = 0;
  long long parents = 0, children = 0, cosets = 0, fresh = 0;
  double seconds = 0;
};

struct TcResult {
  int rc = 1;                       // 0 found, 1 above max, 4 coefficient overflow, 5 CUDA error
  int tcount = -1, split_j = 0, split_c = 0, maxt = 16;
  std::vector<std::pair<int, int>> rotations;   // (p, inv)
  long long table_cosets = 0;       // table size (all levels)
  int table_levels = 0;
  bool table_loaded = false, table_built = false, table_resident = false;
  std::string table_path;
  double table_seconds = 0, total_seconds = 0;
  long long launches = 0;
  std::string error;
};

struct TcOptions {
  int table_k = 4, maxt = 16;
  std::string cache_dir = "build";  // table cache: <dir>/tcount-table-n<n>-k<K>.cz.bin (reads the reference's too)
  bool use_cache = true;
};

class TcountContext;                // device state of one engine: resident tables per (n, K)
TcountContext *tcount_context_create(int device, void *stream);
void tcount_context_destroy(TcountContext *);
// release the work buffers (kept at peak size between calls); resident tables stay; returns the bytes released
size_t tcount_context_trim(TcountContext *);
int tcount_run(TcountContext *ctx, const TSpec &sp, const TcOptions &opt,
               const std::function<void(const TcLevel &)> &on_level, TcResult &res);

}  // namespace cz
