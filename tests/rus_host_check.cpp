// Host-compiled check of the RUS search's per-node arithmetic (cheese_b200/csrc/cz_rus_node.h: peel, coset key,
// Clifford equivalence, replay) driven through the same level flow as the sm_100a path (children keyed by the first
// and second key, stable sort by the first key, group head = the first of the run with an equal second key, table
// records sorted by key with (level, index) order inside equal keys). Test infrastructure only; its output is
// compared with the C restatement in oracle/ by tests/test_rus_fixtures.py.
//   rus-host-check RSPEC [--table K] [--max T]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <tuple>
#include <vector>

#include "../cheese_b200/csrc/cz_rus_node.h"

using namespace cz::rus;

static std::vector<int8_t> TR, TS, SG;
static std::vector<uint8_t> PM;
static std::vector<int> BYGEN(1 << 20, -1);
static RDev sp;

struct Tr {                        // a tree: per level (parent, rotation); the top level's matrices and keys
  std::vector<std::vector<uint32_t>> par{{}};
  std::vector<std::vector<uint8_t>> gat{{}};
  std::vector<std::vector<int>> roots;
  std::vector<RM> top;
  std::vector<uint64_t> f1, f2;
  int t() const { return (int)par.size() - 1; }
  RHist hist() const {
    RHist H{};
    for (int l = 1; l <= t(); l++) { H.par[l] = par[l].data(); H.gat[l] = gat[l].data(); }
    return H;
  }
};
struct Rec { uint64_t h1, h2; uint32_t lvl, idx; };
static std::vector<Rec> table;
static std::vector<int> troot;

static RM child(const RM &p, int g, bool &bad) { RM c; bad |= rm_peel(p, c, g, sp); return c; }

static long lookup_one(const RM &A, uint64_t a, uint64_t b, const Tr &D, int maxc, int &cl, bool &bad) {
  auto lo = std::lower_bound(table.begin(), table.end(), std::make_pair(a, b), [](const Rec &r, const std::pair<uint64_t, uint64_t> &k) {
    return r.h1 != k.first ? r.h1 < k.first : r.h2 < k.second;
  });
  long res = -1;
  int rl = 1 << 30;
  cl = -1;
  RHist H = D.hist();
  for (auto x = lo; x != table.end() && x->h1 == a && x->h2 == b; ++x) {
    const int lv = (int)x->lvl;
    if (lv > maxc || lv >= rl) continue;
    RM M, W;
    bad |= rm_replay(M, W, troot.data(), H, lv, x->idx, sp);
    const int c = rm_equiv(M, A, sp);
    if (c >= 0) { res = x - table.begin(); rl = lv; cl = c; }
  }
  return res;
}

static long grow(Tr &T, bool tab, const char *tag) {
  bool bad = false;
  const int t = T.t() + 1;
  const long m = (long)T.top.size(), nc = m * NG;
  std::vector<RM> ch(nc);
  std::vector<uint64_t> k1(nc), k2(nc);
  for (long o = 0; o < nc; o++) { ch[o] = child(T.top[o / NG], (int)(o % NG) + 1, bad); rm_key(ch[o], k1[o], k2[o]); }
  std::vector<uint32_t> ord(nc);
  for (long o = 0; o < nc; o++) ord[o] = (uint32_t)o;
  std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return k1[x] < k1[y]; });
  std::vector<uint32_t> kept;
  for (long j = 0; j < nc; j++) {
    long i = j;
    while (i > 0 && k1[ord[i - 1]] == k1[ord[j]]) i--;
    long h = j;
    for (long q = i; q < j; q++) if (k2[ord[q]] == k2[ord[j]]) { h = q; break; }
    if (h == j || rm_equiv(ch[ord[h]], ch[ord[j]], sp) < 0) kept.push_back(ord[j]);
  }
  if (bad) { std::fprintf(stderr, "coefficient overflow (int32)\n"); std::exit(4); }
  std::sort(kept.begin(), kept.end());
  std::vector<uint32_t> P;
  std::vector<uint8_t> G;
  std::vector<RM> top;
  std::vector<uint64_t> f1, f2;
  for (uint32_t idx : kept) {
    P.push_back(idx / NG); G.push_back((uint8_t)(idx % NG + 1)); top.push_back(ch[idx]);
    f1.push_back(k1[idx]); f2.push_back(k2[idx]);
  }
  T.par.push_back(P); T.gat.push_back(G);
  const long nk = (long)kept.size();
  long fresh = nk;
  if (tab) {
    std::vector<uint32_t> P2;
    std::vector<uint8_t> G2;
    std::vector<RM> top2;
    std::vector<uint64_t> a1, a2;
    for (long j = 0; j < nk; j++) {
      int cl;
      if (lookup_one(top[j], f1[j], f2[j], T, t - 1, cl, bad) >= 0) continue;
      P2.push_back(P[j]); G2.push_back(G[j]); top2.push_back(top[j]); a1.push_back(f1[j]); a2.push_back(f2[j]);
    }
    fresh = (long)P2.size();
    T.par.back() = P2; T.gat.back() = G2;
    top = top2; f1 = a1; f2 = a2;
    for (long j = 0; j < fresh; j++) table.push_back({f1[j], f2[j], (uint32_t)t, (uint32_t)j});
    std::stable_sort(table.begin(), table.end(), [](const Rec &x, const Rec &y) {
      return x.h1 != y.h1 ? x.h1 < y.h1 : x.h2 < y.h2;
    });
  }
  if (bad) { std::fprintf(stderr, "coefficient overflow (int32)\n"); std::exit(4); }
  T.top = top; T.f1 = f1; T.f2 = f2;
  std::printf("{%s\"t\": %d, \"parents\": %ld, \"children\": %ld, \"cosets\": %ld, \"new\": %ld, \"seconds\": 0.00}\n", tag,
              t, m, nc, nk, fresh);
  return fresh;
}

static void read_mat(std::ifstream &in, std::vector<int> &out) {
  int e; in >> e;
  std::vector<int> v(MS, 0);
  for (int i = 0; i < NE; i++) in >> v[i] >> v[NE + i];
  v[2 * NE] = e;
  out.insert(out.end(), v.begin(), v.end());
}

int main(int argc, char **argv) {
  if (argc < 2) return 3;
  std::ifstream in(argv[1]);
  std::string tok;
  int ver, nroot = 0;
  in >> tok >> ver;
  std::vector<int> roots;
  while (in >> tok) {
    if (tok == "table-root") read_mat(in, troot);
    else if (tok == "roots") { in >> nroot; for (int r = 0; r < nroot; r++) read_mat(in, roots); }
    else if (tok == "rotations") {
      int m; in >> m;
      for (int i = 0; i < m * NR; i++) { int a, b; in >> a >> b; TR.push_back((int8_t)a); TS.push_back((int8_t)b); }
    } else if (tok == "cliffords") {
      int m; in >> m;
      for (int i = 0; i < m * NR; i++) { int p, g; in >> p >> g; PM.push_back((uint8_t)p); SG.push_back((int8_t)g); }
    } else if (tok == "end") break;
  }
  const int GEN[4] = {1, 3, 4, 12};
  for (int c = 0; c < NCL; c++) {
    int key = 0;
    for (int g = 0; g < 4; g++) key |= ((PM[c * NR + GEN[g]] << 1) | (SG[c * NR + GEN[g]] < 0)) << (5 * g);
    BYGEN[key] = c;
  }
  sp = RDev{TR.data(), TS.data(), PM.data(), SG.data(), BYGEN.data()};
  int K = 8, maxt = 16;
  for (int i = 2; i < argc; i++) {
    if (!std::strcmp(argv[i], "--table") && i + 1 < argc) K = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--max") && i + 1 < argc) maxt = std::atoi(argv[++i]);
  }
  Tr D;
  RM j00;
  rm_load(j00, troot.data());
  D.top = {j00};
  uint64_t a, b;
  rm_key(j00, a, b);
  table.push_back({a, b, 0, 0});
  for (int l = 1; l <= K; l++) if (!grow(D, true, "\"dir\": \"table\", ")) break;
  Tr T;
  for (int r = 0; r < nroot; r++) {
    RM M;
    rm_load(M, roots.data() + (size_t)r * MS);
    T.top.push_back(M);
    rm_key(M, a, b);
    T.f1.push_back(a); T.f2.push_back(b);
  }
  for (int j = 0; j <= maxt; j++) {
    if (j > 0 && !grow(T, false, "\"dir\": \"search\", ")) break;
    const int maxc = std::min(D.t(), maxt - j);
    long best = -1, bestx = -1;
    int bestc = 1 << 30, bestcl = -1;
    bool bad = false;
    for (long i = 0; i < (long)T.top.size(); i++) {
      int cl;
      const long x = lookup_one(T.top[i], T.f1[i], T.f2[i], D, maxc, cl, bad);
      if (x >= 0 && (int)table[x].lvl < bestc) { bestc = (int)table[x].lvl; best = i; bestx = x; bestcl = cl; }
    }
    if (bad) { std::fprintf(stderr, "coefficient overflow (int32)\n"); return 4; }
    if (best >= 0) {
      std::vector<int> fw(j), tb(bestc);
      uint32_t i = (uint32_t)best;
      for (int l = j; l >= 1; l--) { fw[l - 1] = T.gat[l][i]; i = T.par[l][i]; }
      const uint32_t root = i;
      i = table[bestx].idx;
      for (int l = bestc; l >= 1; l--) { tb[l - 1] = D.gat[l][i]; i = D.par[l][i]; }
      std::printf("{\"tcount\": %d, \"root\": %u, \"fw\": [", j + bestc, root);
      for (int l = 0; l < j; l++) std::printf("%s%d", l ? ", " : "", fw[l]);
      std::printf("], \"cliff\": %d, \"tb\": [", bestcl);
      for (int l = 0; l < bestc; l++) std::printf("%s%d", l ? ", " : "", tb[l]);
      std::printf("], \"split\": [%d, %d], \"seconds\": 0.00}\n", j, bestc);
      return 0;
    }
    if (j + D.t() >= maxt) break;
  }
  std::printf("{\"tcount_above\": %d, \"seconds\": 0.00}\n", maxt);
  return 1;
}
