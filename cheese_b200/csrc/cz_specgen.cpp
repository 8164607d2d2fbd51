// Spec generation on the host, in exact Z[w] arithmetic (w = e^{i pi/4}; an element is a + b w + c w^2 + d w^3, a
// matrix is its entries over sqrt2^k with k as small as possible). Restates the reference's generators:
// python/cheese/spec.py (gate table :16-27, matrices :75-110, candidates :127-136, window rules :139-186, CX table
// :189-228, gate-set flags :317-319, text :322-350) and python/cheese/tcount.py (channel :79-101, rotation tables
// :104-129, text :157-168). Integer overflow is detected, never wrapped.
#include "cz_specgen.h"

#include <algorithm>
#include <array>
#include <cctype>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace cz {
namespace {

struct Z {
  int64_t a = 0, b = 0, c = 0, d = 0;
  bool zero() const { return !a && !b && !c && !d; }
  bool operator==(const Z &o) const { return a == o.a && b == o.b && c == o.c && d == o.d; }
  bool operator!=(const Z &o) const { return !(*this == o); }
};

int64_t chk(__int128 v) {
  if (v > INT64_MAX || v < INT64_MIN) throw std::overflow_error("coefficient exceeds 64 bits");
  return (int64_t)v;
}
Z zadd(const Z &x, const Z &y) {
  return {chk((__int128)x.a + y.a), chk((__int128)x.b + y.b), chk((__int128)x.c + y.c), chk((__int128)x.d + y.d)};
}
Z zmul(const Z &x, const Z &y) {   // w^4 = -1
  const int64_t X[4] = {x.a, x.b, x.c, x.d}, Y[4] = {y.a, y.b, y.c, y.d};
  __int128 o[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    if (!X[i]) continue;
    for (int j = 0; j < 4; j++) {
      if (!Y[j]) continue;
      const __int128 p = (__int128)X[i] * Y[j];
      if (i + j < 4) o[i + j] += p; else o[i + j - 4] -= p;
    }
  }
  return {chk(o[0]), chk(o[1]), chk(o[2]), chk(o[3])};
}
Z wpow(int p) {
  p = ((p % 8) + 8) % 8;
  Z z;
  int64_t *v[4] = {&z.a, &z.b, &z.c, &z.d};
  *v[p % 4] = p < 4 ? 1 : -1;
  return z;
}
Z conj(const Z &x) { return {x.a, -x.d, -x.c, -x.b}; }
bool down(const Z &x, Z &out) {    // x / sqrt2 when it stays in Z[w] (sqrt2 = w - w^3)
  if (((x.a - x.c) & 1) || ((x.b - x.d) & 1)) return false;
  out = {(x.b - x.d) / 2, (x.a + x.c) / 2, (x.b + x.d) / 2, (x.c - x.a) / 2};
  return true;
}
int val(Z x) {                      // how often sqrt2 divides x (at most 400, as the reference caps it)
  int v = 0;
  Z y;
  while (down(x, y)) {
    x = y;
    if (++v > 400) break;
  }
  return v;
}

struct Mat {
  int k = 0, N = 0;
  std::vector<Z> e;                 // row-major N x N
  Z &at(int r, int c) { return e[(size_t)r * N + c]; }
  const Z &at(int r, int c) const { return e[(size_t)r * N + c]; }
};
void normalise(Mat &M) {
  std::vector<Z> D(M.e.size());
  while (M.k > 0) {
    bool ok = true;
    for (size_t i = 0; i < M.e.size() && ok; i++) ok = down(M.e[i], D[i]);
    if (!ok) break;
    M.e.swap(D);
    M.k--;
  }
}
Mat identity(int N) {
  Mat M;
  M.N = N;
  M.e.assign((size_t)N * N, Z{});
  for (int i = 0; i < N; i++) M.at(i, i) = Z{1, 0, 0, 0};
  return M;
}
Mat matmul(const Mat &A, const Mat &B) {
  Mat C;
  C.N = A.N;
  C.k = A.k + B.k;
  C.e.assign((size_t)A.N * A.N, Z{});
  for (int i = 0; i < A.N; i++)
    for (int l = 0; l < A.N; l++) {
      const Z &x = A.at(i, l);
      if (x.zero()) continue;
      for (int j = 0; j < A.N; j++) {
        const Z &y = B.at(l, j);
        if (!y.zero()) C.at(i, j) = zadd(C.at(i, j), zmul(x, y));
      }
    }
  normalise(C);
  return C;
}
Mat dagger(const Mat &A) {
  Mat D = A;
  for (int r = 0; r < A.N; r++)
    for (int c = 0; c < A.N; c++) D.at(r, c) = conj(A.at(c, r));
  return D;
}

// local gate matrices: entry (l, m) = sum of w^p over the listed phases, over sqrt2^k; bit j of a local index is
// the gate's j-th qubit (cx / ccx: the controls first, the target last)
struct GateDef {
  int k = 0, dim = 0;
  std::vector<std::vector<int>> ph;   // dim x dim lists of phase exponents
  Z entry(int l, int m) const {
    Z x;
    for (int p : ph[(size_t)l * dim + m]) x = zadd(x, wpow(p));
    return x;
  }
  int arity() const { return dim == 2 ? 1 : dim == 4 ? 2 : 3; }
};
GateDef diag1(int p) { GateDef g; g.dim = 2; g.ph.assign(4, {}); g.ph[0] = {0}; g.ph[3] = {p}; return g; }
const std::map<std::string, GateDef> &gates() {
  static const std::map<std::string, GateDef> G = [] {
    std::map<std::string, GateDef> m;
    GateDef x; x.dim = 2; x.ph.assign(4, {}); x.ph[1] = {0}; x.ph[2] = {0}; m["x"] = x;
    GateDef y; y.dim = 2; y.ph.assign(4, {}); y.ph[1] = {6}; y.ph[2] = {2}; m["y"] = y;
    m["z"] = diag1(4); m["s"] = diag1(2); m["sdg"] = diag1(6); m["t"] = diag1(1); m["tdg"] = diag1(7);
    GateDef h; h.k = 1; h.dim = 2; h.ph = {{0}, {0}, {0}, {4}}; m["h"] = h;
    GateDef cx; cx.dim = 4; cx.ph.assign(16, {});
    cx.ph[0 * 4 + 0] = {0}; cx.ph[1 * 4 + 3] = {0}; cx.ph[2 * 4 + 2] = {0}; cx.ph[3 * 4 + 1] = {0}; m["cx"] = cx;
    GateDef cz; cz.dim = 4; cz.ph.assign(16, {});
    cz.ph[0] = {0}; cz.ph[5] = {0}; cz.ph[10] = {0}; cz.ph[15] = {4}; m["cz"] = cz;
    GateDef ccx; ccx.dim = 8; ccx.ph.assign(64, {});
    for (int l = 0; l < 8; l++) ccx.ph[(size_t)l * 8 + (l == 3 ? 7 : l == 7 ? 3 : l)] = {0};
    m["ccx"] = ccx;
    return m;
  }();
  return G;
}
std::string dagger_name(const std::string &g) {
  if (g == "s") return "sdg";
  if (g == "sdg") return "s";
  if (g == "t") return "tdg";
  if (g == "tdg") return "t";
  return g;                         // every other gate of the table is its own inverse
}

// 2^n x 2^n matrix of gate g on qubits qs (bit q of an index is qubit q)
Mat gate_matrix(const GateDef &G, const int *qs, int n) {
  const int N = 1 << n, L = G.dim, nq = G.arity();
  int mask = 0;
  for (int j = 0; j < nq; j++) mask |= 1 << qs[j];
  Mat M;
  M.N = N;
  M.k = G.k;
  M.e.assign((size_t)N * N, Z{});
  std::vector<int> idx(L);
  for (int base = 0; base < N; base++) {
    if (base & mask) continue;
    for (int l = 0; l < L; l++) {
      int x = base;
      for (int j = 0; j < nq; j++) x |= ((l >> j) & 1) << qs[j];
      idx[l] = x;
    }
    for (int l = 0; l < L; l++)
      for (int m = 0; m < L; m++)
        for (int p : G.ph[(size_t)l * L + m]) M.at(idx[l], idx[m]) = zadd(M.at(idx[l], idx[m]), wpow(p));
  }
  normalise(M);
  return M;
}

Mat unitary(int n, const std::vector<CircGate> &circ) {
  Mat U = identity(1 << n);
  for (const CircGate &g : circ) U = matmul(gate_matrix(gates().at(g.g), g.q, n), U);
  return U;
}

struct Cand { std::string name, g; int nq; int q[3]; };
std::vector<Cand> candidates(int n, const std::vector<std::string> &gs) {
  std::vector<Cand> out;
  for (const std::string &g : gs) {
    const int ar = gates().at(g).arity();
    std::vector<std::vector<int>> qss;
    if (ar == 1) {
      for (int q = 0; q < n; q++) qss.push_back({q});
    } else if (ar == 2) {
      for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++)
          if (a != b) qss.push_back({a, b});
    } else {                        // permutations of 3 qubits in lexicographic order, controls unordered
      for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++)
          for (int c = 0; c < n; c++)
            if (a != b && a != c && b != c && a < b) qss.push_back({a, b, c});
    }
    for (const auto &qs : qss) {
      Cand c;
      c.g = g;
      c.nq = ar;
      c.name = "L_" + g + "_";
      for (int j = 0; j < ar; j++) {
        c.q[j] = qs[j];
        c.name += (j ? "_" : "") + std::to_string(qs[j]);
      }
      for (int j = ar; j < 3; j++) c.q[j] = -1;
      out.push_back(c);
    }
  }
  return out;
}

// key of a product on its qubits after stripping the qubits it acts on trivially (spec.py canon): the qubit list,
// the exponent and the matrix, serialised
std::string canon_key(std::vector<int> qubits, Mat M) {
  for (int i = (int)qubits.size() - 1; i >= 0; i--) {
    const int N = M.N, bit = 1 << i;
    bool trivial = true;
    for (int r = 0; r < N && trivial; r++)
      for (int c = 0; c < N && trivial; c++) {
        if ((r ^ c) & bit) trivial = M.at(r, c).zero();
        else if (!((r | c) & bit)) trivial = M.at(r, c) == M.at(r | bit, c | bit);
      }
    if (!trivial) continue;
    std::vector<int> keep;
    for (int r = 0; r < N; r++) if (!(r & bit)) keep.push_back(r);
    Mat S;
    S.N = (int)keep.size();
    S.k = M.k;
    S.e.resize((size_t)S.N * S.N);
    for (int r = 0; r < S.N; r++)
      for (int c = 0; c < S.N; c++) S.at(r, c) = M.at(keep[r], keep[c]);
    normalise(S);
    M = S;
    qubits.erase(qubits.begin() + i);
  }
  std::string key;
  auto put = [&](int64_t v) { key.append((const char *)&v, 8); };
  put((int64_t)qubits.size());
  for (int q : qubits) put(q);
  put(M.k);
  put(M.N);
  for (const Z &z : M.e) { put(z.a); put(z.b); put(z.c); put(z.d); }
  return key;
}
std::string product_key(const std::vector<Cand> &cs, const int *seq, int len) {
  std::vector<int> U;
  for (int i = 0; i < len; i++)
    for (int j = 0; j < cs[seq[i]].nq; j++) U.push_back(cs[seq[i]].q[j]);
  std::sort(U.begin(), U.end());
  U.erase(std::unique(U.begin(), U.end()), U.end());
  Mat P = identity(1 << U.size());
  for (int i = 0; i < len; i++) {
    const Cand &c = cs[seq[i]];
    int lq[3] = {0, 0, 0};
    for (int j = 0; j < c.nq; j++) lq[j] = (int)(std::find(U.begin(), U.end(), c.q[j]) - U.begin());
    P = matmul(gate_matrix(gates().at(c.g), lq, (int)U.size()), P);
  }
  return canon_key(U, P);
}

// W2 / W3 window rules (spec.py sym_rules): a pair (triple) is cut when its product equals the identity, a single
// candidate (a pair), or the product of an earlier pair (triple) in the enumeration order
void sym_rules(const std::vector<Cand> &cs, bool use3, std::vector<std::array<int, 2>> &bad2,
               std::vector<std::array<int, 3>> &bad3) {
  const int G = (int)cs.size();
  std::set<std::string> shortk;
  shortk.insert(canon_key({}, identity(1)));
  for (int g = 0; g < G; g++) shortk.insert(product_key(cs, &g, 1));
  std::unordered_map<std::string, int> first;
  std::vector<std::string> keys2;
  std::vector<uint8_t> isbad((size_t)G * G, 0);
  for (int f = 0; f < G; f++)
    for (int g = 0; g < G; g++) {
      const int pr[2] = {f, g};
      std::string k = product_key(cs, pr, 2);
      bool bad = shortk.count(k) > 0;
      if (!bad) {
        auto it = first.find(k);
        if (it == first.end()) first.emplace(k, f * G + g);
        else bad = it->second != f * G + g;
      }
      if (bad) { bad2.push_back({f, g}); isbad[(size_t)f * G + g] = 1; }
      keys2.push_back(std::move(k));
    }
  // triples (f, g, h) with (f, g) and (g, h) both kept, (f, g) ascending; two triples of one (f, g) never share a
  // product (their last gates would be equal operators, and then one of the (g, h) pairs is cut), so which triple
  // of a key comes first does not depend on the order of h
  size_t ntrip = 0;
  for (int f = 0; f < G; f++)
    for (int g = 0; g < G; g++) {
      if (isbad[(size_t)f * G + g]) continue;
      for (int h = 0; h < G; h++) ntrip += !isbad[(size_t)g * G + h];
    }
  if (!use3 || ntrip > 300000) return;
  for (auto &k : keys2) shortk.insert(std::move(k));
  std::unordered_map<std::string, long> first3;
  for (int f = 0; f < G; f++)
    for (int g = 0; g < G; g++) {
      if (isbad[(size_t)f * G + g]) continue;
      for (int h = 0; h < G; h++) {
        if (isbad[(size_t)g * G + h]) continue;
        const int tr[3] = {f, g, h};
        const long id = ((long)f * G + g) * G + h;
        std::string k = product_key(cs, tr, 3);
        bool bad = shortk.count(k) > 0;
        if (!bad) {
          auto it = first3.find(k);
          if (it == first3.end()) first3.emplace(std::move(k), id);
          else bad = it->second != id;
        }
        if (bad) bad3.push_back({f, g, h});
      }
    }
}

// CX lower bound (spec.py cuts / cx_table): per qubit bipartition a demand in [0, 2|A|]; the table holds, for every
// demand vector (mixed radix), the fewest two-qubit gates whose crossings meet every demand
std::vector<std::vector<int>> cuts(int n) {
  std::vector<std::vector<int>> out;
  for (int r = 1; r <= n / 2; r++) {
    std::vector<int> A(r);
    for (int i = 0; i < r; i++) A[i] = i;
    while (true) {
      const bool has0 = std::find(A.begin(), A.end(), 0) != A.end();
      if (!(r == n - r && !has0)) out.push_back(A);
      int i = r - 1;
      while (i >= 0 && A[i] == n - r + i) i--;
      if (i < 0) break;
      A[i]++;
      for (int j = i + 1; j < r; j++) A[j] = A[j - 1] + 1;
    }
  }
  return out;
}
bool cx_table(int n, const std::vector<std::vector<int>> &cs, std::vector<int> &rad, std::vector<int> &best) {
  rad.clear();
  long size = 1;
  for (const auto &A : cs) { rad.push_back(2 * (int)A.size() + 1); size *= rad.back(); }
  if (size > 2000000) return false;
  std::vector<std::array<int, 2>> pairs;
  for (int a = 0; a < n; a++)
    for (int b = a + 1; b < n; b++) pairs.push_back({a, b});
  int top = 0;
  for (int r : rad) top = std::max(top, r - 1);
  const int INF = 1 << 30;
  best.assign(size, INF);
  std::vector<int> x(pairs.size(), 0);
  while (true) {
    long idx = 0, mult = 1;
    int sum = 0;
    for (int v : x) sum += v;
    for (size_t ci = 0; ci < cs.size(); ci++) {
      int cross = 0;
      for (size_t p = 0; p < pairs.size(); p++) {
        const bool ina = std::find(cs[ci].begin(), cs[ci].end(), pairs[p][0]) != cs[ci].end();
        const bool inb = std::find(cs[ci].begin(), cs[ci].end(), pairs[p][1]) != cs[ci].end();
        if (ina != inb) cross += x[p];
      }
      idx += std::min(cross, rad[ci] - 1) * mult;
      mult *= rad[ci];
    }
    best[idx] = std::min(best[idx], sum);
    size_t p = pairs.size();             // next x in itertools.product order (last digit fastest)
    while (p > 0 && x[p - 1] == top) x[--p] = 0;
    if (p == 0) break;
    x[p - 1]++;
  }
  long mult = 1;
  for (int r : rad) {                    // superset minimum, one dimension at a time
    for (long i = size - 1; i >= 0; i--)
      if ((i / mult) % r < r - 1) best[i] = std::min(best[i], best[i + mult]);
    mult *= r;
  }
  return true;
}

// P_b applied to a vector: digits per qubit 0 I, 1 X, 2 Y, 3 Z
std::vector<Z> pauli_apply(int n, int b, const std::vector<Z> &row) {
  std::vector<Z> out(row.size());
  for (size_t x = 0; x < row.size(); x++) {
    if (row[x].zero()) continue;
    int flip = 0, ph = 0;
    for (int q = 0; q < n; q++) {
      const int dg = (b >> (2 * q)) & 3, bit = (int)(x >> q) & 1;
      if (dg == 1) flip |= 1 << q;
      else if (dg == 2) { flip |= 1 << q; ph += 2 + 4 * bit; }
      else if (dg == 3) ph += 4 * bit;
    }
    out[x ^ flip] = zmul(row[x], wpow(ph));
  }
  return out;
}
Z inner(const std::vector<Z> &u, const std::vector<Z> &v) {
  Z acc;
  for (size_t i = 0; i < u.size(); i++)
    if (!u[i].zero() && !v[i].zero()) acc = zadd(acc, zmul(conj(u[i]), v[i]));
  return acc;
}
// the most one gate changes the T bound: the sde of its Pauli-transfer matrix (spec.py ptm_sde)
int ptm_sde(const std::string &g) {
  const GateDef &G = gates().at(g);
  const int nq = G.arity(), N = 1 << nq;
  int qs[3] = {0, 1, 2};
  const Mat U = gate_matrix(G, qs, nq);
  std::vector<std::vector<Z>> cols(N, std::vector<Z>(N));
  for (int c = 0; c < N; c++)
    for (int r = 0; r < N; r++) cols[c][r] = U.at(r, c);
  int best = 0;
  for (int b = 0; b < (1 << (2 * nq)); b++) {
    std::vector<std::vector<Z>> PB(N);
    for (int c = 0; c < N; c++) {
      std::vector<Z> e(N);
      e[c] = Z{1, 0, 0, 0};
      PB[c] = pauli_apply(nq, b, e);
    }
    std::vector<std::vector<Z>> UPBc(N, std::vector<Z>(N));   // column c of U P_b
    for (int r = 0; r < N; r++)
      for (int c = 0; c < N; c++) {
        Z acc;
        for (int x = 0; x < N; x++) acc = zadd(acc, zmul(U.at(r, x), PB[c][x]));
        UPBc[c][r] = acc;
      }
    for (int a = 0; a < (1 << (2 * nq)); a++) {
      Z acc;
      for (int c = 0; c < N; c++) acc = zadd(acc, inner(cols[c], pauli_apply(nq, a, UPBc[c])));
      if (!acc.zero()) best = std::max(best, 2 * (nq + U.k) - val(acc));
    }
  }
  return best;
}

// State targets (spec.py:229-325): the goal side of the state bounds, per goal row (the image of one input basis
// state, over sqrt2^k): its sde, its stabilizer nullity and its Schmidt rank across every cut.

// least s >= 0 with sqrt2^s * (row / sqrt2^k) integral (spec.py row_sde)
int row_sde(int k, const std::vector<Z> &row) {
  int v = -1;
  for (const Z &x : row)
    if (!x.zero()) v = v < 0 ? val(x) : std::min(v, val(x));
  return std::max(0, k - std::max(v, 0));
}
// n - log2 of the number of Paulis P with P|v> = +-|v> (spec.py nullity; the identity always counts)
int nullity(int n, const std::vector<Z> &row) {
  const Z nrm = inner(row, row), neg{-nrm.a, -nrm.b, -nrm.c, -nrm.d};
  long long cnt = 0;
  for (int b = 0; b < (1 << (2 * n)); b++) {
    const Z v = inner(row, pauli_apply(n, b, row));
    cnt += v == nrm || v == neg;
  }
  int bits = 0;
  for (long long c = cnt; c; c >>= 1) bits++;
  return n - (bits - 1);
}
// exact determinant by cofactor expansion along the first row (zero entries skipped); only its zero test is used
Z det(const std::vector<std::vector<Z>> &M) {
  const size_t r = M.size();
  if (r == 1) return M[0][0];
  Z acc;
  for (size_t j = 0; j < r; j++) {
    if (M[0][j].zero()) continue;
    std::vector<std::vector<Z>> sub(r - 1);
    for (size_t i = 1; i < r; i++) {
      sub[i - 1].reserve(r - 1);
      for (size_t c = 0; c < r; c++)
        if (c != j) sub[i - 1].push_back(M[i][c]);
    }
    Z t = zmul(M[0][j], det(sub));
    if (j % 2) t = Z{-t.a, -t.b, -t.c, -t.d};
    acc = zadd(acc, t);
  }
  return acc;
}
// next r-subset of {0 .. m-1} in lexicographic order; false after the last
bool next_subset(std::vector<int> &s, int m) {
  const int r = (int)s.size();
  int i = r - 1;
  while (i >= 0 && s[i] == m - r + i) i--;
  if (i < 0) return false;
  s[i]++;
  for (int j = i + 1; j < r; j++) s[j] = s[j - 1] + 1;
  return true;
}
// rank of the state reshaped as (qubits A) x (the rest): the size of its largest nonzero minor (spec.py schmidt_rank)
int schmidt_rank(int n, const std::vector<int> &A, const std::vector<Z> &row) {
  std::vector<int> B;
  for (int q = 0; q < n; q++)
    if (std::find(A.begin(), A.end(), q) == A.end()) B.push_back(q);
  const int R = 1 << A.size(), C = 1 << B.size();
  std::vector<std::vector<Z>> M(R, std::vector<Z>(C));
  for (size_t x = 0; x < row.size(); x++) {
    int ia = 0, ib = 0;
    for (size_t i = 0; i < A.size(); i++) ia |= (int)((x >> A[i]) & 1) << i;
    for (size_t i = 0; i < B.size(); i++) ib |= (int)((x >> B[i]) & 1) << i;
    M[ia][ib] = row[x];
  }
  for (int r = std::min(R, C); r > 0; r--) {
    std::vector<int> rows(r);
    for (int i = 0; i < r; i++) rows[i] = i;
    do {
      std::vector<int> cols(r);
      for (int i = 0; i < r; i++) cols[i] = i;
      do {
        std::vector<std::vector<Z>> sub(r, std::vector<Z>(r));
        for (int i = 0; i < r; i++)
          for (int j = 0; j < r; j++) sub[i][j] = M[rows[i]][cols[j]];
        if (!det(sub).zero()) return r;
      } while (next_subset(cols, C));
    } while (next_subset(rows, R));
  }
  return 0;
}

// the parts of a spec that depend only on (n, gate set, W3 on/off), cached
struct GateSetPart {
  std::vector<Cand> cs;
  std::vector<std::vector<int>> cuts;
  std::string text;          // "standard" .. through the bad3 block
  std::string cuts_text;     // the "cuts" block
  std::string cx_text;       // "cxtable" .. "end"
  int nbad2 = 0, nbad3 = 0;
};
std::mutex cache_mu;
std::map<std::string, std::shared_ptr<const GateSetPart>> cache;

std::string zs(const Z &x) {
  return std::to_string(x.a) + " " + std::to_string(x.b) + " " + std::to_string(x.c) + " " + std::to_string(x.d);
}

std::shared_ptr<const GateSetPart> gate_set_part(int n, const std::vector<std::string> &gs, bool use3) {
  std::string key = std::to_string(n) + (use3 ? "|w3" : "|w2");
  for (const auto &g : gs) key += "|" + g;
  {
    std::lock_guard<std::mutex> lk(cache_mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  auto P = std::make_shared<GateSetPart>();
  P->cs = candidates(n, gs);
  std::vector<std::array<int, 2>> bad2;
  std::vector<std::array<int, 3>> bad3;
  sym_rules(P->cs, use3, bad2, bad3);
  P->nbad2 = (int)bad2.size();
  P->nbad3 = (int)bad3.size();
  static const std::set<std::string> STANDARD = {"x", "y", "z", "s", "sdg", "t", "tdg", "cx", "cz", "h"};
  bool standard = true, lite = true;
  for (const auto &g : gs) {
    standard = standard && STANDARD.count(g);
    lite = lite && (STANDARD.count(g) || g == "ccx");
  }
  lite = lite && !standard;
  int tdiv = 1;
  if (lite) {
    tdiv = 0;
    for (const auto &g : gs)
      if (g == "t" || g == "tdg" || g == "ccx") tdiv = std::max(tdiv, ptm_sde(g));
  }
  std::string &w = P->text;
  w += "standard " + std::to_string(standard ? 1 : 0) + "\n";
  if (lite) w += "lite 1\ntdiv " + std::to_string(tdiv) + "\n";
  w += "gates " + std::to_string(P->cs.size()) + "\n";
  for (const Cand &c : P->cs) {
    const GateDef &G = gates().at(c.g), &I = gates().at(dagger_name(c.g));
    w += c.name + " " + std::to_string(c.nq);
    for (int j = 0; j < c.nq; j++) w += " " + std::to_string(c.q[j]);
    w += " " + std::to_string(G.k);
    for (int l = 0; l < G.dim; l++)
      for (int m = 0; m < G.dim; m++) w += " " + zs(G.entry(l, m));
    w += " " + std::to_string(I.k);
    for (int l = 0; l < I.dim; l++)
      for (int m = 0; m < I.dim; m++) w += " " + zs(I.entry(l, m));
    w += "\n";
  }
  w += "bad2 " + std::to_string(bad2.size()) + "\n";
  for (const auto &p : bad2) w += std::to_string(p[0]) + " " + std::to_string(p[1]) + "\n";
  w += "bad3 " + std::to_string(bad3.size()) + "\n";
  for (const auto &t : bad3) w += std::to_string(t[0]) + " " + std::to_string(t[1]) + " " + std::to_string(t[2]) + "\n";
  P->cuts = cuts(n);
  const auto &cs = P->cuts;
  std::string &ct = P->cuts_text;
  ct += "cuts " + std::to_string(cs.size()) + "\n";
  for (const auto &A : cs) {
    ct += std::to_string(A.size());
    for (int q : A) ct += " " + std::to_string(q);
    ct += "\n";
  }
  std::string &tl = P->cx_text;
  std::vector<int> rad, best;
  if (!cx_table(n, cs, rad, best)) {
    tl += "cxtable 0\n";
  } else {
    tl += "cxtable " + std::to_string(best.size()) + "\n";
    for (size_t i = 0; i < best.size(); i++) tl += (i ? " " : "") + std::to_string(best[i]);
    tl += "\n";
  }
  tl += "end\n";
  std::lock_guard<std::mutex> lk(cache_mu);
  auto it = cache.emplace(key, P).first;
  return it->second;
}

// P_p on n qubits, digits per qubit (0 I, 1 X, 2 Y, 3 Z) at bits 2q (tcount.py pauli_matrix)
std::vector<Mat> pauli_mats(int n) {
  const int P = 1 << (2 * n), N = 1 << n;
  std::vector<Mat> paulis(P);
  for (int p = 0; p < P; p++) {
    Mat M;
    M.N = N;
    M.e.assign((size_t)N * N, Z{});
    for (int x = 0; x < N; x++) {
      int flip = 0, ph = 0;
      for (int q = 0; q < n; q++) {
        const int dg = (p >> (2 * q)) & 3, bit = (x >> q) & 1;
        if (dg == 1) flip |= 1 << q;
        else if (dg == 2) { flip |= 1 << q; ph += 2 + 4 * bit; }
        else if (dg == 3) ph += 4 * bit;
      }
      M.at(x ^ flip, x) = wpow(ph);
    }
    paulis[p] = M;
  }
  return paulis;
}
// the rotation tables (tcount.py pauli_tables): for each P_p (p >= 1) and Pauli c, (-1, 0) when they commute, else
// (r, sign) with i P_p P_c = sign P_r; false if some product is not a signed Pauli
bool rotation_block(int n, const std::vector<Mat> &paulis, std::string &out) {
  const int P = 1 << (2 * n);
  out += "rotations " + std::to_string(P - 1) + "\n";
  const Z iw{0, 0, 1, 0};
  for (int p = 1; p < P; p++) {
    for (int c = 0; c < P; c++) {
      const Mat M1 = matmul(paulis[p], paulis[c]), M2 = matmul(paulis[c], paulis[p]);
      int hr = -1, hs = 0;
      if (M1.e != M2.e) {
        std::vector<Z> M(M1.e.size());
        for (size_t i = 0; i < M.size(); i++) M[i] = zmul(iw, M1.e[i]);
        for (int r = 0; r < P && hr < 0; r++)
          for (int sign : {1, -1}) {
            bool eq = true;
            for (size_t i = 0; i < M.size() && eq; i++) {
              const Z &q = paulis[r].e[i];
              eq = M[i] == Z{sign * q.a, sign * q.b, sign * q.c, sign * q.d};
            }
            if (eq) { hr = r; hs = sign; }
          }
        if (hr < 0) return false;
      }
      out += (c ? " " : "") + std::to_string(hr) + " " + std::to_string(hs);
    }
    out += "\n";
  }
  return true;
}

// ---------- RUS specs (python/cheese/rus.py): roots of a two-qubit RUS circuit, table root, Clifford list ----------

// exact rationals (reduced, denominator > 0); numerators and denominators stay below 2^62 so products fit __int128
struct Rat { __int128 n = 0, d = 1; };
__int128 gcd128(__int128 a, __int128 b) {
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b) { const __int128 t = a % b; a = b; b = t; }
  return a;
}
Rat rat(__int128 n, __int128 d) {
  if (d == 0) throw std::overflow_error("division by zero");
  if (d < 0) { n = -n; d = -d; }
  const __int128 g = gcd128(n, d);
  if (g > 1) { n /= g; d /= g; }
  const __int128 lim = (__int128)1 << 62;
  if (n >= lim || n <= -lim || d >= lim) throw std::overflow_error("coefficient exceeds 62 bits");
  return {n, d};
}
Rat radd(const Rat &a, const Rat &b) { return rat(a.n * b.d + b.n * a.d, a.d * b.d); }
Rat rsub(const Rat &a, const Rat &b) { return rat(a.n * b.d - b.n * a.d, a.d * b.d); }
Rat rmul(const Rat &a, const Rat &b) { return rat(a.n * b.n, a.d * b.d); }
Rat rint(int64_t v) { return Rat{v, 1}; }
using QW = std::array<Rat, 4>;                     // an element of Q(w), coefficients of 1, w, w^2, w^3
QW qw(const Z &z) { return {rint(z.a), rint(z.b), rint(z.c), rint(z.d)}; }
QW qmul(const QW &x, const QW &y) {                // w^4 = -1
  QW o = {rint(0), rint(0), rint(0), rint(0)};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      const Rat p = rmul(x[i], y[j]);
      o[(i + j) % 4] = i + j < 4 ? radd(o[(i + j) % 4], p) : rsub(o[(i + j) % 4], p);
    }
  return o;
}
QW qup(const QW &z) { return {rsub(z[1], z[3]), radd(z[0], z[2]), radd(z[1], z[3]), rsub(z[2], z[0])}; }   // times sqrt2

// |z|^2 = A + B sqrt2 for z in Z[w]
std::pair<int64_t, int64_t> norm2(const Z &z) {
  return {chk((__int128)z.a * z.a + (__int128)z.b * z.b + (__int128)z.c * z.c + (__int128)z.d * z.d),
          chk((__int128)z.a * z.b + (__int128)z.b * z.c + (__int128)z.c * z.d - (__int128)z.a * z.d)};
}
// iteration order of the Python set {s, -s} (CPython: 8 slots, hash(v) = v except hash(-1) = -2, probe
// i = 5 i + 1 + perturb with perturb shifted right by 5), which orders the reference's norm solutions
std::vector<int64_t> py_pair_order(int64_t s) {
  if (s == 0) return {0};
  int64_t slot[8] = {0};
  bool used[8] = {false};
  for (int64_t v : {s, -s}) {
    const uint64_t h = (uint64_t)(v == -1 ? -2 : v);
    uint64_t i = h & 7, perturb = h;
    while (used[i]) { perturb >>= 5; i = (i * 5 + 1 + perturb) & 7; }
    used[i] = true;
    slot[i] = v;
  }
  std::vector<int64_t> out;
  for (int i = 0; i < 8; i++) if (used[i]) out.push_back(slot[i]);
  return out;
}
// every z in Z[w] with |z|^2 = A + B sqrt2, in the reference's enumeration order (rus.py norm_solutions)
std::vector<Z> norm_solutions(int64_t A, int64_t B) {
  if (A < 0) throw std::overflow_error("negative norm: not a RUS circuit");
  int64_t r = 0;
  while ((r + 1) * (r + 1) <= A) r++;
  r += 1;
  std::map<int64_t, int64_t> sq;
  for (int64_t i = 0; i <= r; i++) sq[i * i] = i;
  std::vector<Z> out;
  for (int64_t x0 = -r; x0 <= r; x0++)
    for (int64_t x1 = -r; x1 <= r; x1++)
      for (int64_t x2 = -r; x2 <= r; x2++) {
        auto it = sq.find(A - x0 * x0 - x1 * x1 - x2 * x2);
        if (it == sq.end()) continue;
        for (int64_t x3 : py_pair_order(it->second))
          if (x0 * x1 + x1 * x2 + x2 * x3 - x0 * x3 == B) out.push_back(Z{x0, x1, x2, x3});
      }
  return out;
}

// a Pauli transfer matrix of a 4 x 2 isometry: 16 x 4 entries (x + y sqrt2) / sqrt2^e
struct Ptm {
  int e = 0;
  std::vector<std::array<int64_t, 2>> v;           // row-major 16 x 4
};
// Jc[a][b] = Tr(P_a J P_b J^dag) / 2, normalised (rus.py ptm); J is 4 x 2 over sqrt2^k, row 2 i + ancilla
Ptm ptm(const std::vector<Z> &J, int k) {
  const std::vector<Mat> P16 = pauli_mats(2), P1 = pauli_mats(1);
  Ptm X;
  X.v.resize(64);
  for (int b = 0; b < 4; b++) {
    Z A[4][4];                                      // J P_b J^dag, over sqrt2^(2k)
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) {
        Z acc;
        for (int i = 0; i < 2; i++)
          for (int j = 0; j < 2; j++) {
            const Z &p = P1[b].at(i, j);
            if (p.zero() || J[r * 2 + i].zero() || J[c * 2 + j].zero()) continue;
            acc = zadd(acc, zmul(zmul(J[r * 2 + i], p), conj(J[c * 2 + j])));
          }
        A[r][c] = acc;
      }
    for (int a = 0; a < 16; a++) {
      Z tr;
      for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
          if (!P16[a].at(r, c).zero() && !A[c][r].zero()) tr = zadd(tr, zmul(P16[a].at(r, c), A[c][r]));
      if (tr.c != 0 || tr.d != -tr.b) throw std::overflow_error("transfer-matrix entry not real");
      X.v[a * 4 + b] = {tr.a, tr.b};
    }
  }
  X.e = 2 * k + 2;                                  // the trace's sqrt2^(2k) and the 1/2
  while (X.e > 0) {
    bool even = true;
    for (const auto &t : X.v) even = even && (t[0] % 2 == 0);
    if (!even) break;
    for (auto &t : X.v) t = {t[1], t[0] / 2};       // (x + y s) / s = y + (x / 2) s
    X.e--;
  }
  return X;
}

// the 11520 two-qubit Cliffords mod phase as row actions C^dag P_a C = s P_pi(a), in breadth-first order over the
// generators h q0, h q1, s q0, s q1, cz (rus.py cliffords)
struct CliffordList {
  std::vector<std::array<int8_t, 16>> perm, sign;
  std::map<std::array<int, 4>, int> bygen;          // images (row, sign) of X_q0, Z_q0, X_q1, Z_q1 -> index
};
const CliffordList &clifford_list() {
  static const CliffordList L = [] {
    CliffordList out;
    const std::vector<Mat> P16 = pauli_mats(2);
    const std::pair<const char *, std::array<int, 2>> gens[5] = {
        {"h", {0, -1}}, {"h", {1, -1}}, {"s", {0, -1}}, {"s", {1, -1}}, {"cz", {0, 1}}};
    std::vector<std::array<int8_t, 16>> gp(5), gs(5);
    for (int g = 0; g < 5; g++) {
      const Mat C = gate_matrix(gates().at(gens[g].first), gens[g].second.data(), 2), Cd = dagger(C);
      for (int a = 0; a < 16; a++) {
        const Mat A = matmul(matmul(Cd, P16[a]), C);
        int hb = -1, hs = 0;
        for (int b = 0; b < 16 && hb < 0; b++)
          for (int sg : {1, -1}) {
            bool eq = true;
            for (size_t i = 0; i < A.e.size() && eq; i++) {
              const Z &q = P16[b].e[i];
              eq = A.e[i] == Z{sg * q.a, sg * q.b, sg * q.c, sg * q.d};
            }
            if (eq && hb < 0) { hb = b; hs = sg; }
          }
        if (hb < 0) throw std::logic_error("Clifford generator does not map Paulis to Paulis");
        gp[g][a] = (int8_t)hb;
        gs[g][a] = (int8_t)hs;
      }
    }
    std::array<int8_t, 16> ip, is;
    for (int a = 0; a < 16; a++) { ip[a] = (int8_t)a; is[a] = 1; }
    std::set<std::pair<std::array<int8_t, 16>, std::array<int8_t, 16>>> seen{{ip, is}};
    out.perm.push_back(ip); out.sign.push_back(is);
    std::vector<size_t> frontier{0};
    while (!frontier.empty()) {
      std::vector<size_t> nxt;
      for (size_t f : frontier)
        for (int g = 0; g < 5; g++) {               // G C: (G C)^dag P (G C) = C^dag (G^dag P G) C
          std::array<int8_t, 16> bp, bs;
          for (int x = 0; x < 16; x++) {
            bp[x] = out.perm[f][gp[g][x]];
            bs[x] = (int8_t)(gs[g][x] * out.sign[f][gp[g][x]]);
          }
          if (seen.insert({bp, bs}).second) {
            out.perm.push_back(bp); out.sign.push_back(bs);
            nxt.push_back(out.perm.size() - 1);
          }
        }
      frontier = nxt;
    }
    if (out.perm.size() != 11520) throw std::logic_error("two-qubit Clifford group order");
    const int G4[4] = {1, 3, 4, 12};
    for (size_t c = 0; c < out.perm.size(); c++) {
      std::array<int, 4> key;
      for (int g = 0; g < 4; g++) key[g] = out.perm[c][G4[g]] * 2 + (out.sign[c][G4[g]] < 0);
      out.bygen.emplace(key, (int)c);
    }
    return out;
  }();
  return L;
}
// some Clifford c with B = C_c A (B[x] = s_c(x) A[pi_c(x)] for every row)
bool ptm_equivalent(const Ptm &A, const Ptm &B) {
  if (A.e != B.e) return false;
  const CliffordList &L = clifford_list();
  auto row_eq = [&](int ra, int s, int rb) {
    for (int c = 0; c < 4; c++)
      if (s * A.v[ra * 4 + c][0] != B.v[rb * 4 + c][0] || s * A.v[ra * 4 + c][1] != B.v[rb * 4 + c][1]) return false;
    return true;
  };
  const int G4[4] = {1, 3, 4, 12};
  std::vector<int> cand[4];
  for (int g = 0; g < 4; g++) {
    for (int r = 1; r < 16; r++)
      for (int s : {1, -1})
        if (row_eq(r, s, G4[g])) cand[g].push_back(r * 2 + (s < 0));
    if (cand[g].empty()) return false;
  }
  for (int i0 : cand[0]) for (int i1 : cand[1]) for (int i2 : cand[2]) for (int i3 : cand[3]) {
    auto it = L.bygen.find({i0, i1, i2, i3});
    if (it == L.bygen.end()) continue;
    const int c = it->second;
    bool ok = true;
    for (int x = 0; x < 16 && ok; x++) ok = row_eq(L.perm[c][x], L.sign[c][x], x);
    if (ok) return true;
  }
  return false;
}

// 1 x 1 normal form of A when A is a multiple of the identity (rus.py scalar)
bool scalar(const Mat &A, int &k, Z &z) {
  for (int r = 0; r < A.N; r++)
    for (int c = 0; c < A.N; c++)
      if (r != c ? !A.at(r, c).zero() : A.at(r, c) != A.at(0, 0)) return false;
  Mat S;
  S.N = 1; S.k = A.k; S.e = {A.at(0, 0)};
  normalise(S);
  k = S.k;
  z = S.e[0];
  return true;
}
// B / sqrt2^k proportional to a one-qubit Clifford: B B^dag = q I and B P B^dag Q = +-q I (rus.py clifford_block)
bool clifford_block(const Mat &B) {
  int kg;
  Z zg;
  if (!scalar(matmul(B, dagger(B)), kg, zg) || zg.zero()) return false;
  const std::vector<Mat> P1 = pauli_mats(1);
  for (int p : {1, 3}) {
    const Mat A = matmul(matmul(B, P1[p]), dagger(B));
    bool any = false;
    for (int q : {1, 2, 3}) {
      int k;
      Z z;
      if (scalar(matmul(A, P1[q]), k, z) && k == kg && (z == zg || z == Z{-zg.a, -zg.b, -zg.c, -zg.d})) any = true;
    }
    if (!any) return false;
  }
  return true;
}

int check_circuit(int n, const std::vector<CircGate> &circ, std::string &err) {
  if (n < 1 || n > 6) { err = "n = " + std::to_string(n) + " out of range (1..6)"; return 2; }
  for (const CircGate &g : circ) {
    auto it = gates().find(g.g);
    if (it == gates().end()) { err = "unknown gate " + g.g; return 2; }
    if (g.nq != it->second.arity()) { err = "gate " + g.g + " needs " + std::to_string(it->second.arity()) + " qubits"; return 2; }
    for (int j = 0; j < g.nq; j++) {
      if (g.q[j] < 0 || g.q[j] >= n) { err = "qubit " + std::to_string(g.q[j]) + " out of range"; return 2; }
      for (int i = 0; i < j; i++)
        if (g.q[i] == g.q[j]) { err = "gate " + g.g + " repeats qubit " + std::to_string(g.q[j]); return 2; }
    }
  }
  return 0;
}

}  // namespace

int parse_qasm(const char *text, size_t len, int &n, std::vector<CircGate> &circ, std::string &err) {
  n = 0;
  circ.clear();
  size_t pos = 0;
  while (pos < len) {
    size_t e = pos;
    while (e < len && text[e] != '\n') e++;
    std::string line(text + pos, e - pos);
    pos = e + 1;
    const size_t cm = line.find("//");
    if (cm != std::string::npos) line = line.substr(0, cm);
    size_t a = 0, b = line.size();
    while (a < b && isspace((unsigned char)line[a])) a++;
    while (b > a && isspace((unsigned char)line[b - 1])) b--;
    line = line.substr(a, b - a);
    auto digits_in_brackets = [](const std::string &s, size_t from, int &v, size_t &end) {
      if (from >= s.size() || s[from] != '[') return false;
      size_t i = from + 1;
      if (i >= s.size() || !isdigit((unsigned char)s[i])) return false;
      long x = 0;
      while (i < s.size() && isdigit((unsigned char)s[i])) x = x * 10 + (s[i++] - '0');
      if (i >= s.size() || s[i] != ']') return false;
      v = (int)x;
      end = i + 1;
      return true;
    };
    int v;
    size_t end;
    if (line.compare(0, 4, "qreg") == 0 && line.size() > 4 && isspace((unsigned char)line[4])) {
      size_t i = 4;
      while (i < line.size() && isspace((unsigned char)line[i])) i++;
      const size_t w0 = i;
      while (i < line.size() && (isalnum((unsigned char)line[i]) || line[i] == '_')) i++;
      if (i > w0 && digits_in_brackets(line, i, v, end)) { n = v; continue; }
    }
    if (line.compare(0, 5, "qubit") == 0 && digits_in_brackets(line, 5, v, end)) { n = v; continue; }
    size_t i = 0;
    while (i < line.size() && line[i] >= 'a' && line[i] <= 'z') i++;
    if (i == 0 || i >= line.size() || !isspace((unsigned char)line[i])) continue;
    const std::string g = line.substr(0, i);
    const size_t semi = line.rfind(';');
    if (semi == std::string::npos || semi < i) continue;
    if (!gates().count(g)) continue;
    CircGate cg;
    cg.g = g;
    const std::string args = line.substr(i, semi - i);
    for (size_t k = 0; k < args.size(); k++) {
      if (args[k] != '[') continue;
      if (digits_in_brackets(args, k, v, end)) {
        if (cg.nq < 3) cg.q[cg.nq] = v;
        cg.nq++;
        k = end - 1;
      }
    }
    circ.push_back(cg);
  }
  if (n <= 0) { err = "no qubit register"; return 2; }
  return check_circuit(n, circ, err);
}

int spec_generate(int n, const std::vector<CircGate> &circ, int depth, bool use_w3, const std::vector<int> &inputs,
                  std::string &out, SpecGenInfo &info, std::string &err) {
  try {
    if (int rc = check_circuit(n, circ, err)) return rc;
    const int N = 1 << n, m = (int)inputs.size();
    if (m > N) { err = std::to_string(m) + " inputs for " + std::to_string(N) + " basis states"; return 2; }
    for (int x : inputs)
      if (x < 0 || x >= N) { err = "input " + std::to_string(x) + " out of range"; return 2; }
    std::set<std::string> gs = {"x", "z", "h", "s", "sdg", "t", "tdg", "cx"};
    for (const CircGate &g : circ) gs.insert(g.g);
    const std::vector<std::string> gl(gs.begin(), gs.end());   // byte order, as Python's sorted()
    const auto P = gate_set_part(n, gl, use_w3);
    const Mat U = unitary(n, circ);
    auto block = [&](const Mat &M) {
      std::string t = std::to_string(M.k) + "\n";
      for (int r = 0; r < M.N; r++) {
        for (int c = 0; c < M.N; c++) t += (c ? " " : "") + zs(M.at(r, c));
        t += "\n";
      }
      return t;
    };
    out = "cheese-spec 1\nn " + std::to_string(n) + "\nmode " + (m ? "states" : "unitary") + "\nphase exact\ndepth " +
          std::to_string(depth) + "\n";
    out += P->text;
    if (!m) {
      out += "target " + block(U);
      out += P->cuts_text;
    } else {
      // start rows e_x and goal rows U e_x (the transposed images, spec.py state_pairs), zero rows up to N; the goal
      // rows share one exponent, normalised together
      Mat S, G;
      S.N = G.N = N;
      S.e.assign((size_t)N * N, Z{});
      G.e.assign((size_t)N * N, Z{});
      G.k = U.k;
      for (int j = 0; j < m; j++) {
        S.at(j, inputs[j]) = Z{1, 0, 0, 0};
        for (int r = 0; r < N; r++) G.at(j, r) = U.at(r, inputs[j]);
      }
      normalise(G);
      out += "pairs " + std::to_string(m) + "\n";
      out += "start " + block(S);
      out += "target " + block(G);
      out += P->cuts_text;
      out += "goal " + std::to_string(m) + "\n";
      for (int j = 0; j < m; j++) {
        const std::vector<Z> row(G.e.begin() + (size_t)j * N, G.e.begin() + (size_t)(j + 1) * N);
        out += std::to_string(row_sde(G.k, row)) + " " + std::to_string(nullity(n, row));
        for (const auto &A : P->cuts) out += " " + std::to_string(schmidt_rank(n, A, row));
        out += "\n";
      }
    }
    out += P->cx_text;
    info.candidates = (int)P->cs.size();
    info.bad2 = P->nbad2;
    info.bad3 = P->nbad3;
    return 0;
  } catch (const std::overflow_error &e) {
    err = e.what();
    return 2;
  }
}

int tspec_generate(int n, const std::vector<CircGate> &circ, std::string &out, std::string &err) {
  try {
    if (int rc = check_circuit(n, circ, err)) return rc;
    if (n > 4) { err = "T-count specs for n <= 4"; return 2; }
    const Mat U = unitary(n, circ);
    const int P = 1 << (2 * n), N = 1 << n;
    const std::vector<Mat> paulis = pauli_mats(n);
    // channel: Uc[a][b] = Tr(P_a U P_b U^dag) / 2^n = (x + y sqrt2) / sqrt2^e, one exponent for the matrix
    const Mat Ud = dagger(U);
    std::vector<int> ks((size_t)P * P);
    std::vector<std::array<int64_t, 2>> xy((size_t)P * P);
    int kmax = 0;
    for (int b = 0; b < P; b++) {
      const Mat A = matmul(matmul(U, paulis[b]), Ud);
      for (int a = 0; a < P; a++) {
        const Mat T = matmul(paulis[a], A);
        Z tr;
        for (int i = 0; i < N; i++) tr = zadd(tr, T.at(i, i));
        if (tr.c != 0 || tr.d != -tr.b) { err = "channel entry not real"; return 2; }
        ks[(size_t)a * P + b] = T.k;
        xy[(size_t)a * P + b] = {tr.a, tr.b};
        kmax = std::max(kmax, T.k);
      }
    }
    int E = kmax + 2 * n;
    for (size_t i = 0; i < xy.size(); i++)
      for (int s = 0; s < E - 2 * n - ks[i]; s++) xy[i] = {chk((__int128)2 * xy[i][1]), xy[i][0]};   // times sqrt2
    while (E > 0) {
      bool even = true;
      for (const auto &v : xy) even = even && (v[0] % 2 == 0);
      if (!even) break;
      for (auto &v : xy) v = {v[1], v[0] / 2};                                                      // over sqrt2
      E--;
    }
    out = "tcount-spec 1\nn " + std::to_string(n) + "\nchannel " + std::to_string(E) + "\n";
    for (int a = 0; a < P; a++) {
      for (int b = 0; b < P; b++)
        out += (b ? " " : "") + std::to_string(xy[(size_t)a * P + b][0]) + " " + std::to_string(xy[(size_t)a * P + b][1]);
      out += "\n";
    }
    // rotation tables: for each P_p (p >= 1) and Pauli c, (-1, 0) when they commute, else (r, sign) with
    // i P_p P_c = sign P_r
    if (!rotation_block(n, paulis, out)) { err = "i P Q is not a signed Pauli"; return 2; }
    out += "end\n";
    return 0;
  } catch (const std::overflow_error &e) {
    err = e.what();
    return 2;
  }
}

int rspec_generate(int n, const std::vector<CircGate> &circ, const std::string &qasm_text, int outcome,
                   std::string &out, RusSpecInfo &info, std::string &err) {
  try {
    if (int rc = check_circuit(n, circ, err)) return rc;
    if (n != 2) { err = "RUS mode: two qubits (q0 ancilla, measured; q1 data)"; return 2; }
    const Mat W = unitary(n, circ);
    // blocks B_o[i][j] = <o, i| W |0, j> (ancilla q0 = bit 0 of an index)
    Mat Bk[2];
    for (int o = 0; o < 2; o++) {
      Bk[o].N = 2; Bk[o].k = W.k; Bk[o].e.assign(4, Z{});
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) Bk[o].at(i, j) = W.at(o + 2 * i, 2 * j);
    }
    int ks = outcome;
    if (ks < 0) {                                   // a "success outcome K" comment, else the non-Clifford branch
      const size_t at = qasm_text.find("success outcome ");
      if (at != std::string::npos && at + 16 < qasm_text.size() && isdigit((unsigned char)qasm_text[at + 16])) {
        ks = qasm_text[at + 16] - '0';
      } else {
        const bool c0 = clifford_block(Bk[0]), c1 = clifford_block(Bk[1]);
        if (c0 == c1) { err = "not a RUS circuit: need exactly one branch proportional to a Clifford"; return 2; }
        ks = c0 ? 1 : 0;
      }
    }
    if (ks != 0 && ks != 1) { err = "success outcome must be 0 or 1"; return 2; }
    const Mat &M = Bk[ks];
    const int kW = W.k, m = kW + 1;                 // Pr[success] = (A + B sqrt2) / 2^m
    int64_t A = 0, Bs = 0;
    for (const Z &z : M.e) { const auto nz = norm2(z); A = chk((__int128)A + nz.first); Bs = chk((__int128)Bs + nz.second); }
    if (m > 60) { err = "coefficient overflow"; return 2; }
    std::vector<Z> gam = norm_solutions(((int64_t)1 << m) - A, -Bs);   // gamma = g / sqrt2^m, |gamma|^2 = 1 - p
    // one gamma per orbit {w^k gamma}: keyed by the smallest w^k gamma, first position, last value (a Python dict)
    std::vector<std::pair<std::array<int64_t, 4>, Z>> orbit;
    for (const Z &g : gam) {
      std::array<int64_t, 4> key{};
      for (int k = 0; k < 8; k++) {
        const Z r = zmul(wpow(k), g);
        const std::array<int64_t, 4> t{r.a, r.b, r.c, r.d};
        if (k == 0 || t < key) key = t;
      }
      auto it = std::find_if(orbit.begin(), orbit.end(), [&](const auto &e) { return e.first == key; });
      if (it == orbit.end()) orbit.push_back({key, g}); else it->second = g;
    }
    // rescalings u = h / m0 (|u| = 1) that keep u M exact
    Z m0;
    for (const Z &z : M.e) if (!z.zero()) { m0 = z; break; }
    if (m0.zero()) { err = "zero success block"; return 2; }
    const auto nm = norm2(m0);
    const Rat d = rat((__int128)nm.first * nm.first - (__int128)2 * nm.second * nm.second, 1);
    const Rat invd = rat(d.d, d.n);                 // 1 / |m0|^2 = (a0 - b0 sqrt2) / (a0^2 - 2 b0^2)
    const QW inv = {rmul(rint(nm.first), invd), rmul(rint(-nm.second), invd), rint(0), rmul(rint(nm.second), invd)};
    std::vector<QW> us;
    for (const Z &h : norm_solutions(nm.first, nm.second)) {
      const QW u = qmul(qmul(qw(h), qw(conj(m0))), inv);
      bool exact = true;
      for (const Z &z : M.e) {
        const QW v = qmul(u, qw(z));
        for (const Rat &c : v) exact = exact && ((c.d & (c.d - 1)) == 0);
      }
      if (exact) us.push_back(u);
    }
    // one-qubit Cliffords mod phase, one per coset of the left Paulis (6 of 24), in breadth-first order over h, s
    const std::vector<Mat> P1 = pauli_mats(1);
    auto phase_key = [](const Mat &U) {             // min over global phases of the entries, then the exponent
      std::vector<int64_t> best;
      for (int ph = 0; ph < 8; ph++) {
        std::vector<int64_t> t;
        for (const Z &x : U.e) { const Z r = zmul(wpow(ph), x); t.insert(t.end(), {r.a, r.b, r.c, r.d}); }
        if (ph == 0 || t < best) best = t;
      }
      best.push_back(U.k);
      return best;
    };
    const int q0[1] = {0};
    const Mat Hg = gate_matrix(gates().at("h"), q0, 1), Sg = gate_matrix(gates().at("s"), q0, 1);
    std::vector<Mat> D1, fr{identity(2)};
    std::set<std::vector<int64_t>> allD, seenD;
    while (!fr.empty()) {
      std::vector<Mat> nx;
      for (const Mat &U : fr) {
        if (!allD.insert(phase_key(U)).second) continue;
        nx.push_back(matmul(Hg, U));
        nx.push_back(matmul(Sg, U));
        std::vector<int64_t> coset;
        for (int q = 0; q < 4; q++) {
          const std::vector<int64_t> k = phase_key(matmul(P1[q], U));
          if (q == 0 || k < coset) coset = k;
        }
        if (seenD.insert(coset).second) D1.push_back(U);
      }
      fr = nx;
    }
    if (allD.size() != 24 || D1.size() != 6) { err = "one-qubit Clifford enumeration"; return 2; }
    // roots: success block u M (outcome moved to 0), failure block gamma D, distinct up to left Cliffords
    std::vector<Ptm> roots;
    for (const QW &u : us)
      for (const auto &og : orbit)
        for (const Mat &D : D1) {
          QW vals[8];
          for (int i = 0; i < 2; i++)
            for (int anc = 0; anc < 2; anc++)
              for (int j = 0; j < 2; j++) {
                QW v;
                int k;
                if (anc == 0) { v = qmul(u, qw(M.at(i, j))); k = kW; }
                else { v = qw(zmul(og.second, D.at(i, j))); k = m + D.k; }
                for (int t = 0; t < k; t++) {
                  v = qup(v);
                  for (Rat &c : v) c = rat(c.n, c.d * 2);
                }
                vals[4 * i + 2 * anc + j] = v;
              }
          int E = 0;
          for (;;) {
            bool integral = true;
            for (const QW &v : vals) for (const Rat &c : v) integral = integral && c.d == 1;
            if (integral) break;
            for (QW &v : vals) v = qup(v);
            if (++E > 200) { err = "coefficient overflow"; return 2; }
          }
          std::vector<Z> J(8);
          for (int r = 0; r < 8; r++) J[r] = Z{(int64_t)vals[r][0].n, (int64_t)vals[r][1].n, (int64_t)vals[r][2].n,
                                               (int64_t)vals[r][3].n};
          const Ptm X = ptm(J, E);
          bool fresh = true;
          for (const Ptm &Y : roots) fresh = fresh && !ptm_equivalent(Y, X);
          if (fresh) roots.push_back(X);
        }
    auto mat = [](const Ptm &X) {
      std::string t = std::to_string(X.e) + "\n";
      for (int a = 0; a < 16; a++) {
        for (int b = 0; b < 4; b++)
          t += (b ? " " : "") + std::to_string(X.v[a * 4 + b][0]) + " " + std::to_string(X.v[a * 4 + b][1]);
        t += "\n";
      }
      return t;
    };
    std::vector<Z> j00(8);
    j00[0] = Z{1, 0, 0, 0};                         // J00 = |0> x I: row 2 i + 0, column i
    j00[5] = Z{1, 0, 0, 0};
    out = "rus-spec 1\ntable-root\n" + mat(ptm(j00, 0));
    out += "roots " + std::to_string(roots.size()) + "\n";
    for (const Ptm &X : roots) out += mat(X);
    if (!rotation_block(2, pauli_mats(2), out)) { err = "i P Q is not a signed Pauli"; return 2; }
    const CliffordList &L = clifford_list();
    out += "cliffords " + std::to_string(L.perm.size()) + "\n";
    for (size_t c = 0; c < L.perm.size(); c++) {
      for (int x = 0; x < 16; x++) out += (x ? " " : "") + std::to_string(L.perm[c][x]) + " " + std::to_string(L.sign[c][x]);
      out += "\n";
    }
    out += "end\n";
    info.outcome = ks;
    info.roots = (int)roots.size();
    info.p[0] = A; info.p[1] = Bs; info.p[2] = m;
    info.rescalings = (int)us.size();
    info.failure_amplitudes = (int)orbit.size();
    return 0;
  } catch (const std::overflow_error &e) {
    err = e.what();
    return 2;
  }
}

}  // namespace cz
