// Spec parsing, symmetry group and gate properties (host side of the boundary).
#include "cz_spec.h"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <atomic>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

namespace cz {

namespace {

// whitespace tokenizer with std::istream-like failure: a failed numeric read poisons the stream
struct Reader {
  const char *p, *end;
  bool fail = false;
  bool tok(std::string &s) {
    while (p < end && std::isspace((unsigned char)*p)) p++;
    if (p >= end) return false;
    const char *b = p;
    while (p < end && !std::isspace((unsigned char)*p)) p++;
    s.assign(b, p);
    return true;
  }
  int64_t num() {
    std::string s;
    if (fail || !tok(s)) { fail = true; return 0; }
    char *e;
    const long long v = std::strtoll(s.c_str(), &e, 10);
    if (e == s.c_str()) { fail = true; return 0; }
    return v;
  }
  Zw zw() { Zw z; z.a = num(); z.b = num(); z.c = num(); z.d = num(); return z; }
};

// local Pauli P_b (digits per qubit: 0 I, 1 X, 2 Y, 3 Z): column x has w^phase at row x ^ flip
void pauli_local(int b, int nq, std::vector<Zw> &M) {
  const int L = 1 << nq;
  M.assign(L * L, Zw{0, 0, 0, 0});
  int flip = 0, ym = 0, zm = 0;
  for (int q = 0; q < nq; q++) {
    const int d = (b >> (2 * q)) & 3;
    if (d == 1 || d == 2) flip |= 1 << q;
    if (d == 2) ym |= 1 << q;
    if (d == 3) zm |= 1 << q;
  }
  for (int x = 0; x < L; x++)
    M[(x ^ flip) * L + x] = zwpow(2 * __builtin_popcount(ym) + 4 * __builtin_popcount(x & (ym | zm)));
}

// A is Clifford iff A P A^dag is a scalar times a Pauli for every local Pauli P (exact over Z[w])
bool is_clifford(const std::array<Zw, LMAX * LMAX> &A, int nq) {
  const int L = 1 << nq, P = 1 << (2 * nq);
  std::vector<Zw> Pb, Q, B(L * L), AP(L * L);
  for (int b = 1; b < P; b++) {
    pauli_local(b, nq, Pb);
    for (int r = 0; r < L; r++)
      for (int c = 0; c < L; c++) {
        Zw acc{0, 0, 0, 0};
        for (int m = 0; m < L; m++) acc = zadd(acc, zmul(A[r * L + m], Pb[m * L + c]));
        AP[r * L + c] = acc;
      }
    for (int r = 0; r < L; r++)
      for (int c = 0; c < L; c++) {
        Zw acc{0, 0, 0, 0};
        for (int m = 0; m < L; m++) acc = zadd(acc, zmul(AP[r * L + m], zconj(A[c * L + m])));
        B[r * L + c] = acc;
      }
    bool found = false;
    for (int q = 1; q < P && !found; q++) {      // B Q^dag = s I with s != 0
      pauli_local(q, nq, Q);
      Zw s{0, 0, 0, 0};
      bool ok = true;
      for (int r = 0; r < L && ok; r++)
        for (int c = 0; c < L && ok; c++) {
          Zw acc{0, 0, 0, 0};
          for (int m = 0; m < L; m++) acc = zadd(acc, zmul(B[r * L + m], zconj(Q[c * L + m])));
          if (r == c) { if (r == 0) s = acc; else ok = zeq(acc, s); }
          else ok = zzero(acc);
        }
      found = ok && !zzero(s);
    }
    if (!found) return false;
  }
  return true;
}

// monomial (one nonzero per row and column) with a permutation that is affine over GF(2)
bool is_monomial_affine(const std::array<Zw, LMAX * LMAX> &A, int nq) {
  const int L = 1 << nq;
  int pi[LMAX];
  for (int c = 0; c < L; c++) {
    int nz = 0;
    for (int r = 0; r < L; r++) if (!zzero(A[r * L + c])) { nz++; pi[c] = r; }
    if (nz != 1) return false;
  }
  for (int j = 0; j < L; j++) {
    int x = pi[0];
    for (int i = 0; i < nq; i++) if ((j >> i) & 1) x ^= pi[1 << i] ^ pi[0];
    if (pi[j] != x) return false;
  }
  return true;
}

// w-power p of a unit z = w^p, -1 otherwise
int unit_power(const Zw &z) {
  const int64_t c[4] = {z.a, z.b, z.c, z.d};
  int nz = -1;
  for (int i = 0; i < 4; i++) if (c[i]) { if (nz >= 0) return -1; nz = i; }
  if (nz < 0) return -1;
  if (c[nz] == 1) return nz;
  if (c[nz] == -1) return nz + 4;
  return -1;
}

// rank over F_p (p = 998244353, w -> 3^((p-1)/8)) of a two-qubit gate reshaped across its two qubits
int schmidt_rank_p(const std::array<Zw, LMAX * LMAX> &A) {
  const uint64_t P = PRIME;
  auto pw = [&](uint64_t b, uint64_t e) { uint64_t r = 1; b %= P; while (e) { if (e & 1) r = r * b % P; b = b * b % P; e >>= 1; } return r; };
  const uint64_t w = pw(3, (P - 1) / 8), w2 = w * w % P, w3 = w2 * w % P;
  auto md = [&](int64_t v) { int64_t m = v % (int64_t)P; return (uint64_t)(m < 0 ? m + (int64_t)P : m); };
  uint64_t M[4][4];
  for (int o = 0; o < 4; o++)
    for (int i = 0; i < 4; i++) {
      const Zw z = A[o * 4 + i];
      M[((o & 1) << 1) | (i & 1)][(((o >> 1) & 1) << 1) | ((i >> 1) & 1)] =
          (md(z.a) + md(z.b) * w % P + md(z.c) * w2 % P + md(z.d) * w3 % P) % P;
    }
  int rank = 0;
  for (int c = 0; c < 4 && rank < 4; c++) {
    int piv = -1;
    for (int r = rank; r < 4; r++) if (M[r][c]) { piv = r; break; }
    if (piv < 0) continue;
    for (int j = 0; j < 4; j++) std::swap(M[piv][j], M[rank][j]);
    const uint64_t inv = pw(M[rank][c], P - 2);
    for (int r = rank + 1; r < 4; r++) {
      const uint64_t f = M[r][c] * inv % P;
      for (int j = 0; j < 4; j++) M[r][j] = (M[r][j] + P - f * M[rank][j] % P) % P;
    }
    rank++;
  }
  return rank;
}

}  // namespace

int parse_spec(const char *text, size_t len, HostSpec &s, std::string &err) {
  static std::atomic<uint64_t> next_uid{1};
  s = HostSpec{};
  s.uid = next_uid++;
  Reader in{text, text + len};
  std::string tok;
  bool have_start = false, have_goal_rows = false, have_ginfo = false;
  if (!in.tok(tok) || tok != "cheese-spec") { err = "not a spec"; return RC_SPEC; }
  (void)in.num();
  while (!in.fail && in.tok(tok)) {
    if (tok == "n") s.n = (int)in.num();
    else if (tok == "mode" || tok == "phase") {
      std::string v;
      if (!in.tok(v)) break;
      if (v == "states") s.states = 1;
      else if (v != "unitary" && v != "exact") { err = "unsupported " + tok + " " + v; return RC_SPEC; }
    } else if (tok == "pairs") s.m = (int)in.num();
    else if (tok == "start") {                 // state targets: the rows e_in_j (the residual's start)
      const int k = (int)in.num();
      if (s.n < 1 || s.n > NQMAX) { in.fail = true; break; }
      const int N = 1 << s.n;
      s.target.assign((size_t)N * N, Zw{0, 0, 0, 0});
      for (int i = 0; i < N * N; i++) s.target[i] = in.zw();
      s.tk = k;
      have_start = true;
    } else if (tok == "goal") {                // state targets: per pair sde, nullity, Schmidt rank per cut
      const int m = (int)in.num();
      const int w = 2 + (int)s.cutmask.size();
      s.ginfo.assign((size_t)std::max(0, m * w), 0);
      for (int i = 0; i < m * w; i++) s.ginfo[i] = (int)in.num();
      have_ginfo = m * w > 0;
    } else if (tok == "depth") s.depth = (int)in.num();
    else if (tok == "standard") s.standard = (int)in.num();
    else if (tok == "lite") s.lite = (int)in.num();
    else if (tok == "tdiv") s.tdiv = (int)in.num();
    else if (tok == "gates") {
      s.G = (int)in.num();
      if (s.G > GMAX) { err = "too many gates"; return RC_SPEC; }
      if (s.G < 0) { in.fail = true; break; }
      for (int g = 0; g < s.G && !in.fail; g++) {
        std::string name;
        if (!in.tok(name)) { in.fail = true; break; }
        const int nq = (int)in.num();
        if (nq < 1 || nq > 3) { in.fail = true; break; }
        std::array<int, 3> q{0, 0, 0};
        for (int j = 0; j < nq; j++) q[j] = (int)in.num();
        const int L = 1 << nq;
        const int fk = (int)in.num();                   // forward exponent and matrix
        std::array<Zw, LMAX * LMAX> fwd{};
        for (int i = 0; i < L * L; i++) fwd[i] = in.zw();
        int ik = (int)in.num();
        std::array<Zw, LMAX * LMAX> inv{};
        for (int i = 0; i < L * L; i++) inv[i] = in.zw();
        if (s.states) {          // rows are images of the inputs (transposed): a gate multiplies them by its transpose
          ik = fk;
          for (int a = 0; a < L; a++)
            for (int b = 0; b < L; b++) inv[a * L + b] = fwd[b * L + a];
        }
        s.names.push_back(name); s.gnq.push_back(nq); s.gq.push_back(q); s.gik.push_back(ik); s.ginv.push_back(inv);
      }
    } else if (tok == "bad2") {
      const int m = (int)in.num();
      s.bad2.assign((size_t)s.G * s.G, 0);
      for (int i = 0; i < m && !in.fail; i++) {
        const int a = (int)in.num(), b = (int)in.num();
        if (a >= 0 && b >= 0 && a < s.G && b < s.G) s.bad2[a * s.G + b] = 1;
      }
    } else if (tok == "bad3") {
      const int m = (int)in.num();
      s.bad3.assign(((size_t)s.G * s.G * s.G + 31) / 32, 0);
      for (int i = 0; i < m && !in.fail; i++) {
        const int a = (int)in.num(), b = (int)in.num(), c = (int)in.num();
        if (a < 0 || b < 0 || c < 0 || a >= s.G || b >= s.G || c >= s.G) continue;
        const uint32_t t = (uint32_t)((a * s.G + b) * s.G + c);
        s.bad3[t >> 5] |= 1u << (t & 31);
      }
    } else if (tok == "target") {
      const int k = (int)in.num();
      if (s.n < 1 || s.n > NQMAX) { err = "n = " + std::to_string(s.n) + " not built"; return RC_USAGE; }
      const int N = 1 << s.n;
      std::vector<Zw> M(N * N);
      for (auto &x : M) x = in.zw();
      if (!s.states) { s.target = M; s.tk = k; s.gk = 0; }
      else { s.goal = M; s.gk = k; have_goal_rows = true; }
    } else if (tok == "cuts") {
      const int m = (int)in.num();
      for (int i = 0; i < m && !in.fail; i++) {
        const int sz = (int)in.num();
        if (sz < 1 || sz > 30) { err = "bad cut"; return RC_SPEC; }
        int mask = 0;
        for (int j = 0; j < sz; j++) {
          const int q = (int)in.num();
          if (q < 0 || q > 30 || (mask >> q & 1)) { err = "bad cut"; return RC_SPEC; }
          mask |= 1 << q;
        }
        if ((int)s.cutmask.size() < CUTMAX) { s.cutmask.push_back(mask); s.cutsize.push_back(sz); s.rad.push_back(2 * sz + 1); }
      }
    } else if (tok == "cxtable") {
      const int m = (int)in.num();
      if (m < 0 || m > (1 << 22)) { err = "cxtable too large"; return RC_SPEC; }
      s.cxtable.resize(m);
      for (auto &v : s.cxtable) v = (int)in.num();
    } else if (tok == "end") break;
    else { err = "unknown spec field " + tok; return RC_SPEC; }
  }
  if (s.states) {                              // the reference's reader: every part of a state spec present
    if (!have_start || !have_goal_rows || !have_ginfo || s.m < 1 || s.m > (1 << std::max(0, std::min(s.n, 6))) ||
        s.ginfo.size() != (size_t)s.m * (2 + s.cutmask.size())) {
      err = "states spec incomplete";
      return RC_SPEC;
    }
  }
  if (s.n < 1 || s.n > NQMAX) { err = "n = " + std::to_string(s.n) + " not built"; return RC_USAGE; }
  const int N = 1 << s.n;
  if ((int)s.target.size() != N * N) { s.target.assign(N * N, Zw{0, 0, 0, 0}); }
  if (s.bad2.empty()) s.bad2.assign((size_t)s.G * s.G, 0);
  if (s.bad3.empty()) s.bad3.assign(((size_t)s.G * s.G * s.G + 31) / 32, 0);
  // the window tables are indexed by candidate on the device: their sizes must be those of the final gate list
  if ((int)s.names.size() != s.G || s.bad2.size() != (size_t)s.G * s.G ||
      s.bad3.size() != ((size_t)s.G * s.G * s.G + 31) / 32) {
    err = "window rules do not match the gate list";
    return RC_SPEC;
  }
  if (s.tdiv < 1) s.tdiv = 1;
  for (int g = 0; g < s.G; g++) {
    for (int j = 0; j < s.gnq[g]; j++)
      if (s.gq[g][j] < 0 || s.gq[g][j] >= s.n) { err = "gate " + s.names[g] + " acts outside the register"; return RC_SPEC; }
    uint8_t f = 0;
    if (is_clifford(s.ginv[g], s.gnq[g])) f |= GF_CLIFFORD;
    if (s.gnq[g] == 1) f |= GF_ONEQ;
    if (is_monomial_affine(s.ginv[g], s.gnq[g])) f |= GF_MONAFF;
    if (s.gnq[g] == 1 && zzero(s.ginv[g][1]) && zzero(s.ginv[g][2])) {
      const int p0 = unit_power(s.ginv[g][0]), p1 = unit_power(s.ginv[g][3]);
      if (p0 >= 0 && p1 >= 0 && ((p1 - p0) & 1)) f |= GF_TDIAG;
    }
    if (s.gnq[g] == 2 && schmidt_rank_p(s.ginv[g]) <= 2) f |= GF_RANK2;
    s.gflags.push_back(f);
  }
  for (size_t i = 0; i < s.cutmask.size(); i++) {
    if (s.cutsize[i] > s.n / 2 || s.cutsize[i] < 1) { err = "cut larger than half the register"; return RC_SPEC; }
    if (s.cutmask[i] >> s.n) { err = "cut acts outside the register"; return RC_SPEC; }
  }
  return 0;
}

namespace {
// A candidate name "L_<gate>_<q>[_<q>...]" read once: its gate word and its qubits (std::atoi of each field, as the
// reference's reader takes them). well = the name has a gate field and every qubit lies in the register.
struct CandName {
  std::string word;
  std::vector<int> qs;
  bool well = false;
};
CandName read_cand(const std::string &nm, int n) {
  CandName c;
  std::vector<std::string> f(1);
  for (char ch : nm) {
    if (ch == '_') f.emplace_back();
    else f.back() += ch;
  }
  if (f.size() < 2) return c;
  c.word = f[1];
  c.well = true;
  for (size_t i = 2; i < f.size(); i++) {
    c.qs.push_back(std::atoi(f[i].c_str()));
    if (c.qs.back() < 0 || c.qs.back() >= n) c.well = false;
  }
  return c;
}
// The gate word of a gate's complex conjugate: the phase gates swap with their inverses, the real gates map to
// themselves; "" for any other word (y, whose conjugate is -y, and unknown gates): no conjugating symmetry then.
std::string conjugate_word(const std::string &w) {
  static const std::map<std::string, std::string> table = {
      {"t", "tdg"}, {"tdg", "t"}, {"s", "sdg"}, {"sdg", "s"},
      {"x", "x"}, {"z", "z"}, {"h", "h"}, {"cx", "cx"}, {"cz", "cz"}, {"ccx", "ccx"}};
  const auto it = table.find(w);
  return it == table.end() ? std::string() : it->second;
}
// The qubit relabellings of n qubits (perm[i] = image of qubit i) in lexicographic order, read off an n-digit
// base-n counter (only the bijective digit strings are kept).
std::vector<std::vector<int>> relabellings(int n) {
  std::vector<std::vector<int>> out;
  std::vector<int> d(n, 0);
  for (;;) {
    int seen = 0;
    for (int v : d) seen |= 1 << v;
    if (seen == (1 << n) - 1) out.push_back(d);
    int i = n - 1;
    while (i >= 0 && d[i] == n - 1) d[i--] = 0;
    if (i < 0) break;
    d[i]++;
  }
  return out;
}
}  // namespace

// Elements are ordered conjugation-free first, each half by relabelling in lexicographic order (the element order
// decides which symmetry the class comparisons try first). A relabelling x conjugation is kept when the image of
// every candidate name (gate word conjugated, qubits relabelled, the two ccx controls written in ascending order)
// names a candidate; the image is the first candidate of that name.
SymGroup sym_group(const HostSpec &hs, bool on) {
  const int n = hs.n, N = 1 << n;
  std::vector<CandName> cand;
  std::unordered_map<std::string, int> by_name;
  for (int g = 0; g < hs.G; g++) {
    cand.push_back(read_cand(hs.names[g], n));
    by_name.emplace(hs.names[g], g);          // keeps the first index of a repeated name
  }
  auto image = [&](const CandName &c, const std::vector<int> &perm, bool conj) {
    if (!c.well) return -1;
    const std::string w = conj ? conjugate_word(c.word) : c.word;
    if (w.empty()) return -1;
    std::vector<int> q(c.qs.size());
    for (size_t i = 0; i < q.size(); i++) q[i] = perm[c.qs[i]];
    if (w == "ccx" && q.size() == 3 && q[0] > q[1]) std::swap(q[0], q[1]);
    std::string nm = "L_" + w;
    for (int x : q) nm += "_" + std::to_string(x);
    const auto it = by_name.find(nm);
    return it == by_name.end() ? -1 : it->second;
  };
  std::vector<std::vector<int>> perms = relabellings(n);
  if (!on) perms.resize(1);                     // the identity comes first
  SymGroup g;
  for (int conj = 0; conj <= (on ? 1 : 0); conj++)
    for (const auto &perm : perms) {
      std::vector<int> gm(hs.G);
      int c = 0;
      while (c < hs.G && (gm[c] = image(cand[c], perm, conj != 0)) >= 0) c++;
      if (c < hs.G) continue;
      g.perm.push_back(perm);
      g.conj.push_back((uint8_t)conj);
      g.gmap.push_back(std::move(gm));
      for (int x = 0; x < N; x++) {
        int y = 0;
        for (int b = x; b; b &= b - 1) y |= 1 << perm[__builtin_ctz(b)];
        g.bperm.push_back((uint8_t)y);
      }
    }
  g.nsym = (int)g.conj.size();
  return g;
}

std::vector<int> inverse_gates(const HostSpec &hs) {
  std::vector<int> inv(hs.G, -1);
  for (int g = 0; g < hs.G; g++) {
    const std::string &nm = hs.names[g];
    const size_t a = nm.find('_');
    if (a == std::string::npos) continue;
    const size_t b = nm.find('_', a + 1);
    std::string gate = nm.substr(a + 1, b == std::string::npos ? std::string::npos : b - a - 1);
    if (gate == "t") gate = "tdg"; else if (gate == "tdg") gate = "t";
    else if (gate == "s") gate = "sdg"; else if (gate == "sdg") gate = "s";
    const std::string want = nm.substr(0, a + 1) + gate + (b == std::string::npos ? "" : nm.substr(b));
    for (int h = 0; h < hs.G; h++) if (hs.names[h] == want) inv[g] = h;
  }
  return inv;
}

}  // namespace cz
