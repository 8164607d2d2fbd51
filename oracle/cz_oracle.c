/* cz_oracle.c: CPU restatement of the reference's gate-count search (src/cheese.cu). TEST INFRASTRUCTURE ONLY:
 * the checker for the CUDA product path, never linked into it. See cz_oracle.h for what pins it. */
#include "cz_oracle.h"

#include <ctype.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PRIME 998244353ULL /* cheese.cu:57 */

/* ---------------- Z[w]: (a + b w + c w^2 + d w^3), w = e^{i pi/4} (cheese.cu:60-82) ---------------- */
static inline czo_zw zadd(czo_zw x, czo_zw y) { czo_zw r = {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; return r; }
static inline czo_zw zmul(czo_zw x, czo_zw y) {   /* w^4 = -1 */
  czo_zw r = {x.a * y.a - x.b * y.d - x.c * y.c - x.d * y.b, x.a * y.b + x.b * y.a - x.c * y.d - x.d * y.c,
              x.a * y.c + x.b * y.b + x.c * y.a - x.d * y.d, x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a};
  return r;
}
static inline czo_zw zconj(czo_zw x) { czo_zw r = {x.a, -x.d, -x.c, -x.b}; return r; }
static inline int zzero(czo_zw x) { return !(x.a | x.b | x.c | x.d); }
static inline int zeq(czo_zw x, czo_zw y) { return x.a == y.a && x.b == y.b && x.c == y.c && x.d == y.d; }
/* x / sqrt2 stays in Z[w] iff a = c and b = d mod 2 (sqrt2 = w - w^3) */
static inline int zdiv2ok(czo_zw x) { return !((x.a - x.c) & 1) && !((x.b - x.d) & 1); }
static inline czo_zw zdown(czo_zw x) {
  czo_zw r = {(x.b - x.d) / 2, (x.a + x.c) / 2, (x.b + x.d) / 2, (x.c - x.a) / 2};
  return r;
}
static inline czo_zw zwpow(int p) {
  czo_zw r = {0, 0, 0, 0};
  p &= 7;
  const int64_t s = p < 4 ? 1 : -1;
  switch (p & 3) { case 0: r.a = s; break; case 1: r.b = s; break; case 2: r.c = s; break; default: r.d = s; }
  return r;
}
static int zval(czo_zw x) { int v = 0; while (zdiv2ok(x)) { x = zdown(x); if (++v > 200) break; } return v; }
static inline int fits32(int64_t v) { return v >= INT32_MIN && v <= INT32_MAX; }
static inline int zfits32(czo_zw x) { return fits32(x.a) && fits32(x.b) && fits32(x.c) && fits32(x.d); }

/* ---------------- spec reader: the grammar of read_spec (cheese.cu:1149-1226) ---------------- */
typedef struct { const char *p, *end; int fail; } rd;
static int rd_tok(rd *r, char *buf, size_t cap) {
  while (r->p < r->end && isspace((unsigned char)*r->p)) r->p++;
  if (r->p >= r->end) return 0;
  size_t n = 0;
  while (r->p < r->end && !isspace((unsigned char)*r->p)) { if (n + 1 < cap) buf[n++] = *r->p; r->p++; }
  buf[n] = 0;
  return 1;
}
static int64_t rd_int(rd *r) {   /* a failed read poisons the stream, as std::istream does */
  char buf[64];
  if (r->fail || !rd_tok(r, buf, sizeof buf)) { r->fail = 1; return 0; }
  char *e;
  const long long v = strtoll(buf, &e, 10);
  if (e == buf) { r->fail = 1; return 0; }
  return v;
}
static void rd_zw(rd *r, czo_zw *z) { z->a = rd_int(r); z->b = rd_int(r); z->c = rd_int(r); z->d = rd_int(r); }

int czo_spec_parse(const char *text, size_t len, czo_spec *s, char *err, size_t errlen) {
  memset(s, 0, sizeof *s);
  s->tdiv = 1;
  rd r = {text, text + len, 0};
  char tok[128];
  if (!rd_tok(&r, tok, sizeof tok) || strcmp(tok, "cheese-spec")) { snprintf(err, errlen, "not a spec"); return 2; }
  (void)rd_int(&r);
  int have_bad2 = 0, have_bad3 = 0, have_target = 0;
  while (!r.fail && rd_tok(&r, tok, sizeof tok)) {
    if (!strcmp(tok, "n")) s->n = (int)rd_int(&r);
    else if (!strcmp(tok, "mode") || !strcmp(tok, "phase")) {
      char v[64];
      if (!rd_tok(&r, v, sizeof v)) break;
      if (!strcmp(v, "states")) s->states = 1;
      else if (strcmp(v, "unitary") && strcmp(v, "exact")) { snprintf(err, errlen, "unsupported %s %s", tok, v); return 2; }
    } else if (!strcmp(tok, "pairs")) (void)rd_int(&r);
    else if (!strcmp(tok, "start")) { snprintf(err, errlen, "state targets are not part of this build"); return 3; }
    else if (!strcmp(tok, "goal")) { snprintf(err, errlen, "state targets are not part of this build"); return 3; }
    else if (!strcmp(tok, "depth")) s->depth = (int)rd_int(&r);
    else if (!strcmp(tok, "standard")) s->standard = (int)rd_int(&r);
    else if (!strcmp(tok, "lite")) s->lite = (int)rd_int(&r);
    else if (!strcmp(tok, "tdiv")) s->tdiv = (int)rd_int(&r);
    else if (!strcmp(tok, "gates")) {
      s->G = (int)rd_int(&r);
      if (s->G > CZO_GMAX) { snprintf(err, errlen, "too many gates"); return 2; }
      for (int g = 0; g < s->G && !r.fail; g++) {
        if (!rd_tok(&r, s->names[g], sizeof s->names[g])) { r.fail = 1; break; }
        s->gnq[g] = (int)rd_int(&r);
        if (s->gnq[g] < 1 || s->gnq[g] > 3) { r.fail = 1; break; }
        for (int j = 0; j < s->gnq[g]; j++) s->gq[g][j] = (int)rd_int(&r);
        const int L = 1 << s->gnq[g];
        (void)rd_int(&r);                                    /* forward gate exponent */
        czo_zw fwd;
        for (int i = 0; i < L * L; i++) rd_zw(&r, &fwd);     /* forward matrix: unused for unitary targets */
        s->gik[g] = (int)rd_int(&r);
        for (int i = 0; i < L * L; i++) rd_zw(&r, &s->ginv[g][i]);
      }
    } else if (!strcmp(tok, "bad2")) {
      const int m = (int)rd_int(&r);
      memset(s->bad2, 0, sizeof s->bad2);
      have_bad2 = 1;
      for (int i = 0; i < m && !r.fail; i++) {
        const int a = (int)rd_int(&r), b = (int)rd_int(&r);
        if (a >= 0 && b >= 0 && a < s->G && b < s->G) s->bad2[a * s->G + b] = 1;
      }
    } else if (!strcmp(tok, "bad3")) {
      const int m = (int)rd_int(&r);
      memset(s->bad3, 0, sizeof s->bad3);
      have_bad3 = 1;
      for (int i = 0; i < m && !r.fail; i++) {
        const int a = (int)rd_int(&r), b = (int)rd_int(&r), c = (int)rd_int(&r);
        if (a < 0 || b < 0 || c < 0 || a >= s->G || b >= s->G || c >= s->G) continue;
        const uint32_t t = (uint32_t)((a * s->G + b) * s->G + c);
        s->bad3[t >> 5] |= 1u << (t & 31);
      }
    } else if (!strcmp(tok, "target")) {
      s->tk = (int)rd_int(&r);
      if (s->n < 1 || s->n > 3) { snprintf(err, errlen, "n = %d not built", s->n); return 3; }
      const int N = 1 << s->n;
      for (int i = 0; i < N * N; i++) rd_zw(&r, &s->target[i]);
      have_target = 1;
    } else if (!strcmp(tok, "cuts")) {
      const int m = (int)rd_int(&r);
      for (int i = 0; i < m && !r.fail && s->ncuts < CZO_CUTMAX; i++) {
        const int sz = (int)rd_int(&r);
        int mask = 0;
        for (int j = 0; j < sz; j++) mask |= 1 << (int)rd_int(&r);
        s->cutmask[s->ncuts] = mask; s->cutsize[s->ncuts] = sz; s->rad[s->ncuts] = 2 * sz + 1; s->ncuts++;
      }
    } else if (!strcmp(tok, "cxtable")) {
      const int m = (int)rd_int(&r);
      if (m < 0 || m > 4096) { snprintf(err, errlen, "cxtable too large"); return 2; }
      s->ncx = m;
      for (int i = 0; i < m; i++) s->cxtable[i] = (int)rd_int(&r);
    } else if (!strcmp(tok, "end")) break;
    else { snprintf(err, errlen, "unknown spec field %s", tok); return 2; }
  }
  (void)have_bad2; (void)have_bad3;
  if (s->states) { snprintf(err, errlen, "state targets are not part of this build"); return 3; }
  if (!have_target || s->n < 1 || s->n > 3) { snprintf(err, errlen, "n = %d not built", s->n); return 3; }
  s->N = 1 << s->n;
  if (s->tdiv < 1) s->tdiv = 1;
  return 0;
}

/* ---------------- residual update: apply_inv + normalise (cheese.cu:134-174) ---------------- */
static void normalise(int N, czo_zw *S, int *k) {
  while (*k > 0) {
    for (int i = 0; i < N * N; i++) if (!zdiv2ok(S[i])) return;
    for (int i = 0; i < N * N; i++) S[i] = zdown(S[i]);
    (*k)--;
  }
}

int czo_apply_inv(const czo_spec *sp, int g, czo_zw *S, int *k) {
  const int N = sp->N, nq = sp->gnq[g], L = 1 << nq;
  int mask = 0, ovf = 0;
  for (int j = 0; j < nq; j++) mask |= 1 << sp->gq[g][j];
  for (int base = 0; base < N; base++) {
    if (base & mask) continue;
    int idx[CZO_LMAX];
    for (int l = 0; l < L; l++) {
      int x = base;
      for (int j = 0; j < nq; j++) if ((l >> j) & 1) x |= 1 << sp->gq[g][j];
      idx[l] = x;
    }
    for (int r = 0; r < N; r++) {
      czo_zw col[CZO_LMAX];
      for (int lc = 0; lc < L; lc++) {             /* (S g^-1)[r][idx lc] = sum_m S[r][idx m] ginv[m][lc] */
        czo_zw acc = {0, 0, 0, 0};
        for (int m = 0; m < L; m++) {
          const czo_zw gm = sp->ginv[g][m * L + lc];
          if (!zzero(gm)) acc = zadd(acc, zmul(S[r * N + idx[m]], gm));
        }
        col[lc] = acc;
      }
      for (int lc = 0; lc < L; lc++) { S[r * N + idx[lc]] = col[lc]; if (!zfits32(col[lc])) ovf = 1; }
    }
  }
  *k += sp->gik[g];
  normalise(N, S, k);
  return ovf;
}

/* ---------------- cheap bounds (cheese.cu:305-338) ---------------- */
int czo_support(int n, const czo_zw *S) {
  const int N = 1 << n;
  int cnt = 0;
  for (int q = 0; q < n; q++) {
    const int bit = 1 << q;
    int trivial = 1;
    for (int r = 0; r < N && trivial; r++)
      for (int c = 0; c < N && trivial; c++) {
        if ((r ^ c) & bit) { if (!zzero(S[r * N + c])) trivial = 0; }
        else if (!((r | c) & bit) && !zeq(S[r * N + c], S[(r | bit) * N + (c | bit)])) trivial = 0;
      }
    cnt += !trivial;
  }
  return cnt;
}

int czo_h_struct(int n, const czo_zw *S) {   /* 2: monomial with a non-affine permutation */
  const int N = 1 << n;
  int pi[CZO_NMAX];
  for (int c = 0; c < N; c++) {
    int nz = 0, row = 0;
    for (int r = 0; r < N; r++) if (!zzero(S[r * N + c])) { nz++; row = r; }
    if (nz != 1) return 0;
    pi[c] = row;
  }
  for (int j = 0; j < N; j++) {
    int x = pi[0];
    for (int i = 0; i < n; i++) if ((j >> i) & 1) x ^= pi[1 << i] ^ pi[0];
    if (pi[j] != x) return 2;
  }
  return 0;
}

/* ---------------- CX bound: operator-Schmidt rank over F_p (cheese.cu:257-303, 585-597) ---------------- */
static inline uint64_t mulmod(uint64_t a, uint64_t b) { return (a * b) % PRIME; }
static uint64_t powmod(uint64_t a, uint64_t e) { uint64_t r = 1; while (e) { if (e & 1) r = mulmod(r, a); a = mulmod(a, a); e >>= 1; } return r; }
static inline uint64_t tomod(int64_t v) { int64_t m = v % (int64_t)PRIME; return (uint64_t)(m < 0 ? m + (int64_t)PRIME : m); }
static uint64_t g_w8, g_w82, g_w83;
static void init_w8(void) {   /* w -> 3^((p-1)/8), a primitive 8th root of unity mod p (cheese.cu:1775) */
  if (g_w8) return;
  g_w8 = powmod(3, (PRIME - 1) / 8); g_w82 = mulmod(g_w8, g_w8); g_w83 = mulmod(g_w82, g_w8);
}
static inline uint64_t zmod(czo_zw x) {
  return (tomod(x.a) + mulmod(tomod(x.b), g_w8) + mulmod(tomod(x.c), g_w82) + mulmod(tomod(x.d), g_w83)) % PRIME;
}

int czo_cut_rank(int n, const czo_zw *S, int A, int sa) {
  init_w8();
  const int N = 1 << n, R = 1 << (2 * sa), C = (N * N) / R;
  uint64_t M[16][64];
  for (int o = 0; o < N; o++)
    for (int i = 0; i < N; i++) {
      int oa = 0, ob = 0, ia = 0, ib = 0, na = 0, nb = 0;
      for (int q = 0; q < n; q++) {
        if ((A >> q) & 1) { oa |= ((o >> q) & 1) << na; ia |= ((i >> q) & 1) << na; na++; }
        else { ob |= ((o >> q) & 1) << nb; ib |= ((i >> q) & 1) << nb; nb++; }
      }
      M[(oa << na) | ia][(ob << nb) | ib] = zmod(S[o * N + i]);
    }
  int rank = 0;
  for (int c = 0; c < C && rank < R; c++) {   /* row echelon form: the rank does not depend on the pivot order */
    int piv = -1;
    for (int r = rank; r < R; r++) if (M[r][c]) { piv = r; break; }
    if (piv < 0) continue;
    if (piv != rank) for (int j = 0; j < C; j++) { const uint64_t t = M[piv][j]; M[piv][j] = M[rank][j]; M[rank][j] = t; }
    const uint64_t inv = powmod(M[rank][c], PRIME - 2);
    for (int r = rank + 1; r < R; r++) {
      if (!M[r][c]) continue;
      const uint64_t f = mulmod(M[r][c], inv);
      for (int j = c; j < C; j++) M[r][j] = (M[r][j] + PRIME - mulmod(f, M[rank][j])) % PRIME;
    }
    rank++;
  }
  return rank;
}

static int cx_bound(const czo_spec *sp, const czo_zw *S) {
  int idx = 0, mult = 1, mx = 0;
  for (int i = 0; i < sp->ncuts; i++) {
    const int rk = czo_cut_rank(sp->n, S, sp->cutmask[i], sp->cutsize[i]);
    int need = 0;
    while ((1 << need) < rk) need++;
    if (need > sp->rad[i] - 1) need = sp->rad[i] - 1;
    idx += need * mult;
    mult *= sp->rad[i];
    if (need > mx) mx = need;
  }
  return sp->ncx ? sp->cxtable[idx] : mx;
}

/* ---------------- T bound (cheese.cu:340-449) ---------------- */
static void pauli(int b, int nq, int *flip, int *ymask, int *zmask) {
  *flip = *ymask = *zmask = 0;
  for (int q = 0; q < nq; q++) {
    const int d = (b >> (2 * q)) & 3;
    if (d == 1 || d == 2) *flip |= 1 << q;
    if (d == 2) *ymask |= 1 << q;
    if (d == 3) *zmask |= 1 << q;
  }
}
static int pphase(int x, int ymask, int zmask) {
  return (2 * __builtin_popcount(ymask) + 4 * __builtin_popcount(x & (ymask | zmask))) & 7;
}

int czo_ptm_sde(int n, const czo_zw *S, int k) {   /* the direct definition: max over PTM entries of their sde */
  const int N = 1 << n, P = 1 << (2 * n);
  if (k + 2 * n + 6 > 62) return 0;
  int best = 0;
  czo_zw SP[64], M[64];
  for (int b = 0; b < P; b++) {
    int fb, yb, zb;
    pauli(b, n, &fb, &yb, &zb);
    for (int r = 0; r < N; r++)
      for (int c = 0; c < N; c++) {
        const czo_zw x = S[r * N + (c ^ fb)];
        SP[r * N + c] = zzero(x) ? x : zmul(x, zwpow(pphase(c, yb, zb)));
      }
    for (int r = 0; r < N; r++)
      for (int s = 0; s < N; s++) {
        czo_zw acc = {0, 0, 0, 0};
        for (int c = 0; c < N; c++) acc = zadd(acc, zmul(SP[r * N + c], zconj(S[s * N + c])));
        M[r * N + s] = acc;
      }
    for (int a = 0; a < P; a++) {
      int fa, ya, za;
      pauli(a, n, &fa, &ya, &za);
      czo_zw acc = {0, 0, 0, 0};
      for (int x = 0; x < N; x++) acc = zadd(acc, zmul(M[(x ^ fa) * N + x], zwpow(pphase(x ^ fa, ya, za))));
      if (!zzero(acc)) { const int need = 2 * (n + k) - zval(acc); if (need > best) best = need; }
    }
  }
  return best;
}

/* Walsh-Hadamard form over Z[w] mod 2^32 (or 2^64 when 2(n + k) > 64), valuations from the low bits */
#define DEF_PTM(NAME, U)                                                                                      \
  static int NAME(int n, const czo_zw *S, int k) {                                                            \
    const int N = 1 << n, E = N * N, top = 2 * (n + k);                                                       \
    int best = 0;                                                                                             \
    U qa[64], qb[64], qc[64], qd[64];                                                                         \
    for (int fa = 0; fa < N; fa++)                                                                            \
      for (int fb = 0; fb < N; fb++) {                                                                        \
        for (int e = 0; e < E; e++) {                                                                         \
          const int x = e >> n, c = e & (N - 1);                                                              \
          const czo_zw X = S[(x ^ fa) * N + (c ^ fb)], Y = zconj(S[e]);                                      \
          const U xa = (U)X.a, xb = (U)X.b, xc = (U)X.c, xd = (U)X.d;                                        \
          const U ya = (U)Y.a, yb = (U)Y.b, yc = (U)Y.c, yd = (U)Y.d;                                        \
          qa[e] = (U)(xa * ya - xb * yd - xc * yc - xd * yb);                                                 \
          qb[e] = (U)(xa * yb + xb * ya - xc * yd - xd * yc);                                                 \
          qc[e] = (U)(xa * yc + xb * yb + xc * ya - xd * yd);                                                 \
          qd[e] = (U)(xa * yd + xb * yc + xc * yb + xd * ya);                                                 \
        }                                                                                                     \
        for (int h = 1; h < E; h <<= 1)                                                                       \
          for (int e = 0; e < E; e++)                                                                         \
            if (!(e & h)) {                                                                                   \
              U u, v;                                                                                         \
              u = qa[e]; v = qa[e | h]; qa[e] = (U)(u + v); qa[e | h] = (U)(u - v);                           \
              u = qb[e]; v = qb[e | h]; qb[e] = (U)(u + v); qb[e | h] = (U)(u - v);                           \
              u = qc[e]; v = qc[e | h]; qc[e] = (U)(u + v); qc[e | h] = (U)(u - v);                           \
              u = qd[e]; v = qd[e | h]; qd[e] = (U)(u + v); qd[e | h] = (U)(u - v);                           \
            }                                                                                                 \
        for (int e = 0; e < E; e++) {                                                                         \
          const U o = qa[e] | qb[e] | qc[e] | qd[e];                                                          \
          if (!o) continue;                                                                                   \
          const int m = __builtin_ctzll((unsigned long long)o);                                               \
          const int dv = !(((qa[e] >> m) ^ (qc[e] >> m)) & 1) && !(((qb[e] >> m) ^ (qd[e] >> m)) & 1);        \
          const int v = 2 * m + dv;                                                                           \
          if (top - v > best) best = top - v;                                                                 \
        }                                                                                                     \
      }                                                                                                       \
    return best;                                                                                              \
  }
DEF_PTM(ptm32, uint32_t)
DEF_PTM(ptm64, uint64_t)
int czo_ptm_t(int n, const czo_zw *S, int k) { return 2 * (n + k) <= 64 ? ptm32(n, S, k) : ptm64(n, S, k); }

int czo_combine(int h, int t, int c2, int supp) {
  int best = 1 << 30;
  const int hi = c2 > supp ? c2 : supp;
  for (int c = c2; c <= hi; c++) {
    const int one = (h + t > supp - 2 * c) ? h + t : supp - 2 * c;
    if (c + one < best) best = c + one;
  }
  return best;
}

/* ---------------- symmetry group from candidate names (cheese.cu:1379-1429) ---------------- */
typedef struct { int nsym; uint8_t perm[12][CZO_NMAX]; uint8_t conj[12]; } symgrp;

static int sym_gate(const czo_spec *sp, const int *perm, int conj, int g) {
  char buf[40], gate[16], want[40];
  snprintf(buf, sizeof buf, "%s", sp->names[g]);
  char *parts[8];
  int np = 0;
  for (char *p = strtok(buf, "_"); p && np < 8; p = strtok(NULL, "_")) parts[np++] = p;
  if (np < 2) return -1;
  snprintf(gate, sizeof gate, "%s", parts[1]);
  if (conj) {
    if (!strcmp(gate, "t")) strcpy(gate, "tdg"); else if (!strcmp(gate, "tdg")) strcpy(gate, "t");
    else if (!strcmp(gate, "s")) strcpy(gate, "sdg"); else if (!strcmp(gate, "sdg")) strcpy(gate, "s");
    else if (strcmp(gate, "x") && strcmp(gate, "z") && strcmp(gate, "h") && strcmp(gate, "cx") && strcmp(gate, "cz") &&
             strcmp(gate, "ccx")) return -1;
  }
  int qs[6], nq = 0;
  for (int i = 2; i < np; i++) qs[nq++] = perm[atoi(parts[i])];
  if (!strcmp(gate, "ccx") && nq == 3 && qs[0] > qs[1]) { const int t = qs[0]; qs[0] = qs[1]; qs[1] = t; }
  int off = snprintf(want, sizeof want, "L_%s", gate);
  for (int i = 0; i < nq; i++) off += snprintf(want + off, sizeof want - off, "_%d", qs[i]);
  for (int h = 0; h < sp->G; h++) if (!strcmp(sp->names[h], want)) return h;
  return -1;
}

static int next_perm(int *p, int n) {
  int i = n - 2;
  while (i >= 0 && p[i] >= p[i + 1]) i--;
  if (i < 0) return 0;
  int j = n - 1;
  while (p[j] <= p[i]) j--;
  int t = p[i]; p[i] = p[j]; p[j] = t;
  for (int a = i + 1, b = n - 1; a < b; a++, b--) { t = p[a]; p[a] = p[b]; p[b] = t; }
  return 1;
}

static void sym_group(const czo_spec *sp, int on, symgrp *g) {
  const int n = sp->n, N = sp->N;
  int perms[6][3], np = 0, p[3] = {0, 1, 2};
  do { for (int i = 0; i < n; i++) perms[np][i] = p[i]; np++; } while (on && next_perm(p, n));
  g->nsym = 0;
  for (int cj = 0; cj < (on ? 2 : 1); cj++)
    for (int pi = 0; pi < np; pi++) {
      int ok = 1;
      for (int c = 0; c < sp->G && ok; c++) ok = sym_gate(sp, perms[pi], cj, c) >= 0;
      if (!ok) continue;
      for (int x = 0; x < N; x++) {
        int y = 0;
        for (int i = 0; i < n; i++) if ((x >> i) & 1) y |= 1 << perms[pi][i];
        g->perm[g->nsym][x] = (uint8_t)y;
      }
      g->conj[g->nsym] = (uint8_t)cj;
      g->nsym++;
    }
}

/* class key: the smallest 128-bit hash over the orbit (cheese.cu:224-241); the hash function is this oracle's own */
static inline uint64_t smix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static void class_key(const czo_spec *sp, const symgrp *g, const czo_zw *S, int k, uint64_t *h1, uint64_t *h2) {
  const int N = sp->N, n = sp->n;
  *h1 = *h2 = ~0ULL;
  for (int s = 0; s < g->nsym; s++) {
    uint64_t a = 0, b = 0;
    for (int e = 0; e < N * N; e++) {
      const czo_zw v = g->conj[s] ? zconj(S[e]) : S[e];
      const int pos = g->perm[s][e >> n] * N + g->perm[s][e & (N - 1)];
      const uint64_t x = smix(smix(smix(smix((uint64_t)pos * 0x10001ULL + (uint64_t)v.a) + (uint64_t)v.b) + (uint64_t)v.c) + (uint64_t)v.d);
      a += x;
      b += smix(x ^ 0x5bd1e9955bd1e995ULL);
    }
    const uint64_t x1 = smix(a + (uint64_t)k), x2 = smix(b ^ ((uint64_t)k << 32));
    if (x1 < *h1 || (x1 == *h1 && x2 < *h2)) { *h1 = x1; *h2 = x2; }
  }
}
static int same_class(const czo_spec *sp, const symgrp *g, const czo_zw *A, int ka, const czo_zw *B, int kb) {
  const int N = sp->N, n = sp->n;
  if (ka != kb) return 0;
  for (int s = 0; s < g->nsym; s++) {
    int eq = 1;
    for (int e = 0; eq && e < N * N; e++) {
      const czo_zw v = g->conj[s] ? zconj(A[e]) : A[e];
      eq = zeq(v, B[g->perm[s][e >> n] * N + g->perm[s][e & (N - 1)]]);
    }
    if (eq) return 1;
  }
  return 0;
}

/* ---------------- the level loop (cheese.cu:1249-1377) ---------------- */
enum { DEAD = 0, ALIVE = 1, FOUND = 2, W2CUT = 3, W3CUT = 4, OVF = 6 };   /* status codes, cheese.cu:647 */

typedef struct {
  const czo_spec *sp;
  const symgrp *grp;
  int t, depth, store64;
  long m;
  const czo_zw *R;        /* m parent residuals */
  const int *Rk;
  const int16_t *g1, *g2; /* parents' last two gates (-1: none) */
} lvl_in;

static int is_goal(const czo_spec *sp, const czo_zw *S, int k) {   /* unitary target: the residual reaches I, k 0 */
  if (k != 0) return 0;
  for (int r = 0; r < sp->N; r++)
    for (int c = 0; c < sp->N; c++) {
      const czo_zw x = S[r * sp->N + c];
      if (r == c ? !(x.a == 1 && !x.b && !x.c && !x.d) : !zzero(x)) return 0;
    }
  return 1;
}

/* one child: the status of cheese.cu's Cheap + Full passes (649-720); key when ALIVE */
static int child_status(const lvl_in *L, long i, int g, uint64_t *h1, uint64_t *h2) {
  const czo_spec *sp = L->sp;
  const int G = sp->G, g1 = L->g1[i], g2 = L->g2[i];
  if (g1 >= 0 && sp->bad2[g1 * G + g]) return W2CUT;
  if (g2 >= 0) {
    const uint32_t tri = ((uint32_t)g2 * G + (uint32_t)g1) * G + (uint32_t)g;
    if ((sp->bad3[tri >> 5] >> (tri & 31)) & 1) return W3CUT;
  }
  const int N = sp->N;
  czo_zw C[64];
  memcpy(C, L->R + i * N * N, sizeof(czo_zw) * N * N);
  int k = L->Rk[i];
  const int ovf = czo_apply_inv(sp, g, C, &k);
  if (ovf && !L->store64) return OVF;
  if (is_goal(sp, C, k)) return FOUND;
  const int rem = L->depth - L->t;
  if (sp->standard || sp->lite) {
    int h, supp = 0, c2 = 0;
    if (sp->lite) h = k;
    else {
      const int hs = czo_h_struct(sp->n, C);
      h = k > hs ? k : hs;
      supp = czo_support(sp->n, C);
      c2 = cx_bound(sp, C);
    }
    if (czo_combine(h, 0, c2, supp) > rem) return DEAD;
    const int T = (czo_ptm_t(sp->n, C, k) + sp->tdiv - 1) / sp->tdiv;
    if (czo_combine(h, T, c2, supp) > rem) return DEAD;
  }
  class_key(sp, L->grp, C, k, h1, h2);
  return ALIVE;
}

typedef struct { uint64_t h1, h2; long idx; } ckey;
static int ckey_cmp(const void *x, const void *y) {
  const ckey *a = x, *b = y;
  if (a->h1 != b->h1) return a->h1 < b->h1 ? -1 : 1;
  if (a->h2 != b->h2) return a->h2 < b->h2 ? -1 : 1;
  return a->idx < b->idx ? -1 : a->idx > b->idx;
}
static int long_cmp(const void *x, const void *y) { const long a = *(const long *)x, b = *(const long *)y; return a < b ? -1 : a > b; }

int czo_search(const czo_spec *sp, int depth, int dedupe, int sym, int store64, int threads, czo_result *res) {
  memset(res, 0, sizeof *res);
  if (threads > 0) omp_set_num_threads(threads);
  const int N = sp->N, E = N * N, G = sp->G;
  symgrp grp;
  sym_group(sp, sym, &grp);
  res->nsym = grp.nsym;
  /* depth 0 (cheese.cu:1794-1801) */
  for (int i = 0; i < E; i++) if (!store64 && !zfits32(sp->target[i])) { res->rc = 4; return 4; }
  if (is_goal(sp, sp->target, sp->tk)) { res->depth0 = 1; res->rc = 0; return 0; }

  /* frontier: level l has n[l] nodes with parent index and gate; parents' residuals kept for the next level */
  uint32_t *par[CZO_DMAX + 1] = {0};
  uint8_t *gat[CZO_DMAX + 1] = {0};
  long cnt[CZO_DMAX + 1] = {0};
  cnt[0] = 1;
  czo_zw *R = malloc(sizeof(czo_zw) * E);
  int *Rk = malloc(sizeof(int));
  int16_t *g1 = malloc(sizeof(int16_t)), *g2 = malloc(sizeof(int16_t));
  memcpy(R, sp->target, sizeof(czo_zw) * E);
  Rk[0] = sp->tk; g1[0] = -1; g2[0] = -1;
  int rc = 1;
  for (int t = 1; t <= depth; t++) {
    const long m = cnt[t - 1];
    const long nc = m * G;
    const int keep = t < depth;
    lvl_in L = {sp, &grp, t, depth, store64, m, R, Rk, g1, g2};
    uint8_t *st = malloc((size_t)nc);
    uint64_t *k1 = malloc(sizeof(uint64_t) * (size_t)nc), *k2 = malloc(sizeof(uint64_t) * (size_t)nc);
#pragma omp parallel for schedule(dynamic, 64)
    for (long o = 0; o < nc; o++) st[o] = (uint8_t)child_status(&L, o / G, (int)(o % G), &k1[o], &k2[o]);
    long nw2 = 0, nw3 = 0, ndead = 0, nalive = 0, nfound = 0, first = -1, novf = 0;
    for (long o = 0; o < nc; o++) {
      switch (st[o]) {
        case W2CUT: nw2++; break;
        case W3CUT: nw3++; break;
        case DEAD: ndead++; break;
        case ALIVE: nalive++; break;
        case FOUND: nfound++; if (first < 0) first = o; break;
        default: novf++;
      }
    }
    if (novf) { rc = 4; free(st); free(k1); free(k2); break; }
    if (first >= 0) {     /* the lexicographically first circuit of this level (cheese.cu:1311-1318) */
      uint32_t i = (uint32_t)(first / G);
      res->found_len = t;
      res->found[t - 1] = (int)(first % G);
      for (int l = t - 1; l >= 1; l--) { res->found[l - 1] = gat[l][i]; i = par[l][i]; }
      res->n_found = nfound;
      rc = 0;
      free(st); free(k1); free(k2);
      break;
    }
    /* survivors in index order, then one per class: the smallest index (cheese.cu:1335-1343) */
    long na = 0;
    ckey *K = malloc(sizeof(ckey) * (size_t)(keep ? nalive + 1 : 1));
    if (keep) for (long o = 0; o < nc; o++) if (st[o] == ALIVE) { K[na].h1 = k1[o]; K[na].h2 = k2[o]; K[na].idx = o; na++; }
    free(st); free(k1); free(k2);
    long distinct = na;
    long *kept = malloc(sizeof(long) * (size_t)(na + 1));
    if (dedupe && na > 1) {
      qsort(K, (size_t)na, sizeof(ckey), ckey_cmp);
      distinct = 0;
      czo_zw *A = malloc(sizeof(czo_zw) * E), *B = malloc(sizeof(czo_zw) * E);
      for (long s = 0; s < na;) {
        long e = s + 1;
        while (e < na && K[e].h1 == K[s].h1 && K[e].h2 == K[s].h2) e++;
        const long base = distinct;
        for (long j = s; j < e; j++) {      /* exact classes within one key run; first (smallest index) kept */
          int dup = 0;
          if (e - s > 1) {
            int ka = Rk[K[j].idx / G];
            memcpy(A, R + (K[j].idx / G) * E, sizeof(czo_zw) * E);
            czo_apply_inv(sp, (int)(K[j].idx % G), A, &ka);
            for (long x = base; x < distinct && !dup; x++) {
              int kb = Rk[kept[x] / G];
              memcpy(B, R + (kept[x] / G) * E, sizeof(czo_zw) * E);
              czo_apply_inv(sp, (int)(kept[x] % G), B, &kb);
              dup = same_class(sp, &grp, A, ka, B, kb);
            }
          }
          if (!dup) kept[distinct++] = K[j].idx;
        }
        s = e;
      }
      free(A); free(B);
      qsort(kept, (size_t)distinct, sizeof(long), long_cmp);
    } else {
      for (long j = 0; j < na; j++) kept[j] = K[j].idx;
    }
    free(K);
    czo_level *lv = &res->lev[res->nlev++];
    lv->t = t; lv->parents = m; lv->prefixes = m * G - nw2; lv->cut_w3 = nw3; lv->cut_lb = ndead;
    lv->survivors = nalive; lv->distinct = distinct; lv->proved = distinct == 0;
    if (!distinct) { free(kept); rc = 1; break; }
    /* append the level: parent index, gate, residual, last two gates */
    par[t] = malloc(sizeof(uint32_t) * (size_t)distinct);
    gat[t] = malloc((size_t)distinct);
    czo_zw *R2 = malloc(sizeof(czo_zw) * E * (size_t)distinct);
    int *Rk2 = malloc(sizeof(int) * (size_t)distinct);
    int16_t *n1 = malloc(sizeof(int16_t) * (size_t)distinct), *n2 = malloc(sizeof(int16_t) * (size_t)distinct);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < distinct; j++) {
      const long o = kept[j], i = o / G;
      par[t][j] = (uint32_t)i; gat[t][j] = (uint8_t)(o % G);
      memcpy(R2 + j * E, R + i * E, sizeof(czo_zw) * E);
      Rk2[j] = Rk[i];
      czo_apply_inv(sp, (int)(o % G), R2 + j * E, &Rk2[j]);
      n1[j] = (int16_t)(o % G); n2[j] = g1[i];
    }
    cnt[t] = distinct;
    free(kept); free(R); free(Rk); free(g1); free(g2);
    R = R2; Rk = Rk2; g1 = n1; g2 = n2;
  }
  free(R); free(Rk); free(g1); free(g2);
  for (int l = 1; l <= CZO_DMAX; l++) { free(par[l]); free(gat[l]); }
  res->rc = rc;
  return rc;
}
