/* cz_oracle: CPU restatement of cheese's level-synchronous branch-and-bound (gate-count search).
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA product path: tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it, nothing in cheese_b200/ links or calls it. It restates the algorithm of
 * the reference's src/cheese.cu (functions cited per definition in cz_oracle.c) in plain C11 + OpenMP, with its
 * own data layout (stored residuals instead of replay) and its own hash; equality of residual classes is always
 * decided exactly, so neither choice can change a result.
 *
 * Parity is pinned against (1) the reference's own verdicts (tests/check.sh of the reference), (2) the golden
 * per-level JSON produced by the reference CPU build compiled from its sources (oracle/_ref/cheese-cpu, see
 * tests/golden/make_golden.py), (3) the per-level counts quoted in the reference's docs.
 */
#ifndef CZ_ORACLE_H
#define CZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#define CZO_DMAX 48   /* longest prefix            (cheese.cu:53) */
#define CZO_GMAX 64   /* most candidates           (cheese.cu:54) */
#define CZO_LMAX 8    /* largest local dimension   (cheese.cu:55) */
#define CZO_CUTMAX 16 /* most cuts                 (cheese.cu:56) */
#define CZO_NMAX 8    /* 2^n, n <= 3               */

typedef struct { int64_t a, b, c, d; } czo_zw;

typedef struct {
  int n, N, G, depth, standard, lite, tdiv, tk, states;
  char names[CZO_GMAX][40];
  int gnq[CZO_GMAX], gq[CZO_GMAX][3], gik[CZO_GMAX];
  czo_zw ginv[CZO_GMAX][CZO_LMAX * CZO_LMAX];
  uint8_t bad2[CZO_GMAX * CZO_GMAX];
  uint32_t bad3[(CZO_GMAX * CZO_GMAX * CZO_GMAX + 31) / 32];
  czo_zw target[CZO_NMAX * CZO_NMAX];
  int ncuts, cutmask[CZO_CUTMAX], cutsize[CZO_CUTMAX], rad[CZO_CUTMAX];
  int ncx, cxtable[4096];
} czo_spec;

typedef struct {
  int t;
  long parents, prefixes, cut_w3, cut_lb, survivors, distinct;
  int proved;
} czo_level;

typedef struct {
  int rc;                      /* 0 circuit, 1 proof, 4 overflow (store64 = 0 only) */
  int nlev;
  czo_level lev[CZO_DMAX + 1];
  int found_len;
  int found[CZO_DMAX];
  long n_found;
  int depth0;                  /* 1: the target already equals the goal */
  int nsym;
} czo_result;

/* returns 0 or the reference's spec exit code (2); err gets a one-line message */
int czo_spec_parse(const char *text, size_t len, czo_spec *out, char *err, size_t errlen);

/* the plain search (cheese.cu:1762-1849, no --mitm/--table): store64 = 1 keeps int64 residuals (the reference's
 * -DSTORE64 build), 0 aborts with rc 4 on an int32 overflow like the default build */
int czo_search(const czo_spec *sp, int depth, int dedupe, int sym, int store64, int threads, czo_result *res);

/* single-residual helpers for unit tests (S: N*N entries, k: sqrt2 exponent) */
int czo_ptm_t(int n, const czo_zw *S, int k);                 /* ptm_wht (cheese.cu:429-449) */
int czo_ptm_sde(int n, const czo_zw *S, int k);               /* ptm_sde (cheese.cu:361-395) */
int czo_cut_rank(int n, const czo_zw *S, int mask, int sa);   /* cut_rank (cheese.cu:271-303) */
int czo_h_struct(int n, const czo_zw *S);                     /* h_struct (cheese.cu:322-338) */
int czo_support(int n, const czo_zw *S);                      /* support (cheese.cu:305-319) */
int czo_combine(int h, int t, int c2, int supp);              /* combine (cheese.cu:599-607) */
/* S <- S g^-1 then normalise; returns 1 if an int32 narrowing would have failed */
int czo_apply_inv(const czo_spec *sp, int g, czo_zw *S, int *k);

#endif
