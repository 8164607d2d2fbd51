/* rus-oracle: CPU restatement of the reference's RUS T-count search (src/rus.cu). TEST INFRASTRUCTURE ONLY: the
 * checker of cheese_b200's RUS path, never linked into it. Same arguments, stdout lines and exit codes as the
 * reference's rus (rus.cu:512-587), no table cache, "seconds" printed as 0.00:
 *   rus-oracle RSPEC [--table K] [--max T]
 * Practical for tables up to K = 6 or so. Coset grouping uses the exact invariant that the reference hashes
 * (exponent, sign-normalised row 0, multiset of the sign-normalised rows 1..15; rus.cu:120-144), so it is exact by
 * construction; inside a group the reference's rule applies (members equal to the group's first by a Clifford are
 * dropped, rus.cu:262-282), with the Clifford found the reference's way (generator images, rus.cu:152-200). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NR 16
#define NC 4
#define NE (NR * NC)
#define NCL 11520
#define MAXT 32
#define INV (1 + 2 * NC + (NR - 1) * 2 * NC)   /* ints of the grouping invariant */

static const int GEN[4] = {1, 3, 4, 12};       /* X_q0, Z_q0, X_q1, Z_q1 */

/* ---- spec (rus.cu:470-510) ---- */
static int nroot, te, *rx, *ry, *re_, tx[NE], ty[NE], tr[15 * NR], ts[15 * NR], bygen[1 << 20];
static unsigned char perm[NCL * NR];
static signed char sgn[NCL * NR];

static void die(int rc, const char *m) { fprintf(stderr, "%s\n", m); exit(rc); }

static void read_mat(FILE *f, int *x, int *y, int *e) {
  if (fscanf(f, "%d", e) != 1) die(2, "bad matrix");
  for (int i = 0; i < NE; i++)
    if (fscanf(f, "%d %d", &x[i], &y[i]) != 2) die(2, "bad matrix");
}

static void read_spec(const char *path) {
  FILE *f = fopen(path, "r");
  if (!f) die(2, "cannot read spec");
  char tok[64];
  int ver, have_t = 0, have_r = 0, have_c = 0;
  if (fscanf(f, "%63s %d", tok, &ver) != 2 || strcmp(tok, "rus-spec")) die(2, "not a rus spec");
  while (fscanf(f, "%63s", tok) == 1) {
    if (!strcmp(tok, "table-root")) { read_mat(f, tx, ty, &te); have_t = 1; }
    else if (!strcmp(tok, "roots")) {
      if (fscanf(f, "%d", &nroot) != 1 || nroot <= 0) die(2, "bad roots");
      rx = malloc(sizeof(int) * NE * nroot); ry = malloc(sizeof(int) * NE * nroot); re_ = malloc(sizeof(int) * nroot);
      for (int r = 0; r < nroot; r++) read_mat(f, rx + r * NE, ry + r * NE, &re_[r]);
    } else if (!strcmp(tok, "rotations")) {
      int m;
      if (fscanf(f, "%d", &m) != 1 || m != 15) die(2, "incomplete spec");
      for (int i = 0; i < m * NR; i++)
        if (fscanf(f, "%d %d", &tr[i], &ts[i]) != 2) die(2, "bad rotations");
      have_r = 1;
    } else if (!strcmp(tok, "cliffords")) {
      int m;
      if (fscanf(f, "%d", &m) != 1 || m != NCL) die(2, "expected 11520 Cliffords");
      for (int i = 0; i < m * NR; i++) {
        int p, g;
        if (fscanf(f, "%d %d", &p, &g) != 2) die(2, "bad cliffords");
        perm[i] = (unsigned char)p; sgn[i] = (signed char)g;
      }
      have_c = 1;
    } else if (!strcmp(tok, "end")) break;
    else die(2, "unknown field");
  }
  fclose(f);
  if (!nroot || !have_t || !have_r || !have_c) die(2, "incomplete spec");
  memset(bygen, -1, sizeof bygen);
  for (int c = 0; c < NCL; c++) {
    int key = 0;
    for (int g = 0; g < 4; g++) key |= ((perm[c * NR + GEN[g]] << 1) | (sgn[c * NR + GEN[g]] < 0)) << (5 * g);
    if (bygen[key] >= 0) die(2, "Clifford table: generator images not unique");
    bygen[key] = c;
  }
}

/* ---- matrices (x + y sqrt2) / sqrt2^e, rus.cu:86-118 ---- */
typedef struct { int x[NE], y[NE], e; } mat;
static int ovf;

static void peel(mat *M, int p) {
  int nx[NE], ny[NE];
  for (int a = 0; a < NR; a++) {
    const int r = tr[(p - 1) * NR + a], s = ts[(p - 1) * NR + a];
    for (int c = 0; c < NC; c++) {
      const long long ox = M->x[a * NC + c], oy = M->y[a * NC + c];
      long long vx, vy;
      if (r < 0) { vx = 2 * oy; vy = ox; }
      else { vx = ox - (long long)s * M->x[r * NC + c]; vy = oy - (long long)s * M->y[r * NC + c]; }
      if (vx > INT32_MAX || vx < INT32_MIN || vy > INT32_MAX || vy < INT32_MIN) ovf = 1;
      nx[a * NC + c] = (int)vx; ny[a * NC + c] = (int)vy;
    }
  }
  memcpy(M->x, nx, sizeof nx); memcpy(M->y, ny, sizeof ny);
  M->e++;
  for (;;) {
    if (M->e <= 0) break;
    int even = 1;
    for (int i = 0; i < NE && even; i++) even = !(M->x[i] & 1);
    if (!even) break;
    for (int i = 0; i < NE; i++) { const int x = M->x[i]; M->x[i] = M->y[i]; M->y[i] = x / 2; }
    M->e--;
  }
}

/* ---- trees: level l holds parent index and peel (1..15) per node ---- */
typedef struct {
  int top;
  long n[MAXT + 2];
  uint32_t *par[MAXT + 2];
  unsigned char *gat[MAXT + 2];
} tree;

static void build(mat *M, const int *bx, const int *by, const int *be, const tree *T, int t, uint32_t i, int extra,
                  uint32_t *root_out) {
  int seq[MAXT + 2];
  for (int l = t; l >= 1; l--) { seq[l - 1] = T->gat[l][i]; i = T->par[l][i]; }
  memcpy(M->x, bx + (size_t)i * NE, sizeof M->x);
  memcpy(M->y, by + (size_t)i * NE, sizeof M->y);
  M->e = be[i];
  for (int l = 0; l < t; l++) peel(M, seq[l]);
  if (extra) peel(M, extra);
  if (root_out) *root_out = i;
}

/* grouping invariant: exponent, sign-normalised row 0, sorted sign-normalised rows 1..15 */
static int rowless(const int *a, const int *b) {
  for (int i = 0; i < 2 * NC; i++) if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}
static int rowsort(const void *a, const void *b) { return rowless((const int *)a, (const int *)b); }
static void invariant(const mat *M, int *out) {
  int rows[NR][2 * NC];
  for (int a = 0; a < NR; a++) {
    int s = 1;
    for (int c = 0; c < NC; c++) {
      const int x = M->x[a * NC + c], y = M->y[a * NC + c];
      if (x) { s = x > 0 ? 1 : -1; break; }
      if (y) { s = y > 0 ? 1 : -1; break; }
    }
    for (int c = 0; c < NC; c++) { rows[a][2 * c] = s * M->x[a * NC + c]; rows[a][2 * c + 1] = s * M->y[a * NC + c]; }
  }
  qsort(rows[1], NR - 1, sizeof rows[1], rowsort);
  out[0] = M->e;
  memcpy(out + 1, rows, sizeof rows);
}

/* Clifford c with B = C_c A (B[a] = s_c(a) A[pi_c(a)]), else -1: the generator-image enumeration of rus.cu:152-200 */
static int row_eq(const mat *A, int ra, int s, const mat *B, int rb) {
  for (int c = 0; c < NC; c++)
    if (s * A->x[ra * NC + c] != B->x[rb * NC + c] || s * A->y[ra * NC + c] != B->y[rb * NC + c]) return 0;
  return 1;
}
static int com(int p, int q) { return tr[(p - 1) * NR + q] < 0; }
static int equiv(const mat *A, const mat *B) {
  if (A->e != B->e) return -1;
  int cand[4][30], nc[4];
  for (int g = 0; g < 4; g++) {
    nc[g] = 0;
    for (int r = 1; r < NR; r++)
      for (int s = 1; s >= -1; s -= 2)
        if (row_eq(A, r, s, B, GEN[g])) cand[g][nc[g]++] = (r << 1) | (s < 0);
    if (!nc[g]) return -1;
  }
  for (int i0 = 0; i0 < nc[0]; i0++) {
    const int b0 = cand[0][i0] >> 1;
    for (int i1 = 0; i1 < nc[1]; i1++) {
      const int b1 = cand[1][i1] >> 1;
      if (com(b0, b1)) continue;
      for (int i2 = 0; i2 < nc[2]; i2++) {
        const int b2 = cand[2][i2] >> 1;
        if (!com(b0, b2) || !com(b1, b2)) continue;
        for (int i3 = 0; i3 < nc[3]; i3++) {
          const int b3 = cand[3][i3] >> 1;
          if (com(b2, b3) || !com(b0, b3) || !com(b1, b3)) continue;
          const int key = cand[0][i0] | cand[1][i1] << 5 | cand[2][i2] << 10 | cand[3][i3] << 15;
          const int c = bygen[key];
          if (c < 0) continue;
          int ok = 1;
          for (int a = 0; ok && a < NR; a++) ok = row_eq(A, perm[c * NR + a], sgn[c * NR + a], B, a);
          if (ok) return c;
        }
      }
    }
  }
  return -1;
}

/* ---- the table of seen cosets: (invariant, level, index), sorted by invariant then level then index ---- */
typedef struct { int inv[INV]; uint32_t lvl, idx; } entry;
static int entry_cmp(const void *a, const void *b) {
  const entry *x = a, *y = b;
  for (int i = 0; i < INV; i++) if (x->inv[i] != y->inv[i]) return x->inv[i] < y->inv[i] ? -1 : 1;
  if (x->lvl != y->lvl) return x->lvl < y->lvl ? -1 : 1;
  return x->idx < y->idx ? -1 : x->idx > y->idx;
}
static long lower(const entry *D, long n, const int *inv) {
  long lo = 0, hi = n;
  while (lo < hi) {
    const long mid = (lo + hi) / 2;
    int c = 0;
    for (int i = 0; i < INV && !c; i++) if (D[mid].inv[i] != inv[i]) c = D[mid].inv[i] < inv[i] ? -1 : 1;
    if (c < 0) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* a child: its index p * 15 + (g - 1) over the parent level, its invariant */
typedef struct { uint32_t idx; int inv[INV]; } child;
static int child_cmp(const void *a, const void *b) {
  const child *x = a, *y = b;
  for (int i = 0; i < INV; i++) if (x->inv[i] != y->inv[i]) return x->inv[i] < y->inv[i] ? -1 : 1;
  return x->idx < y->idx ? -1 : x->idx > y->idx;
}
static int u32cmp(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

static entry *seen;
static long nseen;

/* one more level of T (peels off the matrices bx/by/be); with table: drop cosets already seen (rus.cu:360-441) */
static long grow(const int *bx, const int *by, const int *be, tree *T, int table, const char *tag) {
  const int t = T->top + 1, tp = t - 1;
  const long m = T->n[tp], nk = m * 15;
  child *C = malloc(sizeof(child) * (nk ? nk : 1));
  mat M;
  for (long o = 0; o < nk; o++) {
    build(&M, bx, by, be, T, tp, (uint32_t)(o / 15), (int)(o % 15) + 1, NULL);
    C[o].idx = (uint32_t)o;
    invariant(&M, C[o].inv);
  }
  if (ovf) die(4, "coefficient overflow (int32)");
  qsort(C, nk, sizeof(child), child_cmp);
  uint32_t *keep = malloc(sizeof(uint32_t) * (nk ? nk : 1));
  long kept = 0;
  mat H, B;
  for (long j = 0, h = 0; j < nk; j++) {
    if (j == 0 || memcmp(C[j].inv, C[j - 1].inv, sizeof C[j].inv)) { h = j; keep[kept++] = C[j].idx; continue; }
    build(&H, bx, by, be, T, tp, C[h].idx / 15, (int)(C[h].idx % 15) + 1, NULL);
    build(&B, bx, by, be, T, tp, C[j].idx / 15, (int)(C[j].idx % 15) + 1, NULL);
    if (equiv(&H, &B) < 0) keep[kept++] = C[j].idx;
  }
  if (ovf) die(4, "coefficient overflow (int32)");
  qsort(keep, kept, sizeof(uint32_t), u32cmp);
  T->top = t;
  T->n[t] = kept;
  T->par[t] = malloc(sizeof(uint32_t) * (kept ? kept : 1));
  T->gat[t] = malloc(kept ? kept : 1);
  for (long j = 0; j < kept; j++) { T->par[t][j] = keep[j] / 15; T->gat[t][j] = (unsigned char)(keep[j] % 15 + 1); }
  long fresh = kept;
  if (table && kept) {
    long nf = 0;
    entry *add = malloc(sizeof(entry) * kept);
    for (long j = 0; j < kept; j++) {
      int inv[INV], hit = 0;
      build(&B, bx, by, be, T, t, (uint32_t)j, 0, NULL);
      invariant(&B, inv);
      for (long x = lower(seen, nseen, inv); !hit && x < nseen && !memcmp(seen[x].inv, inv, sizeof inv); x++) {
        if ((int)seen[x].lvl > t - 1) continue;
        build(&H, bx, by, be, T, (int)seen[x].lvl, seen[x].idx, 0, NULL);
        hit = equiv(&H, &B) >= 0;
      }
      if (!hit) {
        T->par[t][nf] = T->par[t][j]; T->gat[t][nf] = T->gat[t][j];
        memcpy(add[nf].inv, inv, sizeof inv);
        add[nf].lvl = (uint32_t)t; add[nf].idx = (uint32_t)nf;
        nf++;
      }
    }
    if (ovf) die(4, "coefficient overflow (int32)");
    fresh = nf;
    T->n[t] = nf;
    seen = realloc(seen, sizeof(entry) * (nseen + nf));
    memcpy(seen + nseen, add, sizeof(entry) * nf);
    nseen += nf;
    qsort(seen, nseen, sizeof(entry), entry_cmp);
    free(add);
  }
  printf("{%s\"t\": %d, \"parents\": %ld, \"children\": %ld, \"cosets\": %ld, \"new\": %ld, \"seconds\": 0.00}\n", tag, t,
         m, nk, kept, fresh);
  fflush(stdout);
  free(C); free(keep);
  return fresh;
}

int main(int argc, char **argv) {
  if (argc < 2) die(3, "usage: rus-oracle SPEC [--table K] [--max T]");
  read_spec(argv[1]);
  int K = 8, maxt = 16;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--table") && i + 1 < argc) K = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--max") && i + 1 < argc) maxt = atoi(argv[++i]);
  }
  /* table: level 0 is the coset of J00 */
  tree D = {0};
  D.n[0] = 1;
  mat M;
  memcpy(M.x, tx, sizeof tx); memcpy(M.y, ty, sizeof ty); M.e = te;
  seen = malloc(sizeof(entry));
  invariant(&M, seen[0].inv);
  seen[0].lvl = 0; seen[0].idx = 0; nseen = 1;
  for (int l = 1; l <= K; l++)
    if (!grow(tx, ty, &te, &D, 1, "\"dir\": \"table\", ")) break;
  /* search: peel rotations off the roots (rus.cu:549-586) */
  tree T = {0};
  T.n[0] = nroot;
  for (int j = 0; j <= maxt; j++) {
    if (j > 0 && !grow(rx, ry, re_, &T, 0, "\"dir\": \"search\", ")) break;
    const int maxc = D.top < maxt - j ? D.top : maxt - j;
    long best = -1, bestx = -1;
    int bestc = 1 << 30, bestcl = -1;
    mat A, Bm;
    for (long i = 0; i < T.n[j]; i++) {
      int inv[INV];
      build(&A, rx, ry, re_, &T, j, (uint32_t)i, 0, NULL);
      invariant(&A, inv);
      long res = -1;
      int rl = 1 << 30, rc = -1;
      for (long x = lower(seen, nseen, inv); x < nseen && !memcmp(seen[x].inv, inv, sizeof inv); x++) {
        if ((int)seen[x].lvl > maxc || (int)seen[x].lvl >= rl) continue;
        build(&Bm, tx, ty, &te, &D, (int)seen[x].lvl, seen[x].idx, 0, NULL);
        const int c = equiv(&Bm, &A);
        if (c >= 0) { res = x; rl = (int)seen[x].lvl; rc = c; }
      }
      if (res >= 0 && (int)seen[res].lvl < bestc) { bestc = (int)seen[res].lvl; best = i; bestx = res; bestcl = rc; }
    }
    if (ovf) die(4, "coefficient overflow (int32)");
    if (best >= 0) {
      int fw[MAXT + 2], tb[MAXT + 2];
      uint32_t i = (uint32_t)best;
      for (int l = j; l >= 1; l--) { fw[l - 1] = T.gat[l][i]; i = T.par[l][i]; }
      const uint32_t root = i;
      i = seen[bestx].idx;
      for (int l = bestc; l >= 1; l--) { tb[l - 1] = D.gat[l][i]; i = D.par[l][i]; }
      printf("{\"tcount\": %d, \"root\": %u, \"fw\": [", j + bestc, root);
      for (int l = 0; l < j; l++) printf("%s%d", l ? ", " : "", fw[l]);
      printf("], \"cliff\": %d, \"tb\": [", bestcl);
      for (int l = 0; l < bestc; l++) printf("%s%d", l ? ", " : "", tb[l]);
      printf("], \"split\": [%d, %d], \"seconds\": 0.00}\n", j, bestc);
      return 0;
    }
    if (j + D.top >= maxt) break;
  }
  printf("{\"tcount_above\": %d, \"seconds\": 0.00}\n", maxt);
  return 1;
}
