/* tc-oracle: CPU restatement of the reference's T-count search (src/tcount.cu). TEST INFRASTRUCTURE ONLY: the
 * checker of cheese_b200's T-count path, never linked into it. Same arguments, stdout lines and exit codes as the
 * reference's tcount (tcount.cu:452-532), no table cache, "seconds" printed as 0.00:
 *   tc-oracle TSPEC [--table K] [--max T]
 * Practical for small tables (2 qubits with K <= 4, 3 qubits with K <= 2). Coset equality uses a canonical form
 * (exponent + columns sign-normalised and sorted), so it is exact by construction; the reference compares the same
 * multisets of sign-normalised columns (tcount.cu:176-188). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXP 64
#define MAXT 32

static int n, P, G, E0, *UX, *UY, *TR, *TS;

typedef struct { int x[MAXP * MAXP], y[MAXP * MAXP], e; } mat;

/* S <- R(P_p)^-1 S, normalised (tcount.cu:80-113) */
static int peel(mat *M, int p) {
  static __thread int nx[MAXP * MAXP], ny[MAXP * MAXP];
  int ovf = 0;
  for (int a = 0; a < P; a++) {
    const int r = TR[(p - 1) * P + a], s = TS[(p - 1) * P + a];
    for (int c = 0; c < P; c++) {
      const long long ox = M->x[a * P + c], oy = M->y[a * P + c];
      long long vx, vy;
      if (r < 0) { vx = 2 * oy; vy = ox; }
      else { vx = ox - (long long)s * M->x[r * P + c]; vy = oy - (long long)s * M->y[r * P + c]; }
      if (vx > INT32_MAX || vx < INT32_MIN || vy > INT32_MAX || vy < INT32_MIN) ovf = 1;
      nx[a * P + c] = (int)vx; ny[a * P + c] = (int)vy;
    }
  }
  memcpy(M->x, nx, sizeof(int) * P * P); memcpy(M->y, ny, sizeof(int) * P * P);
  M->e++;
  for (;;) {
    if (M->e <= 0) break;
    int even = 1;
    for (int i = 0; i < P * P && even; i++) even = !(M->x[i] & 1);
    if (!even) break;
    for (int i = 0; i < P * P; i++) { const int x = M->x[i]; M->x[i] = M->y[i]; M->y[i] = x / 2; }
    M->e--;
  }
  return ovf;
}

/* canonical form of the coset: exponent, then columns sign-normalised (first nonzero positive) and sorted */
typedef struct { int e; int col[MAXP][2 * MAXP]; } canon;
static int colcmp(const void *a, const void *b) { return memcmp(a, b, sizeof(int) * 2 * P); }
static void canonical(const mat *M, canon *K) {
  memset(K, 0, sizeof *K);
  K->e = M->e;
  for (int c = 0; c < P; c++) {
    int s = 1;
    for (int r = 0; r < P; r++) {
      const int x = M->x[r * P + c], y = M->y[r * P + c];
      if (x || y) { s = (x > 0 || (x == 0 && y > 0)) ? 1 : -1; break; }
    }
    for (int r = 0; r < P; r++) { K->col[c][2 * r] = s * M->x[r * P + c]; K->col[c][2 * r + 1] = s * M->y[r * P + c]; }
  }
  qsort(K->col, P, sizeof K->col[0], colcmp);
}
static uint64_t chash(const canon *K) {
  uint64_t h = 1469598103934665603ULL ^ (uint64_t)K->e;
  for (int c = 0; c < P; c++)
    for (int i = 0; i < 2 * P; i++) { h ^= (uint64_t)(uint32_t)K->col[c][i]; h *= 1099511628211ULL; }
  return h;
}
static int ceq(const canon *A, const canon *B) { return A->e == B->e && !memcmp(A->col, B->col, sizeof(int) * 2 * P * P); }

/* tree of peel sequences; level 0 = the base */
typedef struct { long n[MAXT + 1]; uint32_t *par[MAXT + 1]; uint8_t *gat[MAXT + 1]; int top; } tree;
static void path(const tree *T, int t, uint32_t i, uint8_t *seq) { for (int l = t; l >= 1; l--) { seq[l - 1] = T->gat[l][i]; i = T->par[l][i]; } }
static int build(mat *M, int base_u, const uint8_t *seq, int len) {
  int ovf = 0;
  for (int i = 0; i < P * P; i++) { M->x[i] = base_u ? UX[i] : (i / P == i % P); M->y[i] = base_u ? UY[i] : 0; }
  M->e = base_u ? E0 : 0;
  for (int i = 0; i < len; i++) ovf |= peel(M, seq[i]);
  return ovf;
}
static uint64_t node_key(const tree *T, int base_u, int t, uint32_t i, canon *K, int *ovf) {
  uint8_t seq[MAXT + 1];
  mat M;
  path(T, t, i, seq);
  *ovf |= build(&M, base_u, seq, t);
  canonical(&M, K);
  return chash(K);
}

typedef struct { uint64_t h; long idx; int lvl; } ent;
static int entcmp(const void *a, const void *b) {
  const ent *x = a, *y = b;
  if (x->h != y->h) return x->h < y->h ? -1 : 1;
  if (x->lvl != y->lvl) return x->lvl - y->lvl;
  return x->idx < y->idx ? -1 : x->idx > y->idx;
}
static int ovf_g;
static int longcmp(const void *a, const void *b) { const long x = *(const long *)a, y = *(const long *)b; return x < y ? -1 : x > y; }

/* table: every node so far (level, index), sorted by hash */
typedef struct { ent *e; long n, cap; } table;
static void tab_add(table *S, ent x) {
  if (S->n == S->cap) { S->cap = S->cap ? 2 * S->cap : 1024; S->e = realloc(S->e, sizeof(ent) * S->cap); }
  S->e[S->n++] = x;
}
/* the table entry of a coset equal to K with level <= maxc (smallest level), or -1 */
static long tab_find(const table *S, const tree *D, uint64_t h, const canon *K, int maxc) {
  long lo = 0, hi = S->n;
  while (lo < hi) { const long m = (lo + hi) / 2; if (S->e[m].h < h) lo = m + 1; else hi = m; }
  for (long x = lo; x < S->n && S->e[x].h == h; x++) {   /* sorted by level within a hash */
    if (S->e[x].lvl > maxc) continue;
    canon B;
    node_key(D, 0, S->e[x].lvl, (uint32_t)S->e[x].idx, &B, &ovf_g);
    if (ceq(K, &B)) return x;
  }
  return -1;
}

/* one more level of T (tcount.cu:327-395); table: drop cosets of lower levels and add the rest */
static long grow(tree *T, int base_u, table *S, const char *tag) {
  const int t = T->top + 1, tp = t - 1;
  const long m = T->n[tp], nc = m * G;
  ent *ch = malloc(sizeof(ent) * (nc ? nc : 1));
  canon K;
#pragma omp parallel for schedule(dynamic, 8) private(K)
  for (long i = 0; i < m; i++) {
    uint8_t seq[MAXT + 1];
    mat A, B;
    int ovf = 0;
    path(T, tp, (uint32_t)i, seq);
    ovf |= build(&A, base_u, seq, tp);
    for (int p = 1; p <= G; p++) {
      B = A;
      ovf |= peel(&B, p);
      canonical(&B, &K);
      ch[i * G + p - 1].h = chash(&K); ch[i * G + p - 1].idx = i * G + p - 1; ch[i * G + p - 1].lvl = 0;
    }
    if (ovf) {
#pragma omp atomic write
      ovf_g = 1;
    }
  }
  qsort(ch, nc, sizeof(ent), entcmp);
  /* one child per coset, the smallest index: exact comparison inside equal-hash groups */
  long *kept = malloc(sizeof(long) * (nc ? nc : 1)), nk = 0;
  canon A, B;
  for (long s = 0; s < nc;) {
    long e = s + 1;
    while (e < nc && ch[e].h == ch[s].h) e++;
    const long base = nk;
    for (long j = s; j < e; j++) {
      int dup = 0;
      if (e - s > 1) {
        uint8_t seq[MAXT + 1];
        mat M;
        path(T, tp, (uint32_t)(ch[j].idx / G), seq); seq[tp] = (uint8_t)(ch[j].idx % G + 1);
        ovf_g |= build(&M, base_u, seq, tp + 1);
        canonical(&M, &A);
        for (long x = base; x < nk && !dup; x++) {
          path(T, tp, (uint32_t)(kept[x] / G), seq); seq[tp] = (uint8_t)(kept[x] % G + 1);
          ovf_g |= build(&M, base_u, seq, tp + 1);
          canonical(&M, &B);
          dup = ceq(&A, &B);
        }
      }
      if (!dup) kept[nk++] = ch[j].idx;
    }
    s = e;
  }
  free(ch);
  qsort(kept, nk, sizeof(long), longcmp);
  T->par[t] = malloc(sizeof(uint32_t) * (nk ? nk : 1)); T->gat[t] = malloc(nk ? nk : 1);
  long fresh = 0;
  for (long j = 0; j < nk; j++) {
    const uint32_t par = (uint32_t)(kept[j] / G);
    const uint8_t g = (uint8_t)(kept[j] % G + 1);
    if (S) {                   /* seen at a lower level? */
      T->par[t][fresh] = par; T->gat[t][fresh] = g;
      T->n[t] = fresh + 1; T->top = t;
      const uint64_t h = node_key(T, base_u, t, (uint32_t)fresh, &A, &ovf_g);
      if (tab_find(S, T, h, &A, t - 1) >= 0) continue;
      fresh++;
    } else {
      T->par[t][fresh] = par; T->gat[t][fresh] = g; fresh++;
    }
  }
  T->n[t] = fresh; T->top = t;
  if (S) {
    for (long j = 0; j < fresh; j++) { ent x = {node_key(T, base_u, t, (uint32_t)j, &A, &ovf_g), j, t}; tab_add(S, x); }
    qsort(S->e, S->n, sizeof(ent), entcmp);
  }
  printf("{%s\"t\": %d, \"parents\": %ld, \"children\": %ld, \"cosets\": %ld, \"new\": %ld, \"seconds\": 0.00}\n", tag, t, m,
         nc, nk, fresh);
  fflush(stdout);
  free(kept);
  return fresh;
}

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: tc-oracle SPEC [--table K] [--max T]\n"); return 3; }
  FILE *f = fopen(argv[1], "r");
  char tok[64];
  if (!f || fscanf(f, "%63s", tok) != 1 || strcmp(tok, "tcount-spec")) { fprintf(stderr, "not a tcount spec\n"); return 2; }
  int ver;
  if (fscanf(f, "%d", &ver) != 1) return 2;
  while (fscanf(f, "%63s", tok) == 1) {
    if (!strcmp(tok, "n")) { if (fscanf(f, "%d", &n) != 1) return 2; P = 1 << (2 * n); G = P - 1; }
    else if (!strcmp(tok, "channel")) {
      if (fscanf(f, "%d", &E0) != 1) return 2;
      UX = malloc(sizeof(int) * P * P); UY = malloc(sizeof(int) * P * P);
      for (int i = 0; i < P * P; i++) if (fscanf(f, "%d %d", &UX[i], &UY[i]) != 2) return 2;
    } else if (!strcmp(tok, "rotations")) {
      int m;
      if (fscanf(f, "%d", &m) != 1) return 2;
      TR = malloc(sizeof(int) * m * P); TS = malloc(sizeof(int) * m * P);
      for (int i = 0; i < m * P; i++) if (fscanf(f, "%d %d", &TR[i], &TS[i]) != 2) return 2;
    } else if (!strcmp(tok, "end")) break;
    else { fprintf(stderr, "unknown field %s\n", tok); return 2; }
  }
  fclose(f);
  if (P > MAXP || n < 1) { fprintf(stderr, "n = %d not supported (1 <= n <= 3)\n", n); return 3; }
  int K = 4, maxt = 16;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--table") && i + 1 < argc) K = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--max") && i + 1 < argc) maxt = atoi(argv[++i]);
  }
  static tree D, T;
  static table S;
  D.n[0] = 1; T.n[0] = 1;
  canon A;
  { ent root = {node_key(&D, 0, 0, 0, &A, &ovf_g), 0, 0}; tab_add(&S, root); }
  for (int l = 1; l <= K; l++) if (!grow(&D, 0, &S, "\"dir\": \"table\", ")) break;
  if (ovf_g) { fprintf(stderr, "coefficient overflow (int32)\n"); return 4; }
  fprintf(stderr, "table: %ld cosets with T-count <= %d\n", S.n, D.top);
  for (int j = 0; j <= maxt; j++) {
    if (j > 0 && !grow(&T, 1, NULL, "\"dir\": \"search\", ")) break;
    if (ovf_g) { fprintf(stderr, "coefficient overflow (int32)\n"); return 4; }
    const int maxc = D.top < maxt - j ? D.top : maxt - j;
    long best = -1, bestx = -1;
    int bestc = 1 << 30;
    for (long i = 0; i < T.n[j]; i++) {
      const uint64_t h = node_key(&T, 1, j, (uint32_t)i, &A, &ovf_g);
      const long x = tab_find(&S, &D, h, &A, maxc);
      if (x >= 0 && S.e[x].lvl < bestc) { bestc = S.e[x].lvl; best = i; bestx = x; }
    }
    if (best >= 0) {
      uint8_t fw[MAXT + 1], tb[MAXT + 1];
      path(&T, j, (uint32_t)best, fw);
      path(&D, bestc, (uint32_t)S.e[bestx].idx, tb);
      printf("{\"tcount\": %d, \"rotations\": [", j + bestc);
      int first = 1;
      for (int i = 0; i < j; i++) { printf("%s[%d, 0]", first ? "" : ", ", fw[i]); first = 0; }
      for (int i = bestc - 1; i >= 0; i--) { printf("%s[%d, 1]", first ? "" : ", ", tb[i]); first = 0; }
      printf("], \"split\": [%d, %d], \"seconds\": 0.00}\n", j, bestc);
      return 0;
    }
    if (j + D.top >= maxt) break;
  }
  printf("{\"tcount_above\": %d, \"seconds\": 0.00}\n", maxt);
  return 1;
}
