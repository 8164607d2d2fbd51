/* clifford-oracle: CPU restatement of the reference's cliffopt (src/clifford.cu). TEST INFRASTRUCTURE ONLY: the
 * checker of cheese_b200's Clifford-table path, never linked into it.
 *   clifford-oracle JOB... [--beam B] [--dist-only]
 * Same job grammar, stdout and stderr lines as the reference (clifford.cu:213-384), times printed as 0.0 / 0.00.
 * The reference leaves one thing open: the order of the placement candidates of a T gate (k_cands appends them with
 * an atomic counter, clifford.cu:170-183), which decides ties in the beam. Here, as in cheese_b200, candidates are
 * ordered by (tableau value K, qubit q'), so oracle and product agree exactly; against the reference the BFS counts,
 * zero-T outputs and every segment's optimality agree exactly, and the summed length can differ on ties.
 *
 * Tableau (clifford.cu:16-19, 46-58): u64, row i < n the image of X_i, row n + i the image of Z_i, each row
 * (x bits | z bits << n | sign << 2n), the Hermitian Pauli (-1)^r i^(x.z) X^x Z^z. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { GH, GS, GSDG, GX, GZ, GCX, GY };
typedef struct { int k, a, b; } gate;
static int n, rb;

static uint32_t row(uint64_t T, int i) { return (uint32_t)((T >> (i * rb)) & ((1ULL << rb) - 1)); }
static uint64_t setrow(uint64_t T, int i, uint32_t r) {
  const uint64_t m = ((1ULL << rb) - 1) << (i * rb);
  return (T & ~m) | ((uint64_t)r << (i * rb));
}
static uint32_t mk(uint32_t x, uint32_t z, uint32_t r) { return x | (z << n) | (r << (2 * n)); }
static uint32_t RX(uint32_t w) { return w & ((1u << n) - 1); }
static uint32_t RZ(uint32_t w) { return (w >> n) & ((1u << n) - 1); }
static uint32_t RR(uint32_t w) { return (w >> (2 * n)) & 1; }
static uint64_t identity(void) {
  uint64_t T = 0;
  for (int i = 0; i < n; i++) { T = setrow(T, i, mk(1u << i, 0, 0)); T = setrow(T, n + i, mk(0, 1u << i, 0)); }
  return T;
}
/* G P G^dag on one row (clifford.cu:59-77) */
static uint32_t conj_row(uint32_t w, gate g) {
  uint32_t x = RX(w), z = RZ(w), r = RR(w);
  const uint32_t xa = (x >> g.a) & 1, za = (z >> g.a) & 1;
  if (g.k == GH) { r ^= xa & za; x = (x & ~(1u << g.a)) | (za << g.a); z = (z & ~(1u << g.a)) | (xa << g.a); }
  else if (g.k == GS) { r ^= xa & za; z ^= xa << g.a; }
  else if (g.k == GSDG) { r ^= xa & (za ^ 1); z ^= xa << g.a; }
  else if (g.k == GX) r ^= za;
  else if (g.k == GZ) r ^= xa;
  else if (g.k == GY) r ^= xa ^ za;
  else {
    const uint32_t xt = (x >> g.b) & 1, zt = (z >> g.b) & 1;
    r ^= xa & zt & (xt ^ za ^ 1);
    x ^= xa << g.b; z ^= zt << g.a;
  }
  return mk(x, z, r);
}
static uint64_t apply(uint64_t T, gate g) {
  for (int i = 0; i < 2 * n; i++) T = setrow(T, i, conj_row(row(T, i), g));
  return T;
}
/* image under T of +X^x Z^z (clifford.cu:82-95), tracking the phase as a power of i */
static uint32_t image(uint64_t T, uint32_t x, uint32_t z) {
  int k = __builtin_popcount(x & z);
  uint32_t ax = 0, az = 0;
  for (int q = 0; q < 2 * n; q++) {
    const int on = q < n ? (x >> q) & 1 : (z >> (q - n)) & 1;
    if (!on) continue;
    const uint32_t w = row(T, q), bx = RX(w), bz = RZ(w);
    k += 2 * (int)RR(w) + __builtin_popcount(bx & bz) + 2 * __builtin_popcount(az & bx);
    ax ^= bx; az ^= bz;
  }
  return mk(ax, az, (uint32_t)(((k - __builtin_popcount(ax & az)) & 3) >> 1));
}
static uint64_t compose(uint64_t A, uint64_t B) {  /* A first, then B */
  uint64_t C = 0;
  for (int i = 0; i < 2 * n; i++) {
    const uint32_t w = row(A, i);
    C = setrow(C, i, image(B, RX(w), RZ(w)) ^ (RR(w) << (2 * n)));
  }
  return C;
}
static uint64_t inverse(uint64_t C) {             /* clifford.cu:104-121 */
  const int m = 2 * n;
  uint64_t D = 0;
  for (int i = 0; i < m; i++) {
    uint32_t v = 0;
    const int wi = (i + n) % m;
    for (int j = 0; j < m; j++) {
      const uint32_t sr = row(C, (j + n) % m), bits = RX(sr) | (RZ(sr) << n);
      v |= ((bits >> wi) & 1) << j;
    }
    const uint32_t x = v & ((1u << n) - 1), z = v >> n;
    D = setrow(D, i, mk(x, z, RR(image(C, x, z))));
  }
  return D;
}

/* the table: open addressing, key 0 = empty (clifford.cu:125-146) */
static uint64_t *keys, mask;
static uint8_t *dist;
static uint64_t hmix(uint64_t h) {
  h ^= h >> 33; h *= 0xff51afd7ed558ccdULL; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ULL; h ^= h >> 33;
  return h;
}
static int find(uint64_t k) {
  for (uint64_t s = hmix(k) & mask;; s = (s + 1) & mask) {
    if (keys[s] == k) return dist[s];
    if (!keys[s]) return -1;
  }
}
static int insert(uint64_t k, uint8_t d) {
  for (uint64_t s = hmix(k) & mask;; s = (s + 1) & mask) {
    uint64_t exp = 0;
    if (__atomic_compare_exchange_n(&keys[s], &exp, k, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) { dist[s] = d; return 1; }
    if (exp == k) return 0;
  }
}

static gate G[32];
static int ng;
static gate inv_gate(gate g) { if (g.k == GS) g.k = GSDG; else if (g.k == GSDG) g.k = GS; return g; }

typedef struct { uint64_t K, Kinv; int qp, neg; } cand;
static int candcmp(const void *a, const void *b) {
  const cand *x = a, *y = b;
  if (x->K != y->K) return x->K < y->K ? -1 : 1;
  return x->qp - y->qp;
}
static int u64cmp(const void *a, const void *b) {
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}
static uint64_t flipped_inv(cand c, int dagger) { gate g = {dagger ? GSDG : GS, c.qp, 0}; return apply(c.Kinv, g); }

static int parse_gate(FILE *f, gate *g) {
  char nm[16];
  if (fscanf(f, "%15s", nm) != 1) return -1;
  g->b = 0;
  if (!strcmp(nm, "h")) g->k = GH; else if (!strcmp(nm, "s")) g->k = GS; else if (!strcmp(nm, "sdg")) g->k = GSDG;
  else if (!strcmp(nm, "x")) g->k = GX; else if (!strcmp(nm, "z")) g->k = GZ; else if (!strcmp(nm, "y")) g->k = GY;
  else if (!strcmp(nm, "cx")) g->k = GCX;
  else { fprintf(stderr, "unknown Clifford gate %s\n", nm); exit(2); }
  if (fscanf(f, "%d", &g->a) != 1) return -1;
  if (g->k == GCX && fscanf(f, "%d", &g->b) != 1) return -1;
  return 0;
}
static const char *gname(int k) { static const char *nm[] = {"h", "s", "sdg", "x", "z", "cx", "y"}; return nm[k]; }

/* the table of n qubits: BFS from the identity (clifford.cu:247-276), then the placement candidates per qubit
 * ordered by (K, q') */
static int table_n;
static long cap;
static cand *cands[3];
static long ncand[3];
static int build_table(void) {
  rb = 2 * n + 1;
  ng = 0;
  for (int q = 0; q < n; q++) for (int k = GH; k <= GZ; k++) { gate g = {k, q, 0}; G[ng++] = g; }
  for (int a = 0; a < n; a++) for (int b = 0; b < n; b++) if (a != b) { gate g = {GCX, a, b}; G[ng++] = g; }

  /* 1. BFS from the identity (clifford.cu:247-276) */
  const long order = n == 1 ? 24 : n == 2 ? 11520 : 92897280;
  int lg = 4;
  while ((1L << lg) < order * 4 / 3) lg++;
  cap = 1L << lg;
  mask = (uint64_t)cap - 1;
  free(keys); free(dist);
  keys = calloc(cap, 8); dist = calloc(cap, 1);
  uint64_t *fa = malloc(8 * (order / 2 + 1024)), *fb = malloc(8 * (order / 2 + 1024));
  long nf = 1, total = 1;
  fa[0] = identity();
  keys[hmix(fa[0]) & mask] = fa[0];
  for (int d = 1; nf; d++) {
    long nn = 0;
#pragma omp parallel for schedule(dynamic, 4096)
    for (long i = 0; i < nf; i++)
      for (int j = 0; j < ng; j++) {
        const uint64_t c = apply(fa[i], G[j]);
        if (insert(c, (uint8_t)d)) { const long p = __atomic_fetch_add(&nn, 1, __ATOMIC_RELAXED); fb[p] = c; }
      }
    nf = nn; total += nf;
    if (nf) fprintf(stderr, "  clifford gates %d: %ld\n", d, nf);
    uint64_t *tmp = fa; fa = fb; fb = tmp;
  }
  free(fa); free(fb);
  fprintf(stderr, "clifford table: %ld elements (group order %ld), 0.0 s\n", total, order);
  if (total != order) { fprintf(stderr, "group order mismatch\n"); return 1; }

  for (int q = 0; q < n; q++) {
    long m = 0, mcap = 1024;
    free(cands[q]);
    cands[q] = malloc(sizeof(cand) * mcap);
    for (long s = 0; s < cap; s++) {
      const uint64_t K = keys[s];
      if (!K) continue;
      for (int qp = 0; qp < n; qp++) {
        const uint32_t w = row(K, n + qp);
        if (RX(w) == 0 && RZ(w) == (1u << q)) {
          if (m == mcap) { mcap *= 2; cands[q] = realloc(cands[q], sizeof(cand) * mcap); }
          cand c = {K, inverse(K), qp, (int)RR(w)};
          cands[q][m++] = c;
        }
      }
    }
    qsort(cands[q], m, sizeof(cand), candcmp);
    ncand[q] = m;
  }
  table_n = n;
  return 0;
}

static int run_job(const char *path, int beam, int dist_only) {
  FILE *f = fopen(path, "r");
  int t = 0, bad = !f;
  if (!bad && fscanf(f, "%d %d", &n, &t) != 2) bad = 1;
  if (bad || t < 0 || t > 4096) { if (f) fclose(f); fprintf(stderr, "bad job file\n"); return 2; }
  int *tq = calloc(t + 1, sizeof(int)), *td = calloc(t + 1, sizeof(int));
  for (int i = 0; !bad && i < t; i++) if (fscanf(f, "%d %d", &tq[i], &td[i]) != 2) bad = 1;
  gate **seg = calloc(t + 1, sizeof(gate *));
  int *segn = calloc(t + 1, sizeof(int));
  for (int j = 0; !bad && j <= t; j++) {
    if (fscanf(f, "%d", &segn[j]) != 1 || segn[j] < 0) { bad = 1; break; }
    seg[j] = calloc(segn[j] + 1, sizeof(gate));
    for (int i = 0; i < segn[j]; i++) if (parse_gate(f, &seg[j][i])) { bad = 1; break; }
  }
  if (f) fclose(f);
  if (bad || n < 1 || n > 3) { fprintf(stderr, "bad job file\n"); return 2; }
  if (n != table_n && build_table()) return 4;
  uint64_t *D = malloc(8 * (t + 1));
  for (int j = 0; j <= t; j++) { uint64_t X = identity(); for (int i = 0; i < segn[j]; i++) X = apply(X, seg[j][i]); D[j] = X; }
  if (dist_only) {   /* one line per segment: its minimal gate count */
    for (int j = 0; j <= t; j++) printf("%d\n", find(D[j]));
    return 0;
  }

  /* 2. beam search over the placements (clifford.cu:281-330) */
  int **parent = calloc((size_t)t + 1, sizeof(int *)), **flips = calloc((size_t)t + 1, sizeof(int *));
  cand **chosen = calloc((size_t)t + 1, sizeof(cand *));
  uint64_t Kprev[256];
  int bcost[256], nb = 1;
  bcost[0] = 0; Kprev[0] = 0;
  for (int j = 0; j < t; j++) {
    const cand *C = cands[tq[j]];
    const long nc = ncand[tq[j]], tot = (long)nb * nc * 2;
    /* the reference sorts (cost << 40 | b << 32 | c2) and keeps the first B: by cost, then b, then c2 */
    uint64_t *packed = malloc(8 * tot);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < tot; i++) {
      const int b = (int)(i / (nc * 2));
      const long c2 = i % (nc * 2), c = c2 >> 1;
      const uint64_t left = j == 0 ? D[j] : compose(Kprev[b], D[j]);
      const uint64_t kinv = (c2 & 1) ? flipped_inv(C[c], td[j] ^ C[c].neg) : C[c].Kinv;
      const int d = find(compose(left, kinv));
      packed[i] = ((uint64_t)(bcost[b] + (d < 0 ? 999 : d)) << 40) | ((uint64_t)b << 32) | (uint64_t)c2;
    }
    qsort(packed, tot, 8, u64cmp);
    const int keep = (int)(beam < tot ? beam : tot);
    parent[j] = malloc(sizeof(int) * keep); flips[j] = malloc(sizeof(int) * keep); chosen[j] = malloc(sizeof(cand) * keep);
    uint64_t nk[256];
    int ncost[256];
    for (int i = 0; i < keep; i++) {
      const int b = (int)((packed[i] >> 32) & 0xff);
      const long c2 = (long)(packed[i] & 0xffffffffULL);
      parent[j][i] = b; chosen[j][i] = C[c2 >> 1]; flips[j][i] = (int)(c2 & 1);
      nk[i] = C[c2 >> 1].K; ncost[i] = (int)(packed[i] >> 40);
    }
    free(packed);
    memcpy(Kprev, nk, 8 * keep); memcpy(bcost, ncost, sizeof(int) * keep);
    nb = keep;
    fprintf(stderr, "  T gate %d: %ld placements x beam, best partial %d\n", j + 1, nc, ncost[0]);
  }
  int best = 0, bestv = 1 << 30;
  for (int b = 0; b < nb; b++) {
    const int d = find(t ? compose(Kprev[b], D[t]) : D[t]);
    const int v = bcost[b] + (d < 0 ? 999 : d);
    if (v < bestv) { bestv = v; best = b; }
  }
  cand *K = calloc(t + 1, sizeof(cand));
  int *flip = calloc(t + 1, sizeof(int)), *dag = calloc(t + 1, sizeof(int));
  for (int j = t - 1, b = best; j >= 0; j--) { K[j] = chosen[j][b]; flip[j] = flips[j][b]; b = parent[j][b]; }
  for (int j = 0; j < t; j++) {
    const int d0 = td[j] ^ K[j].neg;
    if (flip[j]) K[j].Kinv = flipped_inv(K[j], d0);
    dag[j] = d0 ^ flip[j];
  }

  /* 3. segments K_j^-1 D_j K_{j-1}, each read back as an optimal word (clifford.cu:343-372) */
  gate **out = calloc(t + 1, sizeof(gate *));
  int *outn = calloc(t + 1, sizeof(int)), total_c = 0, orig = 0;
  for (int j = 0; j <= t; j++) {
    uint64_t X = j > 0 ? compose(K[j - 1].K, D[j]) : D[j];
    if (j < t) X = compose(X, K[j].Kinv);
    int d = find(X);
    if (d < 0) { fprintf(stderr, "segment not in the table\n"); return 4; }
    total_c += d;
    out[j] = calloc(d + 1, sizeof(gate));
    outn[j] = d;
    for (int pos = d - 1; pos >= 0; pos--) {
      int g = 0;
      uint64_t pre = 0;
      for (; g < ng; g++) { pre = apply(X, inv_gate(G[g])); if (find(pre) == pos) break; }
      if (g == ng) { fprintf(stderr, "path reconstruction failed\n"); return 4; }
      out[j][pos] = G[g];
      X = pre;
    }
  }
  for (int j = 0; j <= t; j++) orig += segn[j];
  printf("{\"clifford_gates\": %d, \"clifford_gates_before\": %d, \"t_gates\": %d, \"seconds\": 0.00}\n", total_c, orig, t);
  for (int j = 0; j <= t; j++) {
    for (int i = 0; i < outn[j]; i++) {
      if (out[j][i].k == GCX) printf("cx %d %d\n", out[j][i].a, out[j][i].b);
      else printf("%s %d\n", gname(out[j][i].k), out[j][i].a);
    }
    if (j < t) printf("%s %d\n", dag[j] ? "tdg" : "t", K[j].qp);
  }
  return 0;
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: cliffopt JOB [--beam B]\n"); return 3; }
  int beam = 16, dist_only = 0, njobs = 0;
  const char *jobs[256];
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--beam") && i + 1 < argc) { beam = atoi(argv[++i]); beam = beam < 1 ? 1 : beam > 255 ? 255 : beam; }
    else if (!strcmp(argv[i], "--dist-only")) dist_only = 1;
    else if (njobs < 256) jobs[njobs++] = argv[i];
  }
  /* several jobs share one table per qubit count: each output starts with a "### JOB" line */
  int rc = 0;
  for (int i = 0; i < njobs; i++) {
    if (njobs > 1) { printf("### %s\n", jobs[i]); fflush(stdout); fprintf(stderr, "### %s\n", jobs[i]); }
    rc = run_job(jobs[i], beam, dist_only);
    fflush(stdout);
    if (njobs > 1) printf("### rc %d\n", rc);
  }
  return rc;
}
