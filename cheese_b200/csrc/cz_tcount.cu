// sm_100a kernels and host loop of the T-count search (the reference's src/tcount.cu).
//
// Reference semantics: a level peels every rotation p = 1..P-1 off every node (children in parent-major order,
// tcount.cu:201-207), labels each child by its coset key, keeps one child per coset (the smallest index, exact
// comparison, :232-247, 348-363) and, while building the table, drops cosets already present at a lower level
// (:258-276, 368-390). The search peels rotations off U level by level and looks every node up in the table; the
// first level with a hit gives the optimum, the node with the smallest table level wins (:497-529).
//
// B200 design: one 256-thread CTA per parent holds the parent's 64 x 64 matrix (x and y limbs, int32) in shared
// memory and derives all 63 children from it (the reference replays the whole path for every child); the coset
// key is a sum over columns of a hash of the sign-normalised column (invariant under signed column permutations,
// i.e. right Cliffords) computed with per-column shared-memory atomics; equality of cosets is the exact multiset
// comparison of sign-normalised columns. Dedupe reuses the radix sort of the gate-count search. Tables stay
// resident in HBM for the engine's lifetime.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>

#include "cz_sort.cuh"
#include "cz_tcount.h"

namespace cz {

namespace {

constexpr int TC_T = 256;        // threads per CTA
constexpr int MAXP = 64;         // 4^n, n <= 3
constexpr int MAXT = 32;         // deepest peel sequence
constexpr unsigned FULLM = 0xffffffffu;
constexpr uint32_t TC_CACHE_MAGIC = 0x43545a43u;   // "CZTC": the table file's keys use this build's coset hash
constexpr uint32_t TC_KEY_VERSION = 1;

struct TDev {
  int n, P, lp, G;               // lp = log2 P
  const int *bx, *by;            // base matrix (U's channel, or the identity)
  int be;
  const int8_t *tr, *ts;         // (P - 1) x P partner rows and signs
};
struct THist {
  const uint32_t *par[MAXT + 1];
  const uint8_t *gat[MAXT + 1];
};

__device__ __forceinline__ uint64_t fmix(uint64_t h) {
  h ^= h >> 33; h *= 0xff51afd7ed558ccdULL; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ULL; h ^= h >> 33;
  return h;
}

// shared memory: A and B matrices (x, y limbs) + per-column / per-row arrays
struct TSm {
  int *ax, *ay, *bx, *by;
  int *fa, *fb, *sa, *sb;                     // per column: first nonzero row, sign
  int *gm;                                    // per column: scratch of the exact comparison
  unsigned long long *a1, *a2, *b1, *b2;      // per column: hash partial sums, then column hashes
  unsigned long long *w1, *w2;                // per row weights
  unsigned long long *red;                    // 4 words
  int *misc;                                  // 8 ints
  uint8_t *seq;                               // MAXT + 1
};
__host__ __device__ inline size_t tsm_bytes(int P) {
  return (size_t)4 * P * P * 4 + (size_t)5 * MAXP * 4 + (size_t)6 * MAXP * 8 + 4 * 8 + 8 * 4 + MAXT + 8;
}
__device__ TSm tsm_carve(int P) {
  extern __shared__ unsigned long long smraw[];
  TSm s;
  unsigned long long *q = smraw;
  s.a1 = q; q += MAXP; s.a2 = q; q += MAXP; s.b1 = q; q += MAXP; s.b2 = q; q += MAXP;
  s.w1 = q; q += MAXP; s.w2 = q; q += MAXP; s.red = q; q += 4;
  int *p = (int *)q;
  s.ax = p; p += P * P; s.ay = p; p += P * P; s.bx = p; p += P * P; s.by = p; p += P * P;
  s.fa = p; p += MAXP; s.fb = p; p += MAXP; s.sa = p; p += MAXP; s.sb = p; p += MAXP; s.gm = p; p += MAXP;
  s.misc = p; p += 8;
  s.seq = (uint8_t *)p;
  for (int i = threadIdx.x; i < MAXP; i += blockDim.x) {
    s.w1[i] = fmix(0x243f6a8885a308d3ULL + 0x9e3779b97f4a7c15ULL * (uint64_t)(i + 1)) | 1;
    s.w2[i] = fmix(0x13198a2e03707344ULL + 0xc2b2ae3d27d4eb4fULL * (uint64_t)(i + 1)) | 1;
  }
  __syncthreads();
  return s;
}

// M <- base
__device__ int blk_load(int *mx, int *my, const TDev &sp) {
  for (int i = threadIdx.x; i < sp.P * sp.P; i += blockDim.x) { mx[i] = sp.bx[i]; my[i] = sp.by[i]; }
  __syncthreads();
  return sp.be;
}

// (ox, oy) <- R(P_p)^-1 (ix, iy), normalised; may run in place. Returns the new exponent (block-uniform).
__device__ int blk_peel(const int *ix, const int *iy, int ie, int *ox, int *oy, int p, const TDev &sp, int *ovf) {
  const int P = sp.P, PP = P * P;
  constexpr int PER = MAXP * MAXP / TC_T;
  int vx[PER], vy[PER];
  bool bad = false;
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const int i = threadIdx.x + TC_T * j;
    if (i >= PP) continue;
    const int a = i >> sp.lp, c = i & (P - 1);
    const int r = sp.tr[(p - 1) * P + a], s = sp.ts[(p - 1) * P + a];
    int64_t nx, ny;
    if (r < 0) { nx = 2 * (int64_t)iy[i]; ny = ix[i]; }                 // times sqrt2: (x + y s) s = 2y + x s
    else { nx = ix[i] - s * (int64_t)ix[r * P + c]; ny = iy[i] - s * (int64_t)iy[r * P + c]; }
    if (nx > INT32_MAX || nx < INT32_MIN || ny > INT32_MAX || ny < INT32_MIN) bad = true;
    vx[j] = (int)nx; vy[j] = (int)ny;
  }
  if (bad) atomicOr(ovf, 1);
  __syncthreads();                                                      // in place: everyone has read
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const int i = threadIdx.x + TC_T * j;
    if (i < PP) { ox[i] = vx[j]; oy[i] = vy[j]; }
  }
  int e = ie + 1;
  for (;;) {                                                            // (x + y s) / s = y + (x / 2) s while all x even
    bool even = e > 0;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int i = threadIdx.x + TC_T * j;
      if (i < PP && (ox[i] & 1)) even = false;
    }
    if (!__syncthreads_and(even)) break;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int i = threadIdx.x + TC_T * j;
      if (i < PP) { const int x = ox[i]; ox[i] = oy[i]; oy[i] = x >> 1; }
    }
    e--;
  }
  return e;
}

// replay: base then the peels of seq[0 .. len)
__device__ int blk_build(int *mx, int *my, const TDev &sp, const uint8_t *seq, int len, int *ovf) {
  int e = blk_load(mx, my, sp);
  for (int i = 0; i < len; i++) e = blk_peel(mx, my, e, mx, my, seq[i], sp, ovf);
  return e;
}
// the path of node i at level t of tree H into seq (block-uniform, in shared memory)
__device__ void blk_path(const THist &H, int t, uint32_t i, uint8_t *seq) {
  if (threadIdx.x == 0)
    for (int l = t; l >= 1; l--) { seq[l - 1] = H.gat[l][i]; i = H.par[l][i]; }
  __syncthreads();
}

// per column: first nonzero row and sign; column hashes of the sign-normalised columns into h1/h2; the coset key
// (the column hashes summed, then mixed with the exponent) into k1/k2 (block-uniform)
__device__ void blk_colkey(const int *mx, const int *my, int e, int P, int *first, int *sgn, unsigned long long *h1,
                           unsigned long long *h2, const TSm &s, uint64_t &k1, uint64_t &k2) {
  const int tid = threadIdx.x;
  const int c = tid & (P - 1), q = tid / P, stride = TC_T / P;
  if (tid < P) { first[tid] = P; h1[tid] = 0; h2[tid] = 0; }
  __syncthreads();
  int myf = P;
  for (int a = q; a < P; a += stride)
    if (mx[a * P + c] | my[a * P + c]) { myf = a; break; }
  if (myf < P) atomicMin(&first[c], myf);
  __syncthreads();
  const int fr = first[c];
  int sg = 1;
  if (fr < P) { const int x = mx[fr * P + c], y = my[fr * P + c]; sg = (x > 0 || (x == 0 && y > 0)) ? 1 : -1; }
  uint64_t p1 = 0, p2 = 0;
  for (int a = q; a < P; a += stride) {
    const uint64_t v = (uint64_t)(uint32_t)(sg * mx[a * P + c]) | ((uint64_t)(uint32_t)(sg * my[a * P + c]) << 32);
    p1 += v * s.w1[a];
    p2 += v * s.w2[a];
  }
  atomicAdd(&h1[c], (unsigned long long)p1);
  atomicAdd(&h2[c], (unsigned long long)p2);
  __syncthreads();
  uint64_t t1 = 0, t2 = 0;
  if (tid < P) {
    sgn[tid] = sg;
    t1 = fmix(h1[tid] + 0x632be59bd9b4e019ULL);
    t2 = fmix(h2[tid] ^ 0x8cb92ba72f3d8dd7ULL);
    h1[tid] = t1; h2[tid] = t2;
  }
  if (tid < 64) {
#pragma unroll
    for (int m = 16; m; m >>= 1) { t1 += __shfl_xor_sync(FULLM, t1, m); t2 += __shfl_xor_sync(FULLM, t2, m); }
    if ((tid & 31) == 0) { s.red[2 * (tid >> 5)] = t1; s.red[2 * (tid >> 5) + 1] = t2; }
  }
  __syncthreads();
  const uint64_t sum1 = s.red[0] + s.red[2], sum2 = s.red[1] + s.red[3];
  k1 = fmix(sum1 + (uint64_t)(int64_t)e * 0xa0761d6478bd642fULL);
  k2 = fmix(sum2 ^ ((uint64_t)(int64_t)e * 0xe7037ed1a0b428dbULL + 0x5555ULL));
  __syncthreads();
}

// exact multiset comparison by counting, for the rare case of two different columns with equal hashes
__device__ bool blk_same_counted(const TSm &s, int P) {
  const int tid = threadIdx.x;
  bool eq = true;
  if (tid < P) {
    const int c = tid;
    auto col_eq = [&](const int *xx, const int *yy, const int *sg, int cx, const int *zx, const int *zy, const int *sz,
                      int cz) {
      for (int a = 0; a < P; a++)
        if (sg[cx] * xx[a * P + cx] != sz[cz] * zx[a * P + cz] || sg[cx] * yy[a * P + cx] != sz[cz] * zy[a * P + cz])
          return false;
      return true;
    };
    int na = 0, nb = 0;
    for (int d = 0; d < P; d++) {
      if (s.a1[d] == s.a1[c] && s.a2[d] == s.a2[c] && col_eq(s.ax, s.ay, s.sa, d, s.ax, s.ay, s.sa, c)) na++;
      if (s.b1[d] == s.a1[c] && s.b2[d] == s.a2[c] && col_eq(s.bx, s.by, s.sb, d, s.ax, s.ay, s.sa, c)) nb++;
    }
    eq = na == nb;
  }
  return __syncthreads_and(eq);
}

// exact coset equality of A and B (both keyed by blk_colkey): same exponent and the same multiset of
// sign-normalised columns. Per column: the number of A and of B columns with its hash (equal counts for every
// hash), its group's first A column, first B column and, for B's own columns, first B column; then, in lockstep
// over the rows, every A column equals its group's first A column and first B column, and every B column equals its
// group's first B column. The per-column searches keep no data-dependent inner loop, so a warp never serialises.
// Only when the hash counts agree but a group holds different columns is the counting comparison run.
// (fa and fb, the first nonzero rows, are not needed after the keys: they hold the group indices here.)
__device__ bool blk_same(const TSm &s, int ea, int eb, int P) {
  if (ea != eb) return false;
  const int tid = threadIdx.x;
  bool ok = true;
  if (tid < P) {
    const int c = tid;
    const unsigned long long ha1 = s.a1[c], ha2 = s.a2[c], hb1 = s.b1[c], hb2 = s.b2[c];
    int ka = 0, kb = 0, ra = P, rb = P, rbb = P;
    for (int d = 0; d < P; d++) {
      const bool ia = s.a1[d] == ha1 && s.a2[d] == ha2;
      const bool ib = s.b1[d] == ha1 && s.b2[d] == ha2;
      const bool bb = s.b1[d] == hb1 && s.b2[d] == hb2;
      ka += ia; kb += ib;
      if (ia && d < ra) ra = d;
      if (ib && d < rb) rb = d;
      if (bb && d < rbb) rbb = d;
    }
    ok = ka == kb && rb < P;
    s.fa[c] = ra; s.fb[c] = rbb; s.gm[c] = rb < P ? rb : 0;
  }
  if (!__syncthreads_and(ok)) return false;       // the hash multisets differ, so the column multisets do
  const int c = tid & (P - 1), q = tid / P, stride = TC_T / P;
  const int ra = s.fa[c], rbb = s.fb[c], rb = s.gm[c];
  const int sc = s.sa[c], sra = s.sa[ra], srb = s.sb[rb], sbc = s.sb[c], srbb = s.sb[rbb];
  for (int a = q; a < P && ok; a += stride) {
    const int x = sc * s.ax[a * P + c], y = sc * s.ay[a * P + c];
    if (x != sra * s.ax[a * P + ra] || y != sra * s.ay[a * P + ra]) ok = false;
    if (x != srb * s.bx[a * P + rb] || y != srb * s.by[a * P + rb]) ok = false;
    if (sbc * s.bx[a * P + c] != srbb * s.bx[a * P + rbb] || sbc * s.by[a * P + c] != srbb * s.by[a * P + rbb]) ok = false;
  }
  if (__syncthreads_and(ok)) return true;
  return blk_same_counted(s, P);                  // a hash group holds different columns: count exact matches
}

// ---------------- kernels ----------------
// keys of the nodes [0, n) of level t of tree H (the root when t = 0)
__global__ void __launch_bounds__(TC_T) k_tc_keys(const TDev sp, const THist H, int t, long long n, uint64_t *k1o,
                                                  uint64_t *k2o, int *ovf) {
  const TSm s = tsm_carve(sp.P);
  for (long long i = blockIdx.x; i < n; i += gridDim.x) {
    blk_path(H, t, (uint32_t)i, s.seq);
    const int e = blk_build(s.ax, s.ay, sp, s.seq, t, ovf);
    uint64_t k1, k2;
    blk_colkey(s.ax, s.ay, e, sp.P, s.fa, s.sa, s.a1, s.a2, s, k1, k2);
    if (threadIdx.x == 0) { k1o[i] = k1; k2o[i] = k2; }
  }
}

// child o = parent i * G + (p - 1): parent i of level tp, peeled by rotation p. With pmx, each parent's matrix and
// exponent are kept (2 P^2 ints at pmx + 2 P^2 i, pe[i]) so the exact dedupe rebuilds a child with one peel.
__global__ void __launch_bounds__(TC_T, 2) k_tc_children(const TDev sp, const THist H, int tp, long long m, uint64_t *k1o,
                                                      uint64_t *k2o, int *ovf, int *pmx, int *pe) {
  const TSm s = tsm_carve(sp.P);
  const int G = sp.G, PP = sp.P * sp.P;
  for (long long i = blockIdx.x; i < m; i += gridDim.x) {
    blk_path(H, tp, (uint32_t)i, s.seq);
    const int e = blk_build(s.ax, s.ay, sp, s.seq, tp, ovf);
    if (pmx) {
      int *dst = pmx + (size_t)i * 2 * PP;
      for (int x = threadIdx.x; x < PP; x += blockDim.x) { dst[x] = s.ax[x]; dst[PP + x] = s.ay[x]; }
      if (threadIdx.x == 0) pe[i] = e;
    }
    for (int p = 1; p <= G; p++) {
      const int ec = blk_peel(s.ax, s.ay, e, s.bx, s.by, p, sp, ovf);
      uint64_t k1, k2;
      blk_colkey(s.bx, s.by, ec, sp.P, s.fb, s.sb, s.b1, s.b2, s, k1, k2);
      if (threadIdx.x == 0) { k1o[i * G + p - 1] = k1; k2o[i * G + p - 1] = k2; }
    }
  }
}

struct TcStats { unsigned long long n_work, n_kept; };

__global__ void k_tc_runs(const uint64_t *keys, const uint32_t *vals, size_t n, uint64_t *kept, uint2 *work,
                          TcStats *st) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t hk = (uint32_t)(keys[i] >> 32);
    if (i > 0 && (uint32_t)(keys[i - 1] >> 32) == hk) continue;
    size_t j = i + 1;
    while (j < n && (uint32_t)(keys[j] >> 32) == hk) j++;
    if (j == i + 1) kept[atomicAdd(&st->n_kept, 1ULL)] = vals[i];
    else work[atomicAdd(&st->n_work, 1ULL)] = make_uint2((unsigned)i, (unsigned)(j - i));
  }
}

// keys sorted by all 64 bits of h1 (stable: index order within a run): the first member of every run is kept, every
// other member is listed for a check against its run's first member
__global__ void k_tc_split(const uint64_t *keys, const uint32_t *vals, size_t n, uint64_t *kept, uint32_t *check,
                           TcStats *st) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (i == 0 || keys[i - 1] != keys[i]) kept[atomicAdd(&st->n_kept, 1ULL)] = vals[i];
    else check[atomicAdd(&st->n_work, 1ULL)] = (uint32_t)i;
  }
}
// one CTA per listed member: is it exactly the coset of its run's first member (equal h2 and the same multiset of
// columns)? Children are rebuilt from their kept parents with one peel. A member that is not counts as unresolved:
// the level is then deduped by the sequential resolver instead, which handles any mix of cosets in a run.
__global__ void __launch_bounds__(TC_T) k_tc_dupcheck(const TDev sp, const uint64_t *keys, const uint32_t *vals,
                                                      size_t n, const uint32_t *check, const uint64_t *h2,
                                                      const int *pmx, const int *pe, TcStats *st,
                                                      unsigned long long *unresolved, int *ovf) {
  const TSm s = tsm_carve(sp.P);
  const int G = sp.G, PP = sp.P * sp.P;
  const unsigned long long nw = st->n_work;
  auto child = [&](uint32_t v, int *mx, int *my) {
    const int *src = pmx + (size_t)(v / G) * 2 * PP;
    for (int x = threadIdx.x; x < PP; x += blockDim.x) { mx[x] = src[x]; my[x] = src[PP + x]; }
    __syncthreads();
    return blk_peel(mx, my, pe[v / G], mx, my, (int)(v % G) + 1, sp, ovf);
  };
  for (unsigned long long w = blockIdx.x; w < nw; w += gridDim.x) {
    const uint32_t i = check[w];
    const uint64_t key = keys[i];
    size_t lo = 0, hi = i;                       // the run's first position: lower bound of the key
    while (lo < hi) { const size_t mid = (lo + hi) / 2; if (keys[mid] < key) lo = mid + 1; else hi = mid; }
    const uint32_t v0 = vals[lo], vi = vals[i];
    bool same = h2[v0] == h2[vi];
    if (same) {
      const int ea = child(v0, s.ax, s.ay);
      uint64_t k1, k2;
      blk_colkey(s.ax, s.ay, ea, sp.P, s.fa, s.sa, s.a1, s.a2, s, k1, k2);
      const int eb = child(vi, s.bx, s.by);
      blk_colkey(s.bx, s.by, eb, sp.P, s.fb, s.sb, s.b1, s.b2, s, k1, k2);
      same = blk_same(s, ea, eb, sp.P);
    }
    if (!same && threadIdx.x == 0) atomicAdd(unresolved, 1ULL);
    __syncthreads();
  }
}

// one CTA per run of equal key prefixes: order by (h1, h2, index), keep the first member of every exact coset
__global__ void __launch_bounds__(TC_T) k_tc_resolve(const TDev sp, const THist H, int tp, const uint2 *work,
                                                     const uint32_t *vals, const uint64_t *h1, const uint64_t *h2,
                                                     uint32_t *tmp, uint64_t *kept, TcStats *st, int *ovf,
                                                     const int *pmx, const int *pe) {
  const TSm s = tsm_carve(sp.P);
  const int G = sp.G, PP = sp.P * sp.P;
  // child v of level tp + 1 into (mx, my): its parent's kept matrix peeled once, or rebuilt from the base
  auto child = [&](uint32_t v, int *mx, int *my) {
    if (pmx) {
      const int *src = pmx + (size_t)(v / G) * 2 * PP;
      for (int x = threadIdx.x; x < PP; x += blockDim.x) { mx[x] = src[x]; my[x] = src[PP + x]; }
      __syncthreads();
      return blk_peel(mx, my, pe[v / G], mx, my, (int)(v % G) + 1, sp, ovf);
    }
    blk_path(H, tp, v / G, s.seq);
    if (threadIdx.x == 0) s.seq[tp] = (uint8_t)(v % G + 1);
    __syncthreads();
    return blk_build(mx, my, sp, s.seq, tp + 1, ovf);
  };
  const unsigned long long nw = st->n_work;
  for (unsigned long long w = blockIdx.x; w < nw; w += gridDim.x) {
    const uint2 wk = work[w];
    const unsigned start = wk.x, len = wk.y;
    for (unsigned a = threadIdx.x; a < len; a += blockDim.x) {       // rank of each member in (h1, h2, index)
      const uint32_t va = vals[start + a];
      unsigned rank = 0;
      for (unsigned b = 0; b < len; b++) {
        const uint32_t vb = vals[start + b];
        rank += (h1[vb] < h1[va]) || (h1[vb] == h1[va] && (h2[vb] < h2[va] || (h2[vb] == h2[va] && vb < va)));
      }
      tmp[start + rank] = va;
    }
    __syncthreads();
    unsigned gstart = 0;
    int loaded = -1;                                                  // tmp position of the member held in A
    int ea = 0;
    for (unsigned i = 0; i < len; i++) {
      const uint32_t vi = tmp[start + i] & 0x7fffffffu;
      if (i > 0) {
        const uint32_t vp = tmp[start + i - 1] & 0x7fffffffu;
        if (h1[vp] != h1[vi] || h2[vp] != h2[vi]) gstart = i;
      }
      bool dup = false;
      bool built = false;
      int eb = 0;
      for (unsigned i2 = gstart; i2 < i && !dup; i2++) {
        const uint32_t t2 = tmp[start + i2];
        if (!(t2 & 0x80000000u)) continue;
        if (!built) {                                                 // the candidate into B
          eb = child(vi & 0x7fffffffu, s.bx, s.by);
          uint64_t k1, k2;
          blk_colkey(s.bx, s.by, eb, sp.P, s.fb, s.sb, s.b1, s.b2, s, k1, k2);
          built = true;
        }
        if (loaded != (int)i2) {                                      // the kept member into A
          const uint32_t v2 = t2 & 0x7fffffffu;
          ea = child(v2, s.ax, s.ay);
          uint64_t k1, k2;
          blk_colkey(s.ax, s.ay, ea, sp.P, s.fa, s.sa, s.a1, s.a2, s, k1, k2);
          loaded = (int)i2;
        }
        dup = blk_same(s, ea, eb, sp.P);
      }
      if (!dup && threadIdx.x == 0) {
        tmp[start + i] = vi | 0x80000000u;
        kept[atomicAdd(&st->n_kept, 1ULL)] = vi;
      }
      __syncthreads();
    }
  }
}

// kept child indices (sorted) -> the new level: parent, rotation, key
__global__ void k_tc_gather(const uint64_t *kidx, size_t nk, int G, const uint64_t *h1, const uint64_t *h2,
                            uint32_t *par, uint8_t *gat, uint64_t *f1, uint64_t *f2) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < nk; j += (size_t)gridDim.x * blockDim.x) {
    const uint64_t o = kidx[j];
    par[j] = (uint32_t)(o / (uint64_t)G);
    gat[j] = (uint8_t)(o % (uint64_t)G + 1);
    f1[j] = h1[o];
    f2[j] = h2[o];
  }
}

// node j of level t of (sq, Hq) against the table (st, Ht) with sorted keys S1/S2 and (idx, lvl): the entry of
// an exactly equal coset with level <= maxc, the smallest such level first; -1 if none
__global__ void __launch_bounds__(TC_T) k_tc_lookup(const TDev sq, const THist Hq, int t, const uint64_t *F1,
                                                    const uint64_t *F2, long long n, const TDev st, const THist Ht,
                                                    const uint64_t *S1, const uint64_t *S2, const uint32_t *Sidx,
                                                    const uint32_t *Slvl, long long nd, int maxc, long long *hit,
                                                    int *ovf) {
  const TSm s = tsm_carve(sq.P);
  for (long long j = blockIdx.x; j < n; j += gridDim.x) {
    const uint64_t f1 = F1[j], f2 = F2[j];
    long long lo = 0, hi = nd;                                        // first entry with S1 >= f1
    while (lo < hi) { const long long mid = (lo + hi) >> 1; if (S1[mid] < f1) lo = mid + 1; else hi = mid; }
    long long res = -1;
    int rl = 1 << 30;
    bool built = false;
    int ea = 0;
    for (long long x = lo; x < nd && S1[x] == f1; x++) {
      const int lvl = (int)Slvl[x];
      if (S2[x] != f2 || lvl > maxc || lvl >= rl) continue;
      if (!built) {
        blk_path(Hq, t, (uint32_t)j, s.seq);
        ea = blk_build(s.ax, s.ay, sq, s.seq, t, ovf);
        uint64_t k1, k2;
        blk_colkey(s.ax, s.ay, ea, sq.P, s.fa, s.sa, s.a1, s.a2, s, k1, k2);
        built = true;
      }
      blk_path(Ht, lvl, Sidx[x], s.seq);
      const int eb = blk_build(s.bx, s.by, st, s.seq, lvl, ovf);
      uint64_t k1, k2;
      blk_colkey(s.bx, s.by, eb, st.P, s.fb, s.sb, s.b1, s.b2, s, k1, k2);
      if (blk_same(s, ea, eb, sq.P)) { res = x; rl = lvl; }
    }
    if (threadIdx.x == 0) hit[j] = res;
    __syncthreads();
  }
}

__global__ void k_tc_seen_init(const uint64_t *f1, size_t n, uint64_t *keys, uint32_t *vals) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    keys[i] = f1[i];
    vals[i] = (uint32_t)i;
  }
}
__global__ void k_tc_seen_gather(const uint32_t *order, size_t n, const uint64_t *a1, const uint64_t *a2,
                                 const uint32_t *aidx, const uint32_t *alvl, uint64_t *s1, uint64_t *s2, uint32_t *sidx,
                                 uint32_t *slvl) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t o = order[i];
    s1[i] = a1[o]; s2[i] = a2[o]; sidx[i] = aidx[o]; slvl[i] = alvl[o];
  }
}

// ---------------- host ----------------
double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
struct TcCudaError : std::runtime_error { using std::runtime_error::runtime_error; };
void tck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();            // a failed allocation must not be reported again by the next launch check
    throw TcCudaError(std::string("CUDA error after ") + what + ": " + cudaGetErrorString(e));
  }
}
struct Buf {
  void *p = nullptr;
  size_t cap = 0;
  void ensure(size_t b) {
    if (b <= cap) return;
    if (p) tck(cudaFree(p), "free");
    size_t c = std::max(b, cap + cap / 2);
    c = (c + 255) & ~(size_t)255;
    tck(cudaMalloc(&p, c), "cudaMalloc");
    cap = c;
  }
  template <typename T> T *as() const { return (T *)p; }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

// a tree of peel sequences: level l holds (parent, rotation) per node; keys of the top level
struct Tree {
  std::vector<Buf> par = std::vector<Buf>(1), gat = std::vector<Buf>(1);   // level l at [l]; [0] unused (the root)
  std::vector<long long> n{1};
  Buf F1, F2;                      // keys of the top level
  int top() const { return (int)n.size() - 1; }
  THist hist() const {
    if (par.size() != n.size() || gat.size() != n.size()) throw std::logic_error("tree levels out of step");
    THist H{};
    for (int l = 1; l <= top() && l <= MAXT; l++) { H.par[l] = par[l].as<uint32_t>(); H.gat[l] = gat[l].as<uint8_t>(); }
    return H;
  }
  void release() { for (auto &b : par) b.release(); for (auto &b : gat) b.release(); F1.release(); F2.release(); }
};
struct Table {                     // the coset table: tree from the identity + every node's key, sorted
  Tree D;
  Buf S1, S2, Sidx, Slvl;
  long long ns = 0;
};

}  // namespace

class TcountContext {
 public:
  int dev;
  cudaStream_t s;
  int nsm = 148;
  std::map<std::pair<int, int>, Table *> tables;   // resident: (n, K)
  Buf bx, by, ix, iy, tr, ts, ovf, stats;
  Buf h1, h2, k0, k1, v0, v1, hist, part, work, tmp, kept, hits;
  Buf pmat, pexp;                                  // parents' matrices and exponents of the level being grown
  long long launches = 0;
  TcountContext(int d, void *stream) : dev(d), s((cudaStream_t)stream) {
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  ~TcountContext() {
    cudaSetDevice(dev);
    for (auto &kv : tables) { kv.second->D.release(); kv.second->S1.release(); kv.second->S2.release();
                              kv.second->Sidx.release(); kv.second->Slvl.release(); delete kv.second; }
    for (Buf *b : {&bx, &by, &ix, &iy, &tr, &ts, &ovf, &stats, &h1, &h2, &k0, &k1, &v0, &v1, &hist, &part, &work, &tmp,
                   &kept, &hits, &pmat, &pexp})
      b->release();
  }
  size_t trim() {                              // work buffers back to the device; resident tables stay
    size_t n = 0;
    for (Buf *b : {&bx, &by, &ix, &iy, &tr, &ts, &h1, &h2, &k0, &k1, &v0, &v1, &hist, &part, &work, &tmp, &kept, &hits,
                   &pmat, &pexp}) {
      n += b->cap;
      b->release();
    }
    return n;
  }
  size_t smem(int P) const { return tsm_bytes(P); }
  void check_ovf() {
    int v = 0;
    tck(cudaMemcpyAsync(&v, ovf.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
    tck(cudaStreamSynchronize(s), "sync");
    if (v) throw std::overflow_error("coefficient overflow (int32)");
  }
  unsigned grid(long long n) const { return (unsigned)std::max<long long>(1, std::min<long long>(n, (long long)nsm * 4)); }

  // keys of level t of T (root: t = 0) into T.F1/F2
  void level_keys(const TDev &sp, Tree &T, int t) {
    const long long n = T.n[t];
    T.F1.ensure(n * 8); T.F2.ensure(n * 8);
    k_tc_keys<<<grid(n), TC_T, smem(sp.P), s>>>(sp, T.hist(), t, n, T.F1.as<uint64_t>(), T.F2.as<uint64_t>(), ovf.as<int>());
    launches++;
    tck(cudaGetLastError(), "keys kernel");
  }

  // one more level of T (peels off sp's base); table: drop cosets already in tab. Returns the new nodes.
  long long grow(const TDev &sp, Tree &T, Table *tab, const std::function<void(const TcLevel &)> &cb) {
    const double t0 = now_s();
    const int t = T.top() + 1, tp = t - 1, G = sp.G;
    if (t > MAXT) throw std::runtime_error("peel sequence longer than 32");
    const long long m = T.n[tp], nc = m * G;
    if (nc >= (1LL << 32)) throw std::runtime_error("level too large for 32-bit child indices");
    h1.ensure(nc * 8); h2.ensure(nc * 8);
    // the parents' matrices, kept for the exact dedupe (up to 16 GB; beyond, children are rebuilt from the base)
    const size_t pm_bytes = (size_t)m * 2 * sp.P * sp.P * 4;
    int *pmx = nullptr, *pe = nullptr;
    if (pm_bytes <= ((size_t)16 << 30)) {
      pmat.ensure(pm_bytes + 16); pexp.ensure((size_t)m * 4 + 16);
      pmx = pmat.as<int>(); pe = pexp.as<int>();
    }
    k_tc_children<<<grid(m), TC_T, smem(sp.P), s>>>(sp, T.hist(), tp, m, h1.as<uint64_t>(), h2.as<uint64_t>(), ovf.as<int>(),
                                                    pmx, pe);
    launches++;
    tck(cudaGetLastError(), "children kernel");
    check_ovf();
    // dedupe. With the parents' matrices kept: sort by all 64 bits of h1, keep each run's first member, and check
    // every other member against it in parallel; only if some member is not an exact copy of its run's first (a
    // hash collision) is the level deduped by the sequential resolver below, which is also the path without kept
    // matrices: sort by the top 32 key bits, singletons kept, runs resolved exactly
    const size_t n = (size_t)nc;
    k0.ensure(n * 8); k1.ensure(n * 8); v0.ensure(n * 4); v1.ensure(n * 4);
    hist.ensure(sort_hist_words(n) * 4); part.ensure(scan_partials_words(sort_hist_words(n)) * 4);
    work.ensure(n * sizeof(uint2)); tmp.ensure(n * 4); kept.ensure(n * 8); stats.ensure(sizeof(TcStats) + 16);
    SortScratch sc{hist.as<uint32_t>(), part.as<uint32_t>(), hist.cap / 4, part.cap / 4};
    const unsigned gb = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)nsm * 16);
    TcStats hs{};
    bool resolved = false;
    if (pmx) {
      unsigned long long *unres = (unsigned long long *)(stats.as<TcStats>() + 1);
      k_tc_seen_init<<<gb, 256, 0, s>>>(h1.as<uint64_t>(), n, k0.as<uint64_t>(), v0.as<uint32_t>());
      const bool f = radix_sort(k0.as<uint64_t>(), v0.as<uint32_t>(), k1.as<uint64_t>(), v1.as<uint32_t>(), n, 0, 64,
                                sc, s, nullptr);
      launches += 1 + 40;
      const uint64_t *sk = f ? k1.as<uint64_t>() : k0.as<uint64_t>();
      const uint32_t *sv = f ? v1.as<uint32_t>() : v0.as<uint32_t>();
      tck(cudaMemsetAsync(stats.p, 0, sizeof(TcStats) + 8, s), "memset");
      k_tc_split<<<gb, 256, 0, s>>>(sk, sv, n, kept.as<uint64_t>(), tmp.as<uint32_t>(), stats.as<TcStats>());
      k_tc_dupcheck<<<(unsigned)nsm * 8, TC_T, smem(sp.P), s>>>(sp, sk, sv, n, tmp.as<uint32_t>(), h2.as<uint64_t>(),
                                                                pmx, pe, stats.as<TcStats>(), unres, ovf.as<int>());
      launches += 2;
      tck(cudaGetLastError(), "dedupe");
      unsigned long long hu = 0;
      tck(cudaMemcpyAsync(&hs, stats.p, sizeof hs, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaMemcpyAsync(&hu, unres, 8, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaStreamSynchronize(s), "dedupe");
      check_ovf();
      resolved = hu == 0;
    }
    if (!resolved) {
      k_tc_seen_init<<<gb, 256, 0, s>>>(h1.as<uint64_t>(), n, k0.as<uint64_t>(), v0.as<uint32_t>());
      const bool f = radix_sort(k0.as<uint64_t>(), v0.as<uint32_t>(), k1.as<uint64_t>(), v1.as<uint32_t>(), n, 32, 64,
                                sc, s, nullptr);
      launches += 1 + 20;
      const uint64_t *sk = f ? k1.as<uint64_t>() : k0.as<uint64_t>();
      const uint32_t *sv = f ? v1.as<uint32_t>() : v0.as<uint32_t>();
      tck(cudaMemsetAsync(stats.p, 0, sizeof(TcStats), s), "memset");
      k_tc_runs<<<gb, 256, 0, s>>>(sk, sv, n, kept.as<uint64_t>(), work.as<uint2>(), stats.as<TcStats>());
      k_tc_resolve<<<(unsigned)nsm * 4, TC_T, smem(sp.P), s>>>(sp, T.hist(), tp, work.as<uint2>(), sv, h1.as<uint64_t>(),
                                                               h2.as<uint64_t>(), tmp.as<uint32_t>(), kept.as<uint64_t>(),
                                                               stats.as<TcStats>(), ovf.as<int>(), pmx, pe);
      launches += 2;
      tck(cudaGetLastError(), "dedupe");
      tck(cudaMemcpyAsync(&hs, stats.p, sizeof hs, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaStreamSynchronize(s), "dedupe");
      check_ovf();
    }
    const size_t nk = (size_t)hs.n_kept;
    // index order: radix sort of the kept child indices (< 2^32)
    const bool fk = radix_sort(kept.as<uint64_t>(), v0.as<uint32_t>(), k1.as<uint64_t>(), v1.as<uint32_t>(), nk, 0, 32,
                               sc, s, nullptr);
    if (nk > 1) launches += 20;
    const uint64_t *kidx = fk ? k1.as<uint64_t>() : kept.as<uint64_t>();
    T.par.emplace_back(); T.gat.emplace_back(); T.n.push_back((long long)nk);
    T.par.back().ensure(nk * 4 + 4); T.gat.back().ensure(nk + 4);
    T.F1.ensure(nk * 8 + 8); T.F2.ensure(nk * 8 + 8);
    k_tc_gather<<<(unsigned)std::max<size_t>(1, std::min<size_t>((nk + 255) / 256, (size_t)nsm * 16)), 256, 0, s>>>(
        kidx, nk, G, h1.as<uint64_t>(), h2.as<uint64_t>(), T.par.back().as<uint32_t>(),
        T.gat.back().as<uint8_t>(), T.F1.as<uint64_t>(), T.F2.as<uint64_t>());
    launches++;
    tck(cudaGetLastError(), "gather");
    long long fresh = (long long)nk;
    if (tab && nk) {   // drop cosets present at a lower level, then add the rest to the table
      hits.ensure(nk * 8);
      k_tc_lookup<<<grid(nk), TC_T, smem(sp.P), s>>>(sp, T.hist(), t, T.F1.as<uint64_t>(), T.F2.as<uint64_t>(), (long long)nk,
                                                      sp, T.hist(), tab->S1.as<uint64_t>(), tab->S2.as<uint64_t>(),
                                                      tab->Sidx.as<uint32_t>(), tab->Slvl.as<uint32_t>(), tab->ns, t - 1,
                                                      hits.as<long long>(), ovf.as<int>());
      launches++;
      tck(cudaGetLastError(), "table filter");
      check_ovf();
      std::vector<long long> hh(nk);
      std::vector<uint32_t> hp(nk);
      std::vector<uint8_t> hg(nk);
      std::vector<uint64_t> a1(nk), a2(nk);
      tck(cudaMemcpyAsync(hh.data(), hits.p, nk * 8, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaMemcpyAsync(hp.data(), T.par.back().p, nk * 4, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaMemcpyAsync(hg.data(), T.gat.back().p, nk, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaMemcpyAsync(a1.data(), T.F1.p, nk * 8, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaMemcpyAsync(a2.data(), T.F2.p, nk * 8, cudaMemcpyDeviceToHost, s), "d2h");
      tck(cudaStreamSynchronize(s), "d2h");
      std::vector<uint32_t> np;
      std::vector<uint8_t> ng;
      std::vector<uint64_t> n1, n2;
      for (size_t j = 0; j < nk; j++)
        if (hh[j] < 0) { np.push_back(hp[j]); ng.push_back(hg[j]); n1.push_back(a1[j]); n2.push_back(a2[j]); }
      fresh = (long long)np.size();
      T.n.back() = fresh;
      if (fresh) {
        tck(cudaMemcpyAsync(T.par.back().p, np.data(), fresh * 4, cudaMemcpyHostToDevice, s), "h2d");
        tck(cudaMemcpyAsync(T.gat.back().p, ng.data(), fresh, cudaMemcpyHostToDevice, s), "h2d");
        tck(cudaMemcpyAsync(T.F1.p, n1.data(), fresh * 8, cudaMemcpyHostToDevice, s), "h2d");
        tck(cudaMemcpyAsync(T.F2.p, n2.data(), fresh * 8, cudaMemcpyHostToDevice, s), "h2d");
        tck(cudaStreamSynchronize(s), "h2d");
        add_to_table(*tab, T, t);
      }
    }
    TcLevel L;
    L.table = tab != nullptr; L.t = t; L.parents = m; L.children = nc; L.cosets = (long long)nk; L.fresh = fresh;
    L.seconds = now_s() - t0;
    cb(L);
    return fresh;
  }

  // append level t of T (its nodes and keys T.F1/F2) to the table and keep the keys sorted by h1
  void add_to_table(Table &tab, Tree &T, int t) {
    const long long nn = T.n[t], tot = tab.ns + nn;
    Buf a1, a2, ai, al;
    a1.ensure(tot * 8); a2.ensure(tot * 8); ai.ensure(tot * 4); al.ensure(tot * 4);
    if (tab.ns) {
      tck(cudaMemcpyAsync(a1.p, tab.S1.p, tab.ns * 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(a2.p, tab.S2.p, tab.ns * 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(ai.p, tab.Sidx.p, tab.ns * 4, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(al.p, tab.Slvl.p, tab.ns * 4, cudaMemcpyDeviceToDevice, s), "d2d");
    }
    tck(cudaMemcpyAsync(a1.as<uint64_t>() + tab.ns, T.F1.p, nn * 8, cudaMemcpyDeviceToDevice, s), "d2d");
    tck(cudaMemcpyAsync(a2.as<uint64_t>() + tab.ns, T.F2.p, nn * 8, cudaMemcpyDeviceToDevice, s), "d2d");
    {
      std::vector<uint32_t> idx(nn), lv(nn, (uint32_t)t);
      for (long long i = 0; i < nn; i++) idx[i] = (uint32_t)i;
      tck(cudaMemcpyAsync(ai.as<uint32_t>() + tab.ns, idx.data(), nn * 4, cudaMemcpyHostToDevice, s), "h2d");
      tck(cudaMemcpyAsync(al.as<uint32_t>() + tab.ns, lv.data(), nn * 4, cudaMemcpyHostToDevice, s), "h2d");
      tck(cudaStreamSynchronize(s), "h2d");
    }
    sort_table(tab, a1, a2, ai, al, tot);
  }
  void sort_table(Table &tab, Buf &a1, Buf &a2, Buf &ai, Buf &al, long long tot) {
    const size_t n = (size_t)tot;
    k0.ensure(n * 8); k1.ensure(n * 8); v0.ensure(n * 4); v1.ensure(n * 4);
    hist.ensure(sort_hist_words(n) * 4); part.ensure(scan_partials_words(sort_hist_words(n)) * 4);
    SortScratch sc{hist.as<uint32_t>(), part.as<uint32_t>(), hist.cap / 4, part.cap / 4};
    const unsigned gb = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)nsm * 16);
    k_tc_seen_init<<<gb, 256, 0, s>>>(a1.as<uint64_t>(), n, k0.as<uint64_t>(), v0.as<uint32_t>());
    const bool f = radix_sort(k0.as<uint64_t>(), v0.as<uint32_t>(), k1.as<uint64_t>(), v1.as<uint32_t>(), n, 0, 64, sc,
                              s, nullptr);
    launches += 1 + 40;
    const uint32_t *order = f ? v1.as<uint32_t>() : v0.as<uint32_t>();
    tab.S1.ensure(n * 8); tab.S2.ensure(n * 8); tab.Sidx.ensure(n * 4); tab.Slvl.ensure(n * 4);
    k_tc_seen_gather<<<gb, 256, 0, s>>>(order, n, a1.as<uint64_t>(), a2.as<uint64_t>(), ai.as<uint32_t>(),
                                        al.as<uint32_t>(), tab.S1.as<uint64_t>(), tab.S2.as<uint64_t>(),
                                        tab.Sidx.as<uint32_t>(), tab.Slvl.as<uint32_t>());
    launches++;
    tck(cudaStreamSynchronize(s), "table sort");
    a1.release(); a2.release(); ai.release(); al.release();
    tab.ns = tot;
  }

  // the table of (n, K): resident, else the cache file, else built from the identity
  Table *table(const TDev &si, const TSpec &sp, const TcOptions &opt, const std::function<void(const TcLevel &)> &cb,
               TcResult &res);
  bool load(const std::string &path, const TDev &si, Table &tab, int K);
  void save(const std::string &path, const Table &tab);
};

bool TcountContext::load(const std::string &path, const TDev &si, Table &tab, int K) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  int nl = 0;
  bool ok = std::fread(&nl, sizeof nl, 1, f) == 1 && nl >= 0 && nl <= MAXT && nl <= K;
  std::vector<std::vector<uint32_t>> P;
  std::vector<std::vector<uint8_t>> G;
  for (int l = 1; ok && l <= nl; l++) {
    long n = 0;
    ok = std::fread(&n, sizeof n, 1, f) == 1 && n >= 0 && n <= size;
    if (!ok) break;
    P.emplace_back(n); G.emplace_back(n);
    ok = std::fread(P.back().data(), 4, n, f) == (size_t)n && std::fread(G.back().data(), 1, n, f) == (size_t)n;
  }
  // keys: trusted only when the file ends with this build's trailer (same key hash); else recomputed below
  long ns = 0;
  std::vector<uint64_t> k1, k2;
  std::vector<uint32_t> ki, kl;
  bool trusted = false;
  if (ok && std::fread(&ns, sizeof ns, 1, f) == 1 && ns > 0 && ns <= size) {
    k1.resize(ns); k2.resize(ns); ki.resize(ns); kl.resize(ns);
    bool kok = true;
    for (long i = 0; kok && i < ns; i++)
      kok = std::fread(&k1[i], 8, 1, f) == 1 && std::fread(&k2[i], 8, 1, f) == 1 && std::fread(&ki[i], 4, 1, f) == 1 &&
            std::fread(&kl[i], 4, 1, f) == 1;
    uint32_t trailer[2] = {0, 0};
    trusted = kok && std::fread(trailer, 4, 2, f) == 2 && trailer[0] == TC_CACHE_MAGIC && trailer[1] == TC_KEY_VERSION;
  }
  std::fclose(f);
  // every parent index and rotation in range (a damaged file is rebuilt, never replayed out of bounds), and every
  // trusted key record names a node of the tree
  for (int l = 1; ok && l <= nl; l++) {
    const size_t below = l == 1 ? 1 : P[l - 2].size();
    for (size_t j = 0; ok && j < P[l - 1].size(); j++)
      ok = P[l - 1][j] < below && G[l - 1][j] >= 1 && (int)G[l - 1][j] < si.P;
  }
  if (!ok) return false;
  for (long i = 0; trusted && i < ns; i++)
    trusted = kl[i] == 0 ? ki[i] == 0 : (kl[i] <= (uint32_t)nl && ki[i] < P[kl[i] - 1].size());
  Tree &D = tab.D;
  if (trusted) {
    for (int l = 1; l <= nl; l++) {
      const long long n = (long long)P[l - 1].size();
      D.par.emplace_back(); D.gat.emplace_back(); D.n.push_back(n);
      D.par.back().ensure(n * 4 + 4); D.gat.back().ensure(n + 4);
      tck(cudaMemcpyAsync(D.par.back().p, P[l - 1].data(), n * 4, cudaMemcpyHostToDevice, s), "h2d");
      tck(cudaMemcpyAsync(D.gat.back().p, G[l - 1].data(), n, cudaMemcpyHostToDevice, s), "h2d");
    }
    tab.S1.ensure(ns * 8); tab.S2.ensure(ns * 8); tab.Sidx.ensure(ns * 4); tab.Slvl.ensure(ns * 4);
    tck(cudaMemcpyAsync(tab.S1.p, k1.data(), ns * 8, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaMemcpyAsync(tab.S2.p, k2.data(), ns * 8, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaMemcpyAsync(tab.Sidx.p, ki.data(), ns * 4, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaMemcpyAsync(tab.Slvl.p, kl.data(), ns * 4, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaStreamSynchronize(s), "h2d");
    tab.ns = ns;
    return true;
  }
  // keys made by another program (a reference-written file): recompute every node's key with this build's hash
  for (int l = 1; l <= nl; l++) {
    const long long n = (long long)P[l - 1].size();
    D.par.emplace_back(); D.gat.emplace_back(); D.n.push_back(n);
    D.par.back().ensure(n * 4 + 4); D.gat.back().ensure(n + 4);
    tck(cudaMemcpyAsync(D.par.back().p, P[l - 1].data(), n * 4, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaMemcpyAsync(D.gat.back().p, G[l - 1].data(), n, cudaMemcpyHostToDevice, s), "h2d");
  }
  tck(cudaStreamSynchronize(s), "h2d");
  for (int l = 0; l <= nl; l++) {
    level_keys(si, D, l);
    const long long n = D.n[l], tot = tab.ns + n;
    Buf a1, a2, ai, al;
    a1.ensure(tot * 8); a2.ensure(tot * 8); ai.ensure(tot * 4); al.ensure(tot * 4);
    if (tab.ns) {
      tck(cudaMemcpyAsync(a1.p, tab.S1.p, tab.ns * 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(a2.p, tab.S2.p, tab.ns * 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(ai.p, tab.Sidx.p, tab.ns * 4, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(al.p, tab.Slvl.p, tab.ns * 4, cudaMemcpyDeviceToDevice, s), "d2d");
    }
    tck(cudaMemcpyAsync(a1.as<uint64_t>() + tab.ns, D.F1.p, n * 8, cudaMemcpyDeviceToDevice, s), "d2d");
    tck(cudaMemcpyAsync(a2.as<uint64_t>() + tab.ns, D.F2.p, n * 8, cudaMemcpyDeviceToDevice, s), "d2d");
    std::vector<uint32_t> idx(n), lv(n, (uint32_t)l);
    for (long long i = 0; i < n; i++) idx[i] = (uint32_t)i;
    tck(cudaMemcpyAsync(ai.as<uint32_t>() + tab.ns, idx.data(), n * 4, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaMemcpyAsync(al.as<uint32_t>() + tab.ns, lv.data(), n * 4, cudaMemcpyHostToDevice, s), "h2d");
    tck(cudaStreamSynchronize(s), "h2d");
    sort_table(tab, a1, a2, ai, al, tot);
  }
  check_ovf();
  return true;
}

void TcountContext::save(const std::string &path, const Table &tab) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) { std::fprintf(stderr, "cannot write %s (table not cached)\n", path.c_str()); return; }
  const Tree &D = tab.D;
  const int nl = D.top();
  std::fwrite(&nl, sizeof nl, 1, f);
  for (int l = 1; l <= nl; l++) {
    const long n = (long)D.n[l];
    std::vector<uint32_t> P(n);
    std::vector<uint8_t> G(n);
    cudaMemcpy(P.data(), D.par[l].p, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(G.data(), D.gat[l].p, n, cudaMemcpyDeviceToHost);
    std::fwrite(&n, sizeof n, 1, f); std::fwrite(P.data(), 4, n, f); std::fwrite(G.data(), 1, n, f);
  }
  // table entries in the reference's DKey layout {h1, h2, idx, lvl} (the keys are this build's)
  const long ns = (long)tab.ns;
  std::vector<uint64_t> a1(ns), a2(ns);
  std::vector<uint32_t> ai(ns), al(ns);
  cudaMemcpy(a1.data(), tab.S1.p, ns * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(a2.data(), tab.S2.p, ns * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(ai.data(), tab.Sidx.p, ns * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(al.data(), tab.Slvl.p, ns * 4, cudaMemcpyDeviceToHost);
  std::fwrite(&ns, sizeof ns, 1, f);
  for (long i = 0; i < ns; i++) {
    std::fwrite(&a1[i], 8, 1, f); std::fwrite(&a2[i], 8, 1, f); std::fwrite(&ai[i], 4, 1, f); std::fwrite(&al[i], 4, 1, f);
  }
  const uint32_t trailer[2] = {TC_CACHE_MAGIC, TC_KEY_VERSION};   // past the reference's layout: its reader stops before
  std::fwrite(trailer, 4, 2, f);
  std::fclose(f);
}

Table *TcountContext::table(const TDev &si, const TSpec &sp, const TcOptions &opt,
                            const std::function<void(const TcLevel &)> &cb, TcResult &res) {
  const auto key = std::make_pair(sp.n, opt.table_k);
  auto it = tables.find(key);
  if (it != tables.end()) { res.table_resident = true; return it->second; }
  const double t0 = now_s();
  Table *tab = new Table;
  char mine[512], theirs[512];
  std::snprintf(mine, sizeof mine, "%s/tcount-table-n%d-k%d.cz.bin", opt.cache_dir.c_str(), sp.n, opt.table_k);
  std::snprintf(theirs, sizeof theirs, "%s/tcount-table-n%d-k%d.bin", opt.cache_dir.c_str(), sp.n, opt.table_k);
  res.table_path = mine;
  if (opt.use_cache && (load(mine, si, *tab, opt.table_k) || load(theirs, si, *tab, opt.table_k))) {
    res.table_loaded = true;
  } else {
    tab->D.release();
    tab->D = Tree{};
    tab->ns = 0;
    level_keys(si, tab->D, 0);                                    // level 0: the Clifford coset
    check_ovf();
    {
      Buf a1, a2, ai, al;
      a1.ensure(8); a2.ensure(8); ai.ensure(4); al.ensure(4);
      tck(cudaMemcpyAsync(a1.p, tab->D.F1.p, 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemcpyAsync(a2.p, tab->D.F2.p, 8, cudaMemcpyDeviceToDevice, s), "d2d");
      tck(cudaMemsetAsync(ai.p, 0, 4, s), "memset");
      tck(cudaMemsetAsync(al.p, 0, 4, s), "memset");
      sort_table(*tab, a1, a2, ai, al, 1);
    }
    for (int l = 1; l <= opt.table_k; l++) if (!grow(si, tab->D, tab, cb)) break;
    res.table_built = true;
    if (opt.use_cache) save(mine, *tab);
  }
  res.table_seconds = now_s() - t0;
  tables[key] = tab;
  return tab;
}

int parse_tspec(const char *text, size_t len, TSpec &s, std::string &err) {
  s = TSpec{};
  const char *p = text, *end = text + len;
  auto tok = [&](std::string &out) {
    while (p < end && std::isspace((unsigned char)*p)) p++;
    if (p >= end) return false;
    const char *b = p;
    while (p < end && !std::isspace((unsigned char)*p)) p++;
    out.assign(b, p);
    return true;
  };
  bool fail = false;
  auto num = [&]() -> long long {
    std::string t;
    if (fail || !tok(t)) { fail = true; return 0; }
    char *e;
    const long long v = std::strtoll(t.c_str(), &e, 10);
    if (e == t.c_str()) { fail = true; return 0; }
    return v;
  };
  std::string t;
  if (!tok(t) || t != "tcount-spec") { err = "not a tcount spec"; return 2; }
  (void)num();
  while (!fail && tok(t)) {
    if (t == "n") {
      s.n = (int)num();
      if (s.n < 1 || s.n > 3) { err = "n = " + std::to_string(s.n) + " not supported (1 <= n <= 3)"; return 3; }
      s.P = 1 << (2 * s.n);
    } else if (t == "channel") {
      s.e = (int)num();
      s.x.resize((size_t)s.P * s.P); s.y.resize((size_t)s.P * s.P);
      for (int i = 0; i < s.P * s.P; i++) { s.x[i] = (int)num(); s.y[i] = (int)num(); }
    } else if (t == "rotations") {
      const int m = (int)num();
      if (m < 0 || m > MAXP) { fail = true; break; }
      s.tr.resize((size_t)m * s.P); s.ts.resize((size_t)m * s.P);
      for (int i = 0; i < m * s.P; i++) { s.tr[i] = (int)num(); s.ts[i] = (int)num(); }
    } else if (t == "end") break;
    else { err = "unknown field " + t; return 2; }
  }
  if (s.P > MAXP || s.n < 1) { err = "n = " + std::to_string(s.n) + " not supported (1 <= n <= 3)"; return 3; }
  if ((int)s.tr.size() != (s.P - 1) * s.P || (int)s.x.size() != s.P * s.P) { err = "incomplete tcount spec"; return 2; }
  for (int i = 0; i < (int)s.tr.size(); i++)
    if (s.tr[i] >= s.P || s.tr[i] < -1 || s.ts[i] < -1 || s.ts[i] > 1) { err = "bad rotation table"; return 2; }
  return 0;
}

TcountContext *tcount_context_create(int device, void *stream) { return new TcountContext(device, stream); }
void tcount_context_destroy(TcountContext *c) { delete c; }
size_t tcount_context_trim(TcountContext *c) {
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->s);
  return c->trim();
}

int tcount_run(TcountContext *ctx, const TSpec &sp, const TcOptions &opt,
               const std::function<void(const TcLevel &)> &on_level, TcResult &res) {
  res = TcResult{};
  res.maxt = opt.maxt;
  const double t0 = now_s();
  const long long l0 = ctx->launches;
  try {
    tck(cudaSetDevice(ctx->dev), "cudaSetDevice");
    const int P = sp.P, lp = 2 * sp.n;
    const size_t sm = ctx->smem(P);
    for (const void *k : {(const void *)k_tc_keys, (const void *)k_tc_children, (const void *)k_tc_resolve,
                          (const void *)k_tc_dupcheck, (const void *)k_tc_lookup})
      tck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "smem attribute");
    ctx->bx.ensure(P * P * 4); ctx->by.ensure(P * P * 4); ctx->ix.ensure(P * P * 4); ctx->iy.ensure(P * P * 4);
    ctx->tr.ensure(P * P); ctx->ts.ensure(P * P); ctx->ovf.ensure(4);
    std::vector<int> ix(P * P, 0), iy(P * P, 0);
    for (int i = 0; i < P; i++) ix[i * P + i] = 1;
    std::vector<int8_t> tr8(sp.tr.begin(), sp.tr.end()), ts8(sp.ts.begin(), sp.ts.end());
    tck(cudaMemcpyAsync(ctx->bx.p, sp.x.data(), P * P * 4, cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemcpyAsync(ctx->by.p, sp.y.data(), P * P * 4, cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemcpyAsync(ctx->ix.p, ix.data(), P * P * 4, cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemcpyAsync(ctx->iy.p, iy.data(), P * P * 4, cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemcpyAsync(ctx->tr.p, tr8.data(), tr8.size(), cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemcpyAsync(ctx->ts.p, ts8.data(), ts8.size(), cudaMemcpyHostToDevice, ctx->s), "h2d");
    tck(cudaMemsetAsync(ctx->ovf.p, 0, 4, ctx->s), "memset");
    tck(cudaStreamSynchronize(ctx->s), "upload");
    TDev su{sp.n, P, lp, P - 1, ctx->bx.as<int>(), ctx->by.as<int>(), sp.e, ctx->tr.as<int8_t>(), ctx->ts.as<int8_t>()};
    TDev si = su;
    si.bx = ctx->ix.as<int>(); si.by = ctx->iy.as<int>(); si.be = 0;

    Table *tab = ctx->table(si, sp, opt, on_level, res);
    res.table_cosets = tab->ns;
    res.table_levels = tab->D.top();
    Tree T;                                                       // search: peel rotations off U
    ctx->level_keys(su, T, 0);
    ctx->check_ovf();
    int rc = 1;
    for (int j = 0; j <= opt.maxt; j++) {
      if (j > 0 && !ctx->grow(su, T, nullptr, on_level)) break;
      const long long n = T.n[j];
      const int maxc = std::min(tab->D.top(), opt.maxt - j);
      ctx->hits.ensure(n * 8);
      k_tc_lookup<<<ctx->grid(n), TC_T, sm, ctx->s>>>(su, T.hist(), j, T.F1.as<uint64_t>(), T.F2.as<uint64_t>(), n, si,
                                                      tab->D.hist(), tab->S1.as<uint64_t>(), tab->S2.as<uint64_t>(),
                                                      tab->Sidx.as<uint32_t>(), tab->Slvl.as<uint32_t>(), tab->ns, maxc,
                                                      ctx->hits.as<long long>(), ctx->ovf.as<int>());
      ctx->launches++;
      tck(cudaGetLastError(), "lookup");
      ctx->check_ovf();
      std::vector<long long> hh(n);
      tck(cudaMemcpyAsync(hh.data(), ctx->hits.p, n * 8, cudaMemcpyDeviceToHost, ctx->s), "d2h");
      tck(cudaStreamSynchronize(ctx->s), "d2h");
      long long best = -1, bestx = -1;
      int bestc = 1 << 30;
      for (long long i = 0; i < n; i++) {
        if (hh[i] < 0) continue;
        uint32_t lv = 0;
        tck(cudaMemcpy(&lv, tab->Slvl.as<uint32_t>() + hh[i], 4, cudaMemcpyDeviceToHost), "d2h");
        if ((int)lv < bestc) { bestc = (int)lv; best = i; bestx = hh[i]; }
      }
      if (best >= 0) {
        // U = R(P_1)..R(P_j) S with S = R(Q_c)^-1 .. R(Q_1)^-1 C' (the table entry's peels Q_1..Q_c from I)
        auto seq = [&](const Tree &Tr, int t, uint32_t i) {
          std::vector<int> v(t);
          for (int l = t; l >= 1; l--) {
            uint8_t g; uint32_t pp;
            tck(cudaMemcpy(&g, Tr.gat[l].as<uint8_t>() + i, 1, cudaMemcpyDeviceToHost), "d2h");
            tck(cudaMemcpy(&pp, Tr.par[l].as<uint32_t>() + i, 4, cudaMemcpyDeviceToHost), "d2h");
            v[l - 1] = g; i = pp;
          }
          return v;
        };
        uint32_t eidx = 0;
        tck(cudaMemcpy(&eidx, tab->Sidx.as<uint32_t>() + bestx, 4, cudaMemcpyDeviceToHost), "d2h");
        const std::vector<int> fw = seq(T, j, (uint32_t)best), tb = seq(tab->D, bestc, eidx);
        for (int p : fw) res.rotations.push_back({p, 0});
        for (int i = (int)tb.size() - 1; i >= 0; i--) res.rotations.push_back({tb[i], 1});
        res.tcount = j + bestc;
        res.split_j = j;
        res.split_c = bestc;
        rc = 0;
        break;
      }
      if (j + tab->D.top() >= opt.maxt) break;
    }
    T.release();
    res.rc = rc;
  } catch (const std::overflow_error &e) {
    res.error = e.what();
    res.rc = 4;
  } catch (const std::exception &e) {
    res.error = e.what();
    res.rc = 5;
  }
  res.launches = ctx->launches - l0;
  res.total_seconds = now_s() - t0;
  return res.rc;
}

}  // namespace cz
