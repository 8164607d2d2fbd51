// sm_100a kernels and host loop of the Clifford-table path (the reference's src/clifford.cu, "cliffopt").
//
// Reference semantics: breadth-first search over the n-qubit Clifford group from the identity with generators
// H, S, Sdg, X, Z on every qubit and CX on every ordered pair (clifford.cu:148-166, 247-276), giving the minimal
// gate count of every element; a beam search over the placements K of every T gate, K Z_q' K^-1 = +-Z_q, with
// the cost of a partial placement the summed minimal lengths of the segments fixed so far (:168-201, 281-330);
// every segment read back as an optimal word by walking the distances down (:343-372).
//
// B200 design:
//  * the table is direct-addressed by a perfect rank of the group element (cz_tableau.h): a 92.9 MB byte array of
//    distances at n = 3 that stays in L2 while it is probed, and a visited bitmap for the BFS claims (11.6 MB). No
//    keys, no probing chains, and no element array: the element of a rank is computed back from the rank (unrank)
//    for candidate enumeration and uniform draws, so the BFS writes one byte per new element at a random place;
//  * BFS: one thread per frontier element, all generators applied bit-parallel to the packed tableau, claims by
//    atomicOr on the bitmap after a plain read, warp-aggregated appends to the next frontier;
//  * beam step: dist(X) = dist(X^-1) (the generator set is closed under inverses), and X^-1 is the candidate
//    (a column of the candidate table) composed with the inverse of the beam state's left part, a 4^n-entry row
//    lookup table held in shared memory, so one evaluation is 2n lookups + a rank + one L2 byte load. The B
//    smallest (cost, index) pairs are selected exactly by a cost histogram and an ordered compaction instead of
//    sorting every packed cost;
//  * read-back: one warp per segment, a lane per generator, ballot picks the first generator one step closer.
// Candidates are ordered by their tableau value (the reference leaves their order to an atomic counter).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>

#include "cz_clifford.h"
#include "cz_sort.cuh"
#include "cz_tableau.h"

namespace cz {

namespace {

constexpr int CL_T = 256;
constexpr int HB = 2048;            // cost histogram bins
constexpr int SEL_I = 16, SEL_CH = CL_T * SEL_I;
constexpr int MAXBEAM = 255;
constexpr int WORDMAX = 32;         // longest optimal word read back (13 at n = 3)

struct GateSet {
  int ng;
  int8_t k[32], a[32], b[32];
};
GateSet gate_set(int n) {           // clifford.cu:148-153 order: per qubit h, s, sdg, x, z; then cx over ordered pairs
  GateSet g{};
  for (int q = 0; q < n; q++)
    for (int k : {CG_H, CG_S, CG_SDG, CG_X, CG_Z}) { g.k[g.ng] = (int8_t)k; g.a[g.ng] = (int8_t)q; g.b[g.ng] = 0; g.ng++; }
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++)
      if (a != b) { g.k[g.ng] = CG_CX; g.a[g.ng] = (int8_t)a; g.b[g.ng] = (int8_t)b; g.ng++; }
  return g;
}

// generator j of the n-qubit set in the order of gate_set, computed (no table): per qubit h, s, sdg, x, z, then
// cx over ordered pairs
template <int N>
struct Gen {
  static constexpr int NG = 5 * N + N * (N - 1);
  __host__ __device__ __forceinline__ static void get(int j, int &k, int &a, int &b) {
    if (j < 5 * N) { k = j % 5; a = j / 5; b = 0; return; }
    const int i = j - 5 * N, bb = N > 1 ? i % (N - 1) : 0;
    k = CG_CX;
    a = N > 1 ? i / (N - 1) : 0;
    b = bb + (bb >= a ? 1 : 0);
  }
};

struct ClCudaError : std::runtime_error { using std::runtime_error::runtime_error; };
void clk(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();            // a failed allocation must not be reported again by the next launch check
    throw ClCudaError(std::string("CUDA error after ") + what + ": " + cudaGetErrorString(e));
  }
}
double cl_now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

struct CBuf {
  void *p = nullptr;
  size_t cap = 0;
  void ensure(size_t b) {
    if (b <= cap) return;
    if (p) clk(cudaFree(p), "free");
    size_t c = std::max(b, cap + cap / 2);
    c = (c + 255) & ~(size_t)255;
    clk(cudaMalloc(&p, c), "cudaMalloc");
    cap = c;
  }
  template <typename T> T *as() const { return (T *)p; }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

// ---------------- kernels ----------------
template <int N>
__global__ void __launch_bounds__(CL_T) k_cl_bfs(const uint64_t *front, unsigned long long nf, uint64_t *next,
                                                 unsigned long long cap, unsigned long long *nn, uint32_t *seen,
                                                 uint8_t *dist, uint8_t d, int *ovf) {
  using T = Tb<N>;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += stride) {
    const uint64_t X = front[i];
#pragma unroll
    for (int j = 0; j < Gen<N>::NG; j++) {
      int gk, ga, gb;
      Gen<N>::get(j, gk, ga, gb);
      const uint64_t C = T::gate(X, gk, ga, gb);
      const uint32_t r = T::rank(C);
      bool fresh = false;
      if (r != T::BAD) {
        const uint32_t bit = 1u << (r & 31);
        if (!(__ldcg(&seen[r >> 5]) & bit)) fresh = !(atomicOr(&seen[r >> 5], bit) & bit);
      } else {
        atomicOr(ovf, 2);
      }
      if (fresh) dist[r] = d;
      const unsigned am = __activemask();
      const unsigned bal = __ballot_sync(am, fresh);
      if (bal) {
        const int leader = __ffs((int)am) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(nn, (unsigned long long)__popc(bal));
        base = __shfl_sync(am, base, leader);
        const unsigned long long pos = base + (unsigned)__popc(bal & ((1u << lane) - 1));
        if (fresh) {
          if (pos < cap) next[pos] = C;
          else atomicOr(ovf, 1);
        }
      }
    }
  }
}

// placements of a T on qubit q: every K with K Z_q' K^-1 = +-Z_q for some q' (clifford.cu:170-183)
template <int N>
__global__ void k_cl_cands(unsigned long long order, uint64_t *lists, unsigned long long capq,
                           unsigned long long *cnt, int *ovf) {
  using T = Tb<N>;
  const int lane = threadIdx.x & 31;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long nit = (order + stride - 1) / stride;      // uniform trip count: full-warp ballots
  for (unsigned long long it = 0; it < nit; it++) {
    const unsigned long long r = it * stride + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = r < order;
    const uint64_t K = valid ? T::unrank((uint32_t)r) : 0;   // every rank is an element (the BFS covers the group)
#pragma unroll
    for (int q = 0; q < N; q++) {
      bool hit = false;
      if (valid)
        for (int qp = 0; qp < N; qp++)
          hit |= (T::row(K, N + qp) & T::SYM) == (1u << (N + q));
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (!bal) continue;
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&cnt[q], (unsigned long long)__popc(bal));
      base = __shfl_sync(0xffffffffu, base, 0);
      const unsigned long long pos = base + (unsigned)__popc(bal & ((1u << lane) - 1));
      if (hit) {
        if (pos < capq) lists[(unsigned long long)q * capq + pos] = K;
        else atomicOr(ovf, 1);
      }
    }
  }
}
template <int N>
__global__ void k_cl_cand_meta(const uint64_t *K, size_t n, int q, uint8_t *meta) {
  using T = Tb<N>;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint8_t m = 0;
    for (int qp = 0; qp < N; qp++) {
      const uint32_t w = T::row(K[i], N + qp);
      if ((w & T::SYM) == (1u << (N + q))) m = (uint8_t)(qp | ((w >> T::SB) << 2));
    }
    meta[i] = m;
  }
}
__global__ void k_cl_iota(uint32_t *v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}
__global__ void k_cl_gather_u64(const uint64_t *src, const uint32_t *order, size_t n, uint64_t *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[order[i]];
}

// beam step: cost of (state b, candidate c, flip f) at index (b * nc + c) * 2 + f, histogram relative to cmin
template <int N>
__global__ void __launch_bounds__(CL_T) k_cl_beam(const uint64_t *Kc, const uint8_t *meta, unsigned long long nc, int nb,
                                                  const uint8_t *tabs, const int *bcost, int dagger, int cmin,
                                                  const uint8_t *dist, uint16_t *cost, unsigned *hist) {
  using T = Tb<N>;
  constexpr int TS = 1 << (2 * N);
  __shared__ uint8_t stab[MAXBEAM * TS];
  __shared__ int sbc[MAXBEAM];
  __shared__ unsigned sh[HB];
  for (int i = threadIdx.x; i < nb * TS; i += blockDim.x) stab[i] = tabs[i];
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sbc[i] = bcost[i];
  for (int i = threadIdx.x; i < HB; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += stride) {
    const uint64_t K = Kc[c];
    const int m = meta[c], qp = m & 3, dg = dagger ^ (m >> 2);
    // the flipped placement's K o g^-1 (g = Sdg if the T is a dagger after the sign, else S): row X_qp -> +-Y_qp image
    const uint64_t Kf = T::with_row(K, qp, T::image(K, 1u << qp, 1u << qp) ^ ((dg ? 0u : 1u) << T::SB));
    for (int b = 0; b < nb; b++) {
      const uint8_t *tb = stab + b * TS;
#pragma unroll
      for (int f = 0; f < 2; f++) {
        const uint32_t r = T::rank(T::compose_tab(f ? Kf : K, tb));
        const int dd = r == T::BAD ? 999 : (int)dist[r];
        const int v = sbc[b] + dd;
        cost[((unsigned long long)b * nc + c) * 2 + f] = (uint16_t)v;
        atomicAdd(&sh[min(v - cmin, HB - 1)], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < HB; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}
// histogram of the costs >= base (bins relative to base)
__global__ void k_cl_hist(const uint16_t *cost, unsigned long long tot, int base, unsigned *hist) {
  __shared__ unsigned sh[HB];
  for (int i = threadIdx.x; i < HB; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const int v = cost[i];
    if (v >= base) atomicAdd(&sh[min(v - base, HB - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < HB; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__device__ __forceinline__ unsigned blk_excl_scan256(unsigned v, unsigned &total) {
  __shared__ unsigned ws[CL_T / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  unsigned pre = 0, tot = 0;
#pragma unroll
  for (int i = 0; i < CL_T / 32; i++) { if (i < w) pre += ws[i]; tot += ws[i]; }
  __syncthreads();
  total = tot;
  return pre + inc - v;
}
// entries below the threshold (fewer than the beam) appended as (cost << 32 | index); per-chunk counts of the
// entries at the threshold
__global__ void __launch_bounds__(CL_T) k_cl_sel_count(const uint16_t *cost, unsigned long long tot, int thr,
                                                       uint32_t *blkcnt, unsigned long long *below, unsigned *nbelow,
                                                       int cap) {
  const unsigned long long base = (unsigned long long)blockIdx.x * SEL_CH;
  unsigned eq = 0;
  for (int it = 0; it < SEL_I; it++) {
    const unsigned long long i = base + (unsigned long long)it * CL_T + threadIdx.x;
    if (i >= tot) break;
    const int v = cost[i];
    if (v == thr) eq++;
    else if (v < thr) {
      const unsigned p = atomicAdd(nbelow, 1u);
      if ((int)p < cap) below[p] = ((unsigned long long)v << 32) | i;
    }
  }
  unsigned total;
  (void)blk_excl_scan256(eq, total);
  if (threadIdx.x == 0) blkcnt[blockIdx.x] = total;
}
// the first `need` entries at the threshold, in index order
__global__ void __launch_bounds__(CL_T) k_cl_sel_write(const uint16_t *cost, unsigned long long tot, int thr,
                                                       const uint32_t *blkoff, unsigned need,
                                                       unsigned long long *eqlist) {
  unsigned run = blkoff[blockIdx.x];
  if (run >= need) return;
  const unsigned long long base = (unsigned long long)blockIdx.x * SEL_CH;
  for (int it = 0; it < SEL_I && run < need; it++) {
    const unsigned long long i = base + (unsigned long long)it * CL_T + threadIdx.x;
    const unsigned flag = (i < tot && cost[i] == thr) ? 1u : 0u;
    unsigned total;
    const unsigned pos = run + blk_excl_scan256(flag, total);
    if (flag && pos < need) eqlist[pos] = ((unsigned long long)thr << 32) | i;
    run += total;
  }
}
__global__ void k_cl_pick(const uint64_t *Kc, const uint8_t *meta, const unsigned long long *cidx, int m, uint64_t *oK,
                          uint8_t *oM) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) { oK[i] = Kc[cidx[i]]; oM[i] = meta[cidx[i]]; }
}
template <int N>
__global__ void k_cl_dist(const uint64_t *tab, size_t n, const uint8_t *dist, int *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t r = Tb<N>::rank(tab[i]);
    out[i] = r == Tb<N>::BAD ? -1 : (dist[r] == 0xff ? -1 : (int)dist[r]);
  }
}
template <int N>
__global__ void k_cl_elem(const uint64_t *idx, size_t n, unsigned long long order, uint64_t *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = idx[i] < order ? Tb<N>::unrank((uint32_t)idx[i]) : 0;
}
// one warp per segment: the optimal word of X, generators indexed into gs (clifford.cu:352-371)
template <int N>
__global__ void k_cl_word(const uint64_t *X0, int nseg, const uint8_t *dist, int8_t *out, int *len) {
  using T = Tb<N>;
  const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= nseg) return;
  uint64_t X = X0[w];
  const uint32_t r0 = T::rank(X);
  int d = r0 == T::BAD || dist[r0] == 0xff ? -1 : (int)dist[r0];
  if (d < 0 || d > WORDMAX) { if (lane == 0) len[w] = -1; return; }
  if (lane == 0) len[w] = d;
  for (int pos = d - 1; pos >= 0; pos--) {
    uint64_t pre = 0;
    bool ok = false;
    if (lane < Gen<N>::NG) {
      int gk, ga, gb;
      Gen<N>::get(lane, gk, ga, gb);
      pre = T::gate(X, T::inverse_kind(gk), ga, gb);
      const uint32_t r = T::rank(pre);
      ok = r != T::BAD && dist[r] == pos;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (!bal) { if (lane == 0) len[w] = -2; return; }
    const int g = __ffs((int)bal) - 1;
    X = __shfl_sync(0xffffffffu, pre, g);
    if (lane == 0) out[w * WORDMAX + pos] = (int8_t)g;
  }
}

// host-side tableau ops at runtime n
uint64_t h_identity(int n) { return n == 1 ? Tb<1>::identity() : n == 2 ? Tb<2>::identity() : Tb<3>::identity(); }
uint64_t h_gate(int n, uint64_t T, int k, int a, int b) {
  return n == 1 ? Tb<1>::gate(T, k, a, b) : n == 2 ? Tb<2>::gate(T, k, a, b) : Tb<3>::gate(T, k, a, b);
}
uint64_t h_compose(int n, uint64_t A, uint64_t B) {
  return n == 1 ? Tb<1>::compose(A, B) : n == 2 ? Tb<2>::compose(A, B) : Tb<3>::compose(A, B);
}
uint64_t h_inverse(int n, uint64_t A) { return n == 1 ? Tb<1>::inverse(A) : n == 2 ? Tb<2>::inverse(A) : Tb<3>::inverse(A); }
void h_image_table(int n, uint64_t B, uint8_t *tab) {
  if (n == 1) Tb<1>::image_table(B, tab); else if (n == 2) Tb<2>::image_table(B, tab); else Tb<3>::image_table(B, tab);
}

}  // namespace

struct CTable {
  int n = 0;
  long long order = 0;
  CBuf dist;
  CBuf candK[3], candM[3];
  unsigned long long ncand[3] = {0, 0, 0};
  CliffTableInfo info;
  void release() { dist.release(); for (int q = 0; q < 3; q++) { candK[q].release(); candM[q].release(); } }
};

class CliffordContext {
 public:
  int dev;
  cudaStream_t s;
  int nsm = 148;
  std::map<int, CTable *> tables;
  CBuf ovf, cnt, cost, hist, below, nbelow, blk, blkoff, part, eql, tabs, bc, pk, pm, tmp, out, len;
  long long launches = 0;
  CliffordContext(int d, void *stream) : dev(d), s((cudaStream_t)stream) {
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  ~CliffordContext() {
    cudaSetDevice(dev);
    for (auto &kv : tables) { kv.second->release(); delete kv.second; }
    for (CBuf *b : {&ovf, &cnt, &cost, &hist, &below, &nbelow, &blk, &blkoff, &part, &eql, &tabs, &bc, &pk, &pm, &tmp,
                    &out, &len})
      b->release();
  }
  size_t trim() {                              // work buffers back to the device; resident tables stay
    size_t n = 0;
    for (CBuf *b : {&cnt, &cost, &hist, &below, &nbelow, &blk, &blkoff, &part, &eql, &tabs, &bc, &pk, &pm, &tmp, &out,
                    &len}) {
      n += b->cap;
      b->release();
    }
    return n;
  }
  unsigned grid(unsigned long long n, int per = 8) const {
    return (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>((n + CL_T - 1) / CL_T,
                                                                                   (unsigned long long)nsm * per));
  }
  void sync(const char *what) { clk(cudaStreamSynchronize(s), what); }

  CTable *table(int n, CliffTableInfo &info);
  template <int N> void build(CTable &t);
  template <int N> void beam_step(CTable &t, int q, int dagger, const std::vector<uint64_t> &left,
                                  const std::vector<int> &bcost, int beam, std::vector<unsigned long long> &picked,
                                  std::vector<int> &pcost);
  std::vector<int> dist_of(CTable &t, const std::vector<uint64_t> &x);
  void words(CTable &t, const std::vector<uint64_t> &x, std::vector<std::vector<int>> &w);
};

template <int N>
void CliffordContext::build(CTable &t) {
  using T = Tb<N>;
  const double t0 = cl_now();
  const unsigned long long order = (unsigned long long)clifford_order(N);
  t.n = N;
  t.order = (long long)order;
  t.dist.ensure(order);
  CBuf seen, fa, fb;
  const unsigned long long words = (order + 31) / 32;
  seen.ensure(words * 4);
  fa.ensure(order * 8); fb.ensure(order * 8);
  ovf.ensure(4); cnt.ensure(64);
  clk(cudaMemsetAsync(t.dist.p, 0xff, order, s), "memset");
  clk(cudaMemsetAsync(seen.p, 0, words * 4, s), "memset");
  clk(cudaMemsetAsync(ovf.p, 0, 4, s), "memset");
  const uint64_t id = T::identity();
  const uint32_t r0 = T::rank(id);
  const uint8_t zero = 0;
  const uint32_t bit = 1u << (r0 & 31);
  clk(cudaMemcpyAsync(t.dist.as<uint8_t>() + r0, &zero, 1, cudaMemcpyHostToDevice, s), "h2d");
  clk(cudaMemcpyAsync(seen.as<uint32_t>() + (r0 >> 5), &bit, 4, cudaMemcpyHostToDevice, s), "h2d");
  clk(cudaMemcpyAsync(fa.p, &id, 8, cudaMemcpyHostToDevice, s), "h2d");
  CliffTableInfo &inf = t.info;
  inf = CliffTableInfo{};
  inf.n = N;
  inf.order = (long long)order;
  unsigned long long nf = 1, total = 1;
  for (int d = 1; nf; d++) {
    clk(cudaMemsetAsync(cnt.p, 0, 8, s), "memset");
    k_cl_bfs<N><<<grid(nf), CL_T, 0, s>>>(fa.as<uint64_t>(), nf, fb.as<uint64_t>(), order, cnt.as<unsigned long long>(),
                                          seen.as<uint32_t>(), t.dist.as<uint8_t>(), (uint8_t)d,
                                          ovf.as<int>());
    launches++;
    clk(cudaGetLastError(), "bfs");
    unsigned long long nn = 0;
    int of = 0;
    clk(cudaMemcpyAsync(&nn, cnt.p, 8, cudaMemcpyDeviceToHost, s), "d2h");
    clk(cudaMemcpyAsync(&of, ovf.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
    sync("bfs");
    if (of) throw std::overflow_error("BFS frontier overflow or invalid tableau");
    nf = nn;
    total += nf;
    if (nf) { if (d < 32) inf.per_distance[d] = (long long)nf; inf.max_distance = d; }
    std::swap(fa, fb);
  }
  inf.per_distance[0] = 1;
  inf.elements = (long long)total;
  seen.release(); fa.release(); fb.release();
  if (total != order) throw std::logic_error("group order mismatch");
  // placement candidates per qubit, ordered by tableau value
  const unsigned long long capq = order / ((1ULL << (2 * N)) - 1) * N + 64;
  CBuf lists;
  lists.ensure(capq * N * 8);
  clk(cudaMemsetAsync(cnt.p, 0, 64, s), "memset");
  k_cl_cands<N><<<grid(order), CL_T, 0, s>>>(order, lists.as<uint64_t>(), capq,
                                             cnt.as<unsigned long long>(), ovf.as<int>());
  launches++;
  clk(cudaGetLastError(), "candidates");
  unsigned long long nc[3] = {0, 0, 0};
  int of = 0;
  clk(cudaMemcpyAsync(nc, cnt.p, 24, cudaMemcpyDeviceToHost, s), "d2h");
  clk(cudaMemcpyAsync(&of, ovf.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
  sync("candidates");
  if (of) throw std::overflow_error("candidate buffer too small");
  for (int q = 0; q < N; q++) {
    const size_t m = (size_t)nc[q];
    t.ncand[q] = m;
    t.candK[q].ensure(m * 8 + 8); t.candM[q].ensure(m + 8);
    CBuf k1, v0, v1, hs, pt;
    k1.ensure(m * 8 + 8); v0.ensure(m * 4 + 4); v1.ensure(m * 4 + 4);
    hs.ensure(sort_hist_words(m) * 4 + 4); pt.ensure(scan_partials_words(sort_hist_words(m)) * 4 + 4);
    uint64_t *k0 = lists.as<uint64_t>() + (size_t)q * capq;
    k_cl_iota<<<grid(m), CL_T, 0, s>>>(v0.as<uint32_t>(), m);
    SortScratch sc{hs.as<uint32_t>(), pt.as<uint32_t>(), hs.cap / 4, pt.cap / 4};
    int ln = 0;
    const bool f = radix_sort(k0, v0.as<uint32_t>(), k1.as<uint64_t>(), v1.as<uint32_t>(), m, 0,
                              ((T::RB * T::ROWS + 7) / 8) * 8, sc, s, &ln);
    launches += 1 + ln;
    clk(cudaMemcpyAsync(t.candK[q].p, f ? (void *)k1.p : (void *)k0, m * 8, cudaMemcpyDeviceToDevice, s), "d2d");
    k_cl_cand_meta<N><<<grid(m), CL_T, 0, s>>>(t.candK[q].as<uint64_t>(), m, q, t.candM[q].as<uint8_t>());
    launches++;
    clk(cudaGetLastError(), "candidate meta");
    sync("candidates");
  }
  inf.built = true;
  inf.seconds = cl_now() - t0;
}

CTable *CliffordContext::table(int n, CliffTableInfo &info) {
  auto it = tables.find(n);
  if (it != tables.end()) {
    info = it->second->info;
    info.built = false;
    info.seconds = 0;
    return it->second;
  }
  clk(cudaSetDevice(dev), "cudaSetDevice");
  CTable *t = new CTable;
  try {
    if (n == 1) build<1>(*t); else if (n == 2) build<2>(*t); else build<3>(*t);
  } catch (...) {
    t->release();
    delete t;
    throw;
  }
  tables[n] = t;
  info = t->info;
  return t;
}

std::vector<int> CliffordContext::dist_of(CTable &t, const std::vector<uint64_t> &x) {
  std::vector<int> r(x.size());
  if (x.empty()) return r;
  tmp.ensure(x.size() * 8); out.ensure(x.size() * 4);
  clk(cudaMemcpyAsync(tmp.p, x.data(), x.size() * 8, cudaMemcpyHostToDevice, s), "h2d");
  if (t.n == 1) k_cl_dist<1><<<grid(x.size()), CL_T, 0, s>>>(tmp.as<uint64_t>(), x.size(), t.dist.as<uint8_t>(), out.as<int>());
  else if (t.n == 2) k_cl_dist<2><<<grid(x.size()), CL_T, 0, s>>>(tmp.as<uint64_t>(), x.size(), t.dist.as<uint8_t>(), out.as<int>());
  else k_cl_dist<3><<<grid(x.size()), CL_T, 0, s>>>(tmp.as<uint64_t>(), x.size(), t.dist.as<uint8_t>(), out.as<int>());
  launches++;
  clk(cudaGetLastError(), "dist");
  clk(cudaMemcpyAsync(r.data(), out.p, x.size() * 4, cudaMemcpyDeviceToHost, s), "d2h");
  sync("dist");
  return r;
}

void CliffordContext::words(CTable &t, const std::vector<uint64_t> &x, std::vector<std::vector<int>> &w) {
  const int m = (int)x.size();
  w.assign(m, {});
  if (!m) return;
  tmp.ensure(m * 8); out.ensure((size_t)m * WORDMAX); len.ensure(m * 4);
  clk(cudaMemcpyAsync(tmp.p, x.data(), m * 8, cudaMemcpyHostToDevice, s), "h2d");
  const unsigned blocks = (unsigned)((m * 32 + CL_T - 1) / CL_T);
  if (t.n == 1) k_cl_word<1><<<blocks, CL_T, 0, s>>>(tmp.as<uint64_t>(), m, t.dist.as<uint8_t>(), out.as<int8_t>(), len.as<int>());
  else if (t.n == 2) k_cl_word<2><<<blocks, CL_T, 0, s>>>(tmp.as<uint64_t>(), m, t.dist.as<uint8_t>(), out.as<int8_t>(), len.as<int>());
  else k_cl_word<3><<<blocks, CL_T, 0, s>>>(tmp.as<uint64_t>(), m, t.dist.as<uint8_t>(), out.as<int8_t>(), len.as<int>());
  launches++;
  clk(cudaGetLastError(), "read-back");
  std::vector<int8_t> ho((size_t)m * WORDMAX);
  std::vector<int> hl(m);
  clk(cudaMemcpyAsync(ho.data(), out.p, ho.size(), cudaMemcpyDeviceToHost, s), "d2h");
  clk(cudaMemcpyAsync(hl.data(), len.p, m * 4, cudaMemcpyDeviceToHost, s), "d2h");
  sync("read-back");
  for (int i = 0; i < m; i++) {
    if (hl[i] == -1) throw std::logic_error("segment not in the table");
    if (hl[i] < 0) throw std::logic_error("path reconstruction failed");
    for (int j = 0; j < hl[i]; j++) w[i].push_back(ho[(size_t)i * WORDMAX + j]);
  }
}

// one beam step over the placements of a T gate on qubit q: the kept (cost << 32 | index) in (cost, index) order
template <int N>
void CliffordContext::beam_step(CTable &t, int q, int dagger, const std::vector<uint64_t> &left,
                                const std::vector<int> &bcost, int beam, std::vector<unsigned long long> &picked,
                                std::vector<int> &pcost) {
  constexpr int TS = 1 << (2 * N);
  const int nb = (int)left.size();
  const unsigned long long nc = t.ncand[q], tot = (unsigned long long)nb * nc * 2;
  std::vector<uint8_t> ht((size_t)nb * TS);
  for (int b = 0; b < nb; b++) Tb<N>::image_table(Tb<N>::inverse(left[b]), ht.data() + (size_t)b * TS);
  int cmin = 1 << 30, cmax = 0;
  for (int v : bcost) { cmin = std::min(cmin, v); cmax = std::max(cmax, v); }
  if (cmax + 999 > 65535) throw std::range_error("beam cost out of range");
  tabs.ensure(ht.size()); bc.ensure(nb * 4); hist.ensure(HB * 4); cost.ensure(tot * 2 + 2);
  clk(cudaMemcpyAsync(tabs.p, ht.data(), ht.size(), cudaMemcpyHostToDevice, s), "h2d");
  clk(cudaMemcpyAsync(bc.p, bcost.data(), nb * 4, cudaMemcpyHostToDevice, s), "h2d");
  clk(cudaMemsetAsync(hist.p, 0, HB * 4, s), "memset");
  k_cl_beam<N><<<grid(nc, 16), CL_T, 0, s>>>(t.candK[q].as<uint64_t>(), t.candM[q].as<uint8_t>(), nc, nb,
                                              tabs.as<uint8_t>(), bc.as<int>(), dagger, cmin, t.dist.as<uint8_t>(),
                                              cost.as<uint16_t>(), hist.as<unsigned>());
  launches++;
  clk(cudaGetLastError(), "beam step");
  const unsigned long long keep = std::min<unsigned long long>((unsigned long long)beam, tot);
  // threshold: the cost of the keep-th smallest entry
  unsigned long long nlow = 0;   // entries below the threshold
  int base = cmin, thr = -1;
  std::vector<unsigned> hh(HB);
  for (;;) {
    clk(cudaMemcpyAsync(hh.data(), hist.p, HB * 4, cudaMemcpyDeviceToHost, s), "d2h");
    sync("histogram");
    unsigned long long cum = nlow;
    int k = 0;
    for (; k < HB - 1; k++) {
      if (cum + hh[k] >= keep) break;
      cum += hh[k];
    }
    if (k < HB - 1) { thr = base + k; nlow = cum; break; }
    nlow = cum;                      // everything below base + HB - 1 is kept: zoom into the overflow bin
    base += HB - 1;
    clk(cudaMemsetAsync(hist.p, 0, HB * 4, s), "memset");
    k_cl_hist<<<grid(tot, 16), CL_T, 0, s>>>(cost.as<uint16_t>(), tot, base, hist.as<unsigned>());
    launches++;
  }
  const unsigned long long nblk = (tot + SEL_CH - 1) / SEL_CH;
  const unsigned need = (unsigned)(keep - nlow);
  below.ensure(MAXBEAM * 8 + 8); nbelow.ensure(4); blk.ensure(nblk * 4 + 4); blkoff.ensure(nblk * 4 + 4);
  part.ensure(scan_partials_words(nblk) * 4 + 4); eql.ensure(MAXBEAM * 8 + 8);
  clk(cudaMemsetAsync(nbelow.p, 0, 4, s), "memset");
  k_cl_sel_count<<<(unsigned)nblk, CL_T, 0, s>>>(cost.as<uint16_t>(), tot, thr, blk.as<uint32_t>(),
                                                  below.as<unsigned long long>(), nbelow.as<unsigned>(), MAXBEAM);
  exclusive_scan(blk.as<uint32_t>(), blkoff.as<uint32_t>(), nblk, part.as<uint32_t>(), nullptr, s);
  k_cl_sel_write<<<(unsigned)nblk, CL_T, 0, s>>>(cost.as<uint16_t>(), tot, thr, blkoff.as<uint32_t>(), need,
                                                  eql.as<unsigned long long>());
  launches += 5;
  clk(cudaGetLastError(), "beam selection");
  unsigned nbel = 0;
  std::vector<unsigned long long> hb(MAXBEAM), he(need);
  clk(cudaMemcpyAsync(&nbel, nbelow.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
  clk(cudaMemcpyAsync(hb.data(), below.p, MAXBEAM * 8, cudaMemcpyDeviceToHost, s), "d2h");
  if (need) clk(cudaMemcpyAsync(he.data(), eql.p, need * 8, cudaMemcpyDeviceToHost, s), "d2h");
  sync("beam selection");
  if (nbel != nlow) throw std::logic_error("beam selection count mismatch");
  std::vector<unsigned long long> all(hb.begin(), hb.begin() + nbel);
  all.insert(all.end(), he.begin(), he.end());
  std::sort(all.begin(), all.end());
  picked.clear(); pcost.clear();
  for (unsigned long long e : all) { picked.push_back(e & 0xffffffffULL); pcost.push_back((int)(e >> 32)); }
}

// ---------------- jobs ----------------
int parse_cliff_job(const char *text, size_t len, CliffJob &J, std::string &err) {
  J = CliffJob{};
  const char *p = text, *end = text + len;
  auto tok = [&](std::string &o) {
    while (p < end && std::isspace((unsigned char)*p)) p++;
    if (p >= end) return false;
    const char *b = p;
    while (p < end && !std::isspace((unsigned char)*p)) p++;
    o.assign(b, p);
    return true;
  };
  bool bad = false;
  auto num = [&]() -> long {
    std::string t;
    if (bad || !tok(t)) { bad = true; return 0; }
    char *e;
    const long v = std::strtol(t.c_str(), &e, 10);
    if (e == t.c_str() || *e) bad = true;
    return v;
  };
  J.n = (int)num();
  const long t = num();
  if (bad || J.n < 1 || J.n > 3 || t < 0 || t > 1000000) { err = "bad job file"; return 2; }
  J.tq.resize(t); J.td.resize(t);
  for (long i = 0; i < t && !bad; i++) {
    J.tq[i] = (int)num(); J.td[i] = (int)num();
    if (J.tq[i] < 0 || J.tq[i] >= J.n || J.td[i] < 0 || J.td[i] > 1) bad = true;
  }
  J.seg.resize(t + 1);
  for (long j = 0; j <= t && !bad; j++) {
    const long m = num();
    if (m < 0 || m > 100000000) { bad = true; break; }
    for (long i = 0; i < m && !bad; i++) {
      std::string nm;
      if (!tok(nm)) { bad = true; break; }
      int k;
      if (nm == "h") k = CG_H; else if (nm == "s") k = CG_S; else if (nm == "sdg") k = CG_SDG;
      else if (nm == "x") k = CG_X; else if (nm == "z") k = CG_Z; else if (nm == "y") k = CG_Y;
      else if (nm == "cx") k = CG_CX;
      else { err = "unknown Clifford gate " + nm; return 2; }
      const int a = (int)num();
      const int b = k == CG_CX ? (int)num() : 0;
      if (a < 0 || a >= J.n || (k == CG_CX && (b < 0 || b >= J.n || b == a))) bad = true;
      J.seg[j].push_back(k); J.seg[j].push_back(a); J.seg[j].push_back(b);
    }
  }
  if (bad) { err = "bad job file"; return 2; }
  return 0;
}

CliffordContext *clifford_context_create(int device, void *stream) { return new CliffordContext(device, stream); }
void clifford_context_destroy(CliffordContext *c) { delete c; }
size_t clifford_context_trim(CliffordContext *c) {
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->s);
  return c->trim();
}

int clifford_table(CliffordContext *c, int n, CliffTableInfo &info, std::string &err) {
  if (n < 1 || n > 3) { err = "n must be 1, 2 or 3"; return 3; }
  try {
    c->table(n, info);
    return 0;
  } catch (const std::logic_error &e) {
    err = e.what();
    return 4;
  } catch (const std::overflow_error &e) {
    err = e.what();
    return 4;
  } catch (const std::exception &e) {
    err = e.what();
    return 5;
  }
}

int cliffopt_run(CliffordContext *c, const CliffJob &J, int beam,
                 const std::function<void(int, const CliffStep &)> &on_step, CliffOptResult &res) {
  res = CliffOptResult{};
  const double t0 = cl_now();
  const long long l0 = c->launches;
  beam = std::max(1, std::min(MAXBEAM, beam));
  try {
    clk(cudaSetDevice(c->dev), "cudaSetDevice");
    const int n = J.n, t = (int)J.tq.size();
    CTable &tab = *c->table(n, res.table);
    std::vector<uint64_t> D(t + 1);
    for (int j = 0; j <= t; j++) {
      uint64_t X = h_identity(n);
      for (size_t i = 0; i < J.seg[j].size(); i += 3) X = h_gate(n, X, J.seg[j][i], J.seg[j][i + 1], J.seg[j][i + 2]);
      D[j] = X;
    }
    struct Pick { int parent, flip; uint64_t K; int qp, neg; };
    std::vector<std::vector<Pick>> hist(t);
    std::vector<uint64_t> Kprev{0};
    std::vector<int> bcost{0};
    for (int j = 0; j < t; j++) {
      const int q = J.tq[j];
      std::vector<uint64_t> left(Kprev.size());
      for (size_t b = 0; b < Kprev.size(); b++) left[b] = j == 0 ? D[j] : h_compose(n, Kprev[b], D[j]);
      std::vector<unsigned long long> picked;
      std::vector<int> pcost;
      if (n == 1) c->beam_step<1>(tab, q, J.td[j], left, bcost, beam, picked, pcost);
      else if (n == 2) c->beam_step<2>(tab, q, J.td[j], left, bcost, beam, picked, pcost);
      else c->beam_step<3>(tab, q, J.td[j], left, bcost, beam, picked, pcost);
      const unsigned long long nc = tab.ncand[q];
      const int m = (int)picked.size();
      if (m == 0) throw std::logic_error("no placement candidates");
      std::vector<unsigned long long> cidx(m);
      for (int i = 0; i < m; i++) cidx[i] = (picked[i] % (2 * nc)) >> 1;
      c->tmp.ensure(m * 8 + 8); c->pk.ensure(m * 8 + 8); c->pm.ensure(m + 8);
      clk(cudaMemcpyAsync(c->tmp.p, cidx.data(), m * 8, cudaMemcpyHostToDevice, c->s), "h2d");
      k_cl_pick<<<(m + 63) / 64, 64, 0, c->s>>>(tab.candK[q].as<uint64_t>(), tab.candM[q].as<uint8_t>(),
                                                c->tmp.as<unsigned long long>(), m, c->pk.as<uint64_t>(), c->pm.as<uint8_t>());
      c->launches++;
      std::vector<uint64_t> pK(m);
      std::vector<uint8_t> pM(m);
      clk(cudaMemcpyAsync(pK.data(), c->pk.p, m * 8, cudaMemcpyDeviceToHost, c->s), "d2h");
      clk(cudaMemcpyAsync(pM.data(), c->pm.p, m, cudaMemcpyDeviceToHost, c->s), "d2h");
      c->sync("beam pick");
      hist[j].resize(m);
      Kprev.assign(m, 0);
      bcost = pcost;
      for (int i = 0; i < m; i++) {
        const unsigned long long c2 = picked[i] % (2 * nc);
        hist[j][i] = Pick{(int)(picked[i] / (2 * nc)), (int)(c2 & 1), pK[i], pM[i] & 3, pM[i] >> 2};
        Kprev[i] = pK[i];
      }
      if (on_step) on_step(j, CliffStep{(long long)nc, pcost.empty() ? 0 : pcost[0]});
    }
    int best = 0;
    if (t > 0) {
      std::vector<uint64_t> fin(Kprev.size());
      for (size_t b = 0; b < Kprev.size(); b++) fin[b] = h_compose(n, Kprev[b], D[t]);
      const std::vector<int> fd = c->dist_of(tab, fin);
      int bestv = 1 << 30;
      for (size_t b = 0; b < fin.size(); b++) {
        const int v = bcost[b] + (fd[b] < 0 ? 999 : fd[b]);
        if (v < bestv) { bestv = v; best = (int)b; }
      }
    }
    std::vector<Pick> K(t);
    for (int j = t - 1, b = best; j >= 0; j--) { K[j] = hist[j][b]; b = hist[j][b].parent; }
    std::vector<uint64_t> Kinv(t);
    std::vector<int> dag(t);
    for (int j = 0; j < t; j++) {                       // the placed T: dagger after the sign and the flip
      const int d0 = J.td[j] ^ K[j].neg;
      Kinv[j] = h_inverse(n, K[j].K);
      if (K[j].flip) Kinv[j] = h_gate(n, Kinv[j], d0 ? CG_SDG : CG_S, K[j].qp, 0);
      dag[j] = d0 ^ K[j].flip;
    }
    std::vector<uint64_t> segs(t + 1);
    for (int j = 0; j <= t; j++) {
      uint64_t X = j > 0 ? h_compose(n, K[j - 1].K, D[j]) : D[j];
      if (j < t) X = h_compose(n, X, Kinv[j]);
      segs[j] = X;
    }
    std::vector<std::vector<int>> w;
    c->words(tab, segs, w);
    const GateSet gs = gate_set(n);
    static const char *nm[] = {"h", "s", "sdg", "x", "z", "cx", "y"};
    std::string txt;
    char line[64];
    int total = 0, before = 0;
    for (int j = 0; j <= t; j++) {
      total += (int)w[j].size();
      before += (int)(J.seg[j].size() / 3);
      for (int g : w[j]) {
        if (gs.k[g] == CG_CX) std::snprintf(line, sizeof line, "cx %d %d\n", gs.a[g], gs.b[g]);
        else std::snprintf(line, sizeof line, "%s %d\n", nm[gs.k[g]], gs.a[g]);
        txt += line;
      }
      if (j < t) { std::snprintf(line, sizeof line, "%s %d\n", dag[j] ? "tdg" : "t", K[j].qp); txt += line; }
    }
    res.clifford_gates = total;
    res.before = before;
    res.t_gates = t;
    res.text = std::move(txt);
    res.rc = 0;
  } catch (const std::range_error &e) {
    res.error = e.what();
    res.rc = 3;
  } catch (const std::logic_error &e) {
    res.error = e.what();
    res.rc = 4;
  } catch (const std::overflow_error &e) {
    res.error = e.what();
    res.rc = 4;
  } catch (const std::exception &e) {
    res.error = e.what();
    res.rc = 5;
  }
  res.launches = c->launches - l0;
  res.seconds = cl_now() - t0;
  return res.rc;
}

int clifford_dist(CliffordContext *c, int n, const uint64_t *tabp, size_t count, int *outp, std::string &err) {
  CliffTableInfo info;
  const int rc = clifford_table(c, n, info, err);
  if (rc) return rc;
  try {
    CTable &t = *c->tables[n];
    const std::vector<int> d = c->dist_of(t, std::vector<uint64_t>(tabp, tabp + count));
    std::copy(d.begin(), d.end(), outp);
    return 0;
  } catch (const std::exception &e) {
    err = e.what();
    return 5;
  }
}

int clifford_words(CliffordContext *c, int n, const uint64_t *tabp, size_t count,
                   std::vector<std::vector<int>> &words, std::string &err) {
  CliffTableInfo info;
  const int rc = clifford_table(c, n, info, err);
  if (rc) return rc;
  try {
    std::vector<std::vector<int>> w;
    c->words(*c->tables[n], std::vector<uint64_t>(tabp, tabp + count), w);
    const GateSet gs = gate_set(n);
    words.assign(count, {});
    for (size_t i = 0; i < count; i++)
      for (int g : w[i]) { words[i].push_back(gs.k[g]); words[i].push_back(gs.a[g]); words[i].push_back(gs.b[g]); }
    return 0;
  } catch (const std::logic_error &e) {
    err = e.what();
    return 4;
  } catch (const std::exception &e) {
    err = e.what();
    return 5;
  }
}

int clifford_element(CliffordContext *c, int n, const uint64_t *index, size_t count, uint64_t *tabp, std::string &err) {
  CliffTableInfo info;
  const int rc = clifford_table(c, n, info, err);
  if (rc) return rc;
  if (!count) return 0;
  try {
    CTable &t = *c->tables[n];
    c->tmp.ensure(count * 8); c->pk.ensure(count * 8);
    clk(cudaMemcpyAsync(c->tmp.p, index, count * 8, cudaMemcpyHostToDevice, c->s), "h2d");
    const unsigned g = c->grid(count);
    if (n == 1) k_cl_elem<1><<<g, CL_T, 0, c->s>>>(c->tmp.as<uint64_t>(), count, t.order, c->pk.as<uint64_t>());
    else if (n == 2) k_cl_elem<2><<<g, CL_T, 0, c->s>>>(c->tmp.as<uint64_t>(), count, t.order, c->pk.as<uint64_t>());
    else k_cl_elem<3><<<g, CL_T, 0, c->s>>>(c->tmp.as<uint64_t>(), count, t.order, c->pk.as<uint64_t>());
    c->launches++;
    clk(cudaGetLastError(), "element");
    clk(cudaMemcpyAsync(tabp, c->pk.p, count * 8, cudaMemcpyDeviceToHost, c->s), "d2h");
    c->sync("element");
    return 0;
  } catch (const std::exception &e) {
    err = e.what();
    return 5;
  }
}

}  // namespace cz
