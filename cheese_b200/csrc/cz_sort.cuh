// Device primitives of the frontier dedupe: exclusive scan and a stable LSD radix sort of (u64 key, u32 value)
// pairs over a chosen bit range, 8-bit digits. Reduce-then-scan per pass: per-tile digit histograms (digit-major,
// so one exclusive scan gives every tile's output base per digit), then a stable scatter that ranks keys inside
// the tile with warp match + per-warp digit counts in shared memory. All launches go to the caller's stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace cz {
namespace {   // each translation unit that sorts gets its own copy of these kernels

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 16;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;   // keys per tile
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

// ---------------- exclusive scan of u32 ----------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
// block-wide exclusive scan of one value per thread (blockDim.x == SCAN_THREADS); returns the block total too
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t &total) {
  __shared__ uint32_t ws[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v, lane);
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    const uint32_t x = lane < SCAN_THREADS / 32 ? ws[lane] : 0;
    const uint32_t xi = warp_incl_scan(x, lane);
    if (lane < SCAN_THREADS / 32) ws[lane] = xi - x;
  }
  __syncthreads();
  const uint32_t r = ws[w] + inc - v;
  total = 0;
  __shared__ uint32_t tot;
  if (threadIdx.x == SCAN_THREADS - 1) tot = r + v;
  __syncthreads();
  total = tot;
  __syncthreads();
  return r;
}

__global__ void k_scan_partials(const uint32_t *in, size_t n, uint32_t *partials) {
  const size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
  uint32_t s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++) {
    const size_t j = base + (size_t)i * SCAN_THREADS + threadIdx.x;
    if (j < n) s += in[j];
  }
  uint32_t total;
  (void)block_excl_scan(s, total);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}
// one block: exclusive scan of the partials in place, grand total to *total
__global__ void k_scan_single(uint32_t *p, size_t np, uint32_t *total) {
  uint32_t carry = 0;
  for (size_t b = 0; b < np; b += SCAN_THREADS) {
    const size_t j = b + threadIdx.x;
    const uint32_t v = j < np ? p[j] : 0;
    uint32_t t;
    const uint32_t e = block_excl_scan(v, t);
    if (j < np) p[j] = carry + e;
    carry += t;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}
__global__ void k_scan_apply(const uint32_t *in, size_t n, const uint32_t *partials, uint32_t *out) {
  const size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
  // each thread owns SCAN_ITEMS consecutive values
  uint32_t v[SCAN_ITEMS], s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++) {
    const size_t j = base + (size_t)threadIdx.x * SCAN_ITEMS + i;
    v[i] = j < n ? in[j] : 0;
    s += v[i];
  }
  uint32_t total;
  uint32_t e = block_excl_scan(s, total) + partials[blockIdx.x];
  for (int i = 0; i < SCAN_ITEMS; i++) {
    const size_t j = base + (size_t)threadIdx.x * SCAN_ITEMS + i;
    if (j < n) out[j] = e;
    e += v[i];
  }
}

// partials: >= ceil(n / SCAN_CHUNK) + 1 words; in may equal out
inline void exclusive_scan(const uint32_t *in, uint32_t *out, size_t n, uint32_t *partials, uint32_t *total,
                           cudaStream_t s) {
  const size_t nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  if (nb == 0) { if (total) cudaMemsetAsync(total, 0, 4, s); return; }
  k_scan_partials<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, partials);
  k_scan_single<<<1, SCAN_THREADS, 0, s>>>(partials, nb, total);
  k_scan_apply<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, partials, out);
}
inline size_t scan_partials_words(size_t n) { return (n + SCAN_CHUNK - 1) / SCAN_CHUNK + 1; }

// ---------------- radix sort ----------------
__global__ void k_digit_hist(const uint64_t *keys, size_t n, int shift, uint32_t *hist, uint32_t ntiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * SORT_TILE;
  for (int i = 0; i < SORT_ITEMS; i++) {
    const size_t j = base + (size_t)i * SORT_THREADS + threadIdx.x;
    if (j < n) atomicAdd(&h[(keys[j] >> shift) & 255], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(SORT_THREADS) k_digit_scatter(const uint64_t *kin, const uint32_t *vin, uint64_t *kout,
                                                                uint32_t *vout, size_t n, int shift,
                                                                const uint32_t *offs, uint32_t ntiles) {
  constexpr int NW = SORT_THREADS / 32;
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[NW][256];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  base[tid] = offs[(size_t)tid * ntiles + blockIdx.x];
  for (int x = 0; x < NW; x++) wcnt[x][tid] = 0;
  __syncthreads();
  const size_t start = (size_t)blockIdx.x * SORT_TILE;
  const unsigned lt = (1u << lane) - 1;
  for (int r = 0; r < SORT_ITEMS; r++) {
    const size_t i = start + (size_t)r * SORT_THREADS + tid;
    const bool valid = i < n;
    uint64_t key = 0;
    uint32_t val = 0;
    int d = 256;
    if (valid) { key = kin[i]; val = vin[i]; d = (int)((key >> shift) & 255); }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int lrank = __popc(peers & lt);
    const bool leader = lane == __ffs(peers) - 1;
    if (valid && leader) wcnt[w][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (int x = 0; x < w; x++) pre += wcnt[x][d];
      const uint32_t pos = base[d] + pre + lrank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    if (valid && leader) { atomicAdd(&base[d], (uint32_t)__popc(peers)); wcnt[w][d] = 0; }
    __syncthreads();
  }
}

struct SortScratch {
  uint32_t *hist = nullptr;       // 256 * ntiles
  uint32_t *partials = nullptr;   // scan partials
  size_t cap_hist = 0, cap_part = 0;
};
inline size_t sort_hist_words(size_t n) { return 256 * ((n + SORT_TILE - 1) / SORT_TILE); }

// sorts (k0, v0) by bits [lo, hi) of the key, stable; uses (k1, v1) as the other buffer. Returns true when the
// result ended in (k1, v1). Counts launches into *launches.
inline bool radix_sort(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, size_t n, int lo, int hi,
                       const SortScratch &sc, cudaStream_t s, int *launches) {
  if (n <= 1 || hi <= lo) return false;
  const uint32_t ntiles = (uint32_t)((n + SORT_TILE - 1) / SORT_TILE);
  bool flip = false;
  for (int shift = lo; shift < hi; shift += 8) {
    const uint64_t *ki = flip ? k1 : k0;
    const uint32_t *vi = flip ? v1 : v0;
    uint64_t *ko = flip ? k0 : k1;
    uint32_t *vo = flip ? v0 : v1;
    k_digit_hist<<<ntiles, SORT_THREADS, 0, s>>>(ki, n, shift, sc.hist, ntiles);
    exclusive_scan(sc.hist, sc.hist, (size_t)256 * ntiles, sc.partials, nullptr, s);
    k_digit_scatter<<<ntiles, SORT_THREADS, 0, s>>>(ki, vi, ko, vo, n, shift, sc.hist, ntiles);
    if (launches) *launches += 5;
    flip = !flip;
  }
  return flip;
}

}  // namespace
}  // namespace cz
