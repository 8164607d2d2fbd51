// Device primitives of the frontier dedupe: exclusive scan and a stable LSD radix sort of (u64 key, u32 value)
// pairs over a chosen bit range, 8-bit digits, one launch per digit pass (see radix_sort). All launches go to the
// caller's stream.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
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
// Stable LSD radix sort of (u64 key, u32 value) pairs by bits [lo, hi) of the key, 8-bit digits, one launch per
// digit pass:
//  * k_sort_upsweep reads the keys once and counts every pass's digits (global histograms);
//  * k_sort_onesweep, per pass, takes tiles of OS_TILE keys in the order of an atomic ticket. A tile counts its
//    digits, publishes them, and finds the keys of earlier tiles per digit by looking back over their published
//    words (decoupled look-back: an earlier tile's word is either its own count or, once its look-back is done, the
//    inclusive prefix; walking back stops at the first prefix). Its keys are ranked stably without block barriers
//    between rounds: each warp holds a contiguous eighth of the tile and ranks its keys among its own (warp match,
//    one counter update per digit group), a scan over the warps' counts per digit joins the eighths, and the keys are
//    placed in shared memory in digit order and written out so that neighbouring threads write neighbouring
//    addresses.
// A tile waits only for tiles with smaller tickets, whose blocks are already running, so the waits end; every wait
// is still bounded (OS_SPIN_MAX polls). Should one give up, the tile counts the earlier tiles' digits itself from
// the input (slow, still exact) and the sort records it (sort_failed), so a result is never wrong and nothing hangs.
// Status words: tag (pass + 1, 4 bits) | state (2 bits: 1 count, 2 prefix) | value (58 bits); the scratch is
// cleared once per sort, and the tag tells one pass's words from the previous pass's.
constexpr int OS_THREADS = 256;
constexpr int OS_ITEMS = 8;
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;     // keys per tile
constexpr int OS_MAXPASS = 8;
constexpr long long OS_SPIN_MAX = 1LL << 26;
constexpr size_t OS_HEAD_WORDS = 256 * OS_MAXPASS + 16;   // digit counts per pass, tickets per pass, error flag
constexpr unsigned long long OS_VALUE = (1ULL << 58) - 1;
constexpr size_t OS_SCAN_MIN = (size_t)1 << 22;     // sorts of at least this many keys take the scan path

inline size_t sort_tiles(size_t n) { return (n + OS_TILE - 1) / OS_TILE; }
// 32-bit words of sort scratch for n keys (header + one 64-bit status word per tile and digit)
inline size_t sort_hist_words(size_t n) { return OS_HEAD_WORDS + 2 * 256 * (sort_tiles(n) + 1); }

__global__ void __launch_bounds__(256) k_sort_upsweep(const uint64_t *keys, size_t n, int lo, int npass,
                                                       uint32_t *counts) {
  __shared__ uint32_t h[OS_MAXPASS][256];
  for (int p = 0; p < npass; p++) h[p][threadIdx.x] = 0;
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    for (int p = 0; p < npass; p++) atomicAdd(&h[p][(k >> (lo + 8 * p)) & 255], 1u);
  }
  __syncthreads();
  for (int p = 0; p < npass; p++)
    if (h[p][threadIdx.x]) atomicAdd(&counts[p * 256 + threadIdx.x], h[p][threadIdx.x]);
}

// per-tile digit counts of one pass, digit-major (hist[d * ntiles + tile]), tiles of OS_TILE keys
__global__ void __launch_bounds__(256) k_sort_tilehist(const uint64_t *keys, size_t n, int shift, uint32_t *hist,
                                                       uint32_t ntiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * OS_TILE;
  for (int i = threadIdx.x; i < OS_TILE; i += 256) {
    const size_t j = base + i;
    if (j < n) atomicAdd(&h[(keys[j] >> shift) & 255], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__device__ __forceinline__ unsigned long long os_load(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}
__device__ __forceinline__ void os_store(unsigned long long *p, unsigned long long v) {
  *(volatile unsigned long long *)p = v;
}
// exclusive scan of one u32 per thread over the 256 threads of the block
__device__ __forceinline__ uint32_t os_block_scan(uint32_t v, uint32_t *ws) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = warp_incl_scan(v, lane);
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    const uint32_t x = lane < OS_THREADS / 32 ? ws[lane] : 0;
    const uint32_t xi = warp_incl_scan(x, lane);
    if (lane < OS_THREADS / 32) ws[lane] = xi - x;
  }
  __syncthreads();
  const uint32_t r = ws[w] + inc - v;
  __syncthreads();
  return r;
}

template <bool LOOKBACK>
__global__ void __launch_bounds__(OS_THREADS, 4) k_sort_onesweep(const uint64_t *kin, const uint32_t *vin, uint64_t *kout,
                                                               uint32_t *vout, size_t n, int shift, int pass,
                                                               uint32_t *head, unsigned long long *status,
                                                               unsigned *err, const uint32_t *offs, uint32_t ntiles) {
  constexpr int NW = OS_THREADS / 32;
  __shared__ uint64_t sk[OS_TILE];
  __shared__ uint32_t sv[OS_TILE];
  __shared__ uint32_t lex[256], run[256], wcnt[NW][256], ws[NW];
  __shared__ unsigned long long gbase[256];
  __shared__ unsigned ticket;
  __shared__ int fallback;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t *counts = head + pass * 256;
  unsigned *tickets = head + 256 * OS_MAXPASS;
  if (tid == 0) { ticket = LOOKBACK ? atomicAdd(&tickets[pass], 1u) : blockIdx.x; fallback = 0; }
  for (int x = 0; x < NW; x++) wcnt[x][tid] = 0;
  __syncthreads();
  const size_t tile = ticket, start = tile * OS_TILE;
  const unsigned long long tag = (unsigned long long)(pass + 1) << 60;
  // warp w holds tile positions [w * 32 * OS_ITEMS, (w + 1) * 32 * OS_ITEMS), round r lane l the position
  // w * 32 * OS_ITEMS + 32 r + l: input order is (warp, round, lane)
  uint64_t key[OS_ITEMS];
  uint32_t val[OS_ITEMS], wr[OS_ITEMS];
  int dig[OS_ITEMS];
#pragma unroll
  for (int r = 0; r < OS_ITEMS; r++) {
    const size_t i = start + (size_t)w * 32 * OS_ITEMS + 32 * r + lane;
    dig[r] = 256;
    if (i < n) {
      key[r] = kin[i];
      val[r] = vin[i];
      dig[r] = (int)((key[r] >> shift) & 255);
    }
  }
  // each warp's digit counts and every key's rank among its warp's keys of the same digit (earlier rounds, then
  // lower lanes): one leader per digit group updates the warp's counter, so no atomics and no block barrier
  const unsigned lt = (1u << lane) - 1;
#pragma unroll
  for (int r = 0; r < OS_ITEMS; r++) {
    const int d = dig[r];
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (d < 256 && lane == leader) { old = wcnt[w][d]; wcnt[w][d] = old + (uint32_t)__popc(peers); }
    old = __shfl_sync(0xffffffffu, old, leader);
    wr[r] = old + (uint32_t)__popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // per digit tid: the warps' counts become exclusive prefixes (earlier warps' keys of the digit); the tile's count
  uint32_t mine = 0;
#pragma unroll
  for (int x = 0; x < NW; x++) {
    const uint32_t t = wcnt[x][tid];
    wcnt[x][tid] = mine;
    mine += t;
  }
  if constexpr (LOOKBACK) {
    // this tile's count of digit tid: publish it, then add up the earlier tiles' counts by looking back
    unsigned long long *st = status + tile * 256 + tid;
    unsigned long long before = 0;
    bool ok = true;
    if (tile == 0) {
      os_store(st, tag | (2ULL << 58) | mine);
    } else {
      os_store(st, tag | (1ULL << 58) | mine);
      for (long long j = (long long)tile - 1; j >= 0 && ok; j--) {
        const unsigned long long *q = status + (size_t)j * 256 + tid;
        unsigned long long v = os_load(q);
        long long spins = 0;
        while ((v >> 60) != (tag >> 60) && ++spins < OS_SPIN_MAX) {
          __nanosleep(64);
          v = os_load(q);
        }
        if ((v >> 60) != (tag >> 60)) { ok = false; break; }
        before += v & OS_VALUE;
        if (((v >> 58) & 3) == 2) break;
      }
    }
    if (!ok) { atomicOr(err, 1u); fallback = 1; }
    __syncthreads();
    if (fallback) {                               // a wait gave up: count the earlier tiles' digits directly
      run[tid] = 0;
      __syncthreads();
      for (size_t i = tid; i < start; i += OS_THREADS) atomicAdd(&run[(kin[i] >> shift) & 255], 1u);
      __syncthreads();
      before = run[tid];
      __syncthreads();
    }
    if (tile != 0) os_store(st, tag | (2ULL << 58) | ((before + mine) & OS_VALUE));
    // output base of digit tid for this tile: keys of smaller digits (all tiles) + this digit's in earlier tiles
    const uint32_t dex = os_block_scan(counts[tid], ws);
    gbase[tid] = (unsigned long long)dex + before;
  } else {
    gbase[tid] = offs[(size_t)tid * ntiles + tile];   // the scanned digit-major tile histograms
  }
  lex[tid] = os_block_scan(mine, ws);             // keys of smaller digits in this tile
  __syncthreads();
  // each key to its place in the tile's digit order: smaller digits, earlier warps' keys of its digit, its rank
#pragma unroll
  for (int r = 0; r < OS_ITEMS; r++) {
    const int d = dig[r];
    if (d < 256) {
      const uint32_t pos = lex[d] + wcnt[w][d] + wr[r];
      sk[pos] = key[r];
      sv[pos] = val[r];
    }
  }
  __syncthreads();
  const int tn = (int)(n - start < (size_t)OS_TILE ? n - start : (size_t)OS_TILE);
  for (int i = tid; i < tn; i += OS_THREADS) {
    const uint64_t k = sk[i];
    const int d = (int)((k >> shift) & 255);
    const unsigned long long pos = gbase[d] + (unsigned long long)(i - (int)lex[d]);
    if (pos < n) {                                // always, for a consistent input (nothing else writes the keys)
      kout[pos] = k;
      vout[pos] = sv[i];
    } else {
      atomicOr(err, 2u);
    }
  }
}

struct SortScratch {
  uint32_t *hist = nullptr;       // sort scratch: sort_hist_words(n) words
  uint32_t *partials = nullptr;   // scan partials: scan_partials_words(sort_hist_words(n)) words (large sorts)
  size_t cap_hist = 0, cap_part = 0;
  uint32_t *err = nullptr;        // where a failed look-back is flagged (nullptr: the scratch's own word)
};

// sorts (k0, v0) by bits [lo, hi) of the key (hi - lo a multiple of 8, at most 64), stable; uses (k1, v1) as the
// other buffer. Returns true when the result ended in (k1, v1). Counts launches into *launches.
inline bool radix_sort(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, size_t n, int lo, int hi,
                       const SortScratch &sc, cudaStream_t s, int *launches) {
  if (n <= 1 || hi <= lo) return false;
  const int npass = (hi - lo + 7) / 8;
  const size_t ntiles = sort_tiles(n);
  const bool scan = n >= OS_SCAN_MIN && sc.partials && sc.cap_part >= scan_partials_words(256 * ntiles);
  cudaMemsetAsync(sc.hist, 0, (OS_HEAD_WORDS + (scan ? 0 : 2 * 256 * ntiles)) * 4, s);
  unsigned long long *status = (unsigned long long *)(sc.hist + OS_HEAD_WORDS);
  uint32_t *offs = sc.hist + OS_HEAD_WORDS;                  // scan path: the digit-major tile histograms
  unsigned *err = sc.err ? sc.err : sc.hist + 256 * OS_MAXPASS + OS_MAXPASS;
  if (!scan) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned ub = (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)nsm * 8));
    k_sort_upsweep<<<ub, 256, 0, s>>>(k0, n, lo, npass, sc.hist);
  }
  bool flip = false;
  for (int p = 0; p < npass; p++) {
    const uint64_t *ki = flip ? k1 : k0;
    const uint32_t *vi = flip ? v1 : v0;
    uint64_t *ko = flip ? k0 : k1;
    uint32_t *vo = flip ? v0 : v1;
    if (scan) {
      k_sort_tilehist<<<(unsigned)ntiles, 256, 0, s>>>(ki, n, lo + 8 * p, offs, (uint32_t)ntiles);
      exclusive_scan(offs, offs, 256 * ntiles, sc.partials, nullptr, s);
      k_sort_onesweep<false><<<(unsigned)ntiles, OS_THREADS, 0, s>>>(ki, vi, ko, vo, n, lo + 8 * p, p, sc.hist, status,
                                                                   err, offs, (uint32_t)ntiles);
    } else {
      k_sort_onesweep<true><<<(unsigned)ntiles, OS_THREADS, 0, s>>>(ki, vi, ko, vo, n, lo + 8 * p, p, sc.hist, status,
                                                                  err, nullptr, 0);
    }
    flip = !flip;
  }
  if (launches) *launches += scan ? 5 * npass : 1 + npass;
  return flip;
}
// the last sort's flags on this scratch (synchronises the stream): bit 0, a look-back wait gave up (the result is
// exact all the same: the tile counted its predecessors' digits itself); bit 1, a scatter position fell outside the
// array (the keys changed while the sort ran; those writes were skipped and the result is not to be used)
inline uint32_t sort_failed(const SortScratch &sc, cudaStream_t s) {
  uint32_t e = 0;
  cudaMemcpyAsync(&e, sc.err ? sc.err : sc.hist + 256 * OS_MAXPASS + OS_MAXPASS, 4, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return e;
}

}  // namespace
}  // namespace cz
