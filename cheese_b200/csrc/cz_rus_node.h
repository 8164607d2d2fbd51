// Per-node arithmetic of the RUS T-count search, shared by the sm_100a kernels (cz_rus.cu) and host-compiled checks:
// one node is one 16 x 4 Pauli transfer matrix (x + y sqrt2) / sqrt2^e held by one thread.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define CZ_RUS_FN __host__ __device__ __forceinline__
#else
#define CZ_RUS_FN inline
#endif

namespace cz {
namespace rus {

constexpr int NR = 16, NC = 4, NE = NR * NC;
constexpr int NCL = 11520;        // two-qubit Cliffords mod phase
constexpr int NG = 15;            // rotations per level
constexpr int MAXT = 32;          // deepest peel sequence
constexpr int MS = 132;           // ints per stored matrix: x[64], y[64], e, 3 pad
constexpr int RT = 128;           // threads per CTA

struct RDev {
  const int8_t *tr, *ts;          // 15 x 16
  const uint8_t *perm;            // NCL x 16
  const int8_t *sign;             // NCL x 16
  const int *bygen;               // 2^20: Clifford index from the images of X_q0, Z_q0, X_q1, Z_q1, or -1
};
struct RHist {
  const uint32_t *par[MAXT + 1];
  const uint8_t *gat[MAXT + 1];
};
struct RM { int x[NE], y[NE], e; };

CZ_RUS_FN void rm_load(RM &M, const int *src) {
  for (int i = 0; i < NE; i++) { M.x[i] = src[i]; M.y[i] = src[NE + i]; }
  M.e = src[2 * NE];
}
CZ_RUS_FN void rm_store(const RM &M, int *dst) {
  for (int i = 0; i < NE; i++) { dst[i] = M.x[i]; dst[NE + i] = M.y[i]; }
  dst[2 * NE] = M.e;
}

// B = R(P_p)^-1 A, normalised (rus.cu:86-118): a row that commutes with P_p is multiplied by sqrt2
// ((x + y s) s = 2y + x s), an anticommuting row a becomes row a - s row r; then (x + y s) / s = y + (x / 2) s while
// every x is even and e > 0. Returns true when a value left int32.
CZ_RUS_FN bool rm_peel(const RM &A, RM &B, int p, const RDev &sp) {
  bool bad = false;
  const int8_t *trp = sp.tr + (p - 1) * NR, *tsp = sp.ts + (p - 1) * NR;
  for (int a = 0; a < NR; a++) {
    const int r = trp[a], s = tsp[a];
    for (int c = 0; c < NC; c++) {
      const long long ox = A.x[a * NC + c], oy = A.y[a * NC + c];
      long long vx, vy;
      if (r < 0) { vx = 2 * oy; vy = ox; }
      else { vx = ox - (long long)s * A.x[r * NC + c]; vy = oy - (long long)s * A.y[r * NC + c]; }
      bad |= vx > INT32_MAX || vx < INT32_MIN || vy > INT32_MAX || vy < INT32_MIN;
      B.x[a * NC + c] = (int)vx;
      B.y[a * NC + c] = (int)vy;
    }
  }
  B.e = A.e + 1;
  while (B.e > 0) {
    bool even = true;
    for (int i = 0; i < NE; i++) even &= !(B.x[i] & 1);
    if (!even) break;
    for (int i = 0; i < NE; i++) { const int x = B.x[i]; B.x[i] = B.y[i]; B.y[i] = x / 2; }
    B.e--;
  }
  return bad;
}

CZ_RUS_FN uint64_t fmix64(uint64_t h) {   // the 64-bit finaliser of MurmurHash3
  h ^= h >> 33; h *= 0xff51afd7ed558ccdULL;
  h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ULL;
  h ^= h >> 33;
  return h;
}
// left-coset key: exponent, sign-normalised row 0 and the sum of hashes of the sign-normalised rows 1..15 (a left
// Clifford fixes row 0 and permutes the other rows with signs, so the key is the same over a coset)
CZ_RUS_FN void rm_key(const RM &M, uint64_t &k1, uint64_t &k2) {
  uint64_t s1 = 0, s2 = 0, z1 = 0, z2 = 0;
  for (int a = 0; a < NR; a++) {
    int s = 0;
    for (int c = 0; c < NC && !s; c++) {
      const int x = M.x[a * NC + c], y = M.y[a * NC + c];
      s = x ? (x > 0 ? 1 : -1) : (y ? (y > 0 ? 1 : -1) : 0);
    }
    const uint32_t neg = s < 0 ? 0xffffffffu : 0u;
    uint64_t r1 = 0x243f6a8885a308d3ULL, r2 = 0x13198a2e03707344ULL;
    for (int c = 0; c < NC; c++) {
      const uint32_t ux = ((uint32_t)M.x[a * NC + c] ^ neg) - neg, uy = ((uint32_t)M.y[a * NC + c] ^ neg) - neg;
      const uint64_t v = ((uint64_t)ux << 32) | uy;
      r1 = fmix64(r1 ^ (v + (uint64_t)(c + 1) * 0x9e3779b97f4a7c15ULL));
      r2 = fmix64(r2 + (v ^ (uint64_t)(c + 1) * 0xc2b2ae3d27d4eb4fULL));
    }
    if (a == 0) { z1 = r1; z2 = r2; }
    else { s1 += r1; s2 += r2; }
  }
  k1 = fmix64(s1 ^ fmix64(z1 + (uint64_t)(uint32_t)M.e * 0x9e3779b97f4a7c15ULL));
  k2 = fmix64(s2 + fmix64(z2 ^ ((uint64_t)(uint32_t)M.e << 17)));
}

CZ_RUS_FN bool row_eq(const RM &A, int ra, int s, const RM &B, int rb) {   // s A[ra] == B[rb]
  for (int c = 0; c < NC; c++)
    if (s * A.x[ra * NC + c] != B.x[rb * NC + c] || s * A.y[ra * NC + c] != B.y[rb * NC + c]) return false;
  return true;
}
// sign of a row's first nonzero entry (x before y, column by column); 0 for a zero row. When s A[ra] == B[rb] the
// rows' first nonzero entries sit at the same place, so s is the product of the two rows' signs.
CZ_RUS_FN int row_lead_sign(const RM &A, int r) {
  for (int c = 0; c < NC; c++) {
    if (A.x[r * NC + c]) return A.x[r * NC + c] > 0 ? 1 : -1;
    if (A.y[r * NC + c]) return A.y[r * NC + c] > 0 ? 1 : -1;
  }
  return 0;
}
CZ_RUS_FN int low_bit(uint32_t m) {
#ifdef __CUDA_ARCH__
  return __ffs((int)m) - 1;
#else
  return __builtin_ctz(m);
#endif
}
// The Clifford c with B = C_c A (B[a] = s_c(a) A[pi_c(a)] for every row a), else -1; exact. A Clifford is named by
// its images of the generator rows X_q0, Z_q0, X_q1, Z_q1 (rows 1, 3, 4, 12), each an image row and a sign: 5 bits
// (row << 1 | minus), the key of sp.bygen (-1 for images no Clifford has). The possible images of each generator are
// read off A once, as a mask over (row, sign) with bit 2 (row - 1) + minus, by one comparison per row with the signs
// taken from the rows' leading entries. The Cliffords those masks allow are tried in ascending order of (image of
// X_q0, of Z_q0, of X_q1, of Z_q1), each image ordered by row and then + before -, and the first that maps every
// row is returned: when A repeats a row up to sign several Cliffords qualify, and this order picks the reference's.
CZ_RUS_FN int rm_equiv(const RM &A, const RM &B, const RDev &sp) {
  if (A.e != B.e) return -1;
  const int gen[4] = {1, 3, 4, 12};
  int la[NR];                                   // A's row signs, read once for the four generators
  for (int r = 1; r < NR; r++) la[r] = row_lead_sign(A, r);
  uint32_t mask[4];
  for (int g = 0; g < 4; g++) {
    const int sb = row_lead_sign(B, gen[g]);
    uint32_t m = 0;
    for (int r = 1; r < NR; r++) {
      const int sa = la[r];
      if (!sa && !sb) m |= 3u << (2 * (r - 1));                        // zero rows: equal with either sign
      else if (sa && sb && row_eq(A, r, sa * sb, B, gen[g])) m |= 1u << (2 * (r - 1) + (sa * sb < 0));
    }
    if (!m) return -1;
    mask[g] = m;
  }
  for (uint32_t m0 = mask[0]; m0; m0 &= m0 - 1)
    for (uint32_t m1 = mask[1]; m1; m1 &= m1 - 1)
      for (uint32_t m2 = mask[2]; m2; m2 &= m2 - 1)
        for (uint32_t m3 = mask[3]; m3; m3 &= m3 - 1) {
          int key = 0;
          const uint32_t ms[4] = {m0, m1, m2, m3};
          for (int g = 0; g < 4; g++) {
            const int b = low_bit(ms[g]);
            key |= ((((b >> 1) + 1) << 1) | (b & 1)) << (5 * g);
          }
          const int c = sp.bygen[key];
          if (c < 0) continue;
          bool ok = true;
          for (int a = 0; ok && a < NR; a++) ok = row_eq(A, sp.perm[c * NR + a], sp.sign[c * NR + a], B, a);
          if (ok) return c;
        }
  return -1;
}

// node i of level t of a tree rebuilt from its root (roots: MS ints each) along its peel path; result in M
CZ_RUS_FN bool rm_replay(RM &M, RM &W, const int *roots, const RHist &H, int t, uint32_t i, const RDev &sp) {
  uint8_t seq[MAXT];
  for (int l = t; l >= 1; l--) { seq[l - 1] = H.gat[l][i]; i = H.par[l][i]; }
  rm_load(M, roots + (size_t)i * MS);
  bool bad = false;
  for (int l = 0; l < t; l += 2) {
    bad |= rm_peel(M, W, seq[l], sp);
    if (l + 1 < t) bad |= rm_peel(W, M, seq[l + 1], sp);
    else M = W;
  }
  return bad;
}

}  // namespace rus
}  // namespace cz
