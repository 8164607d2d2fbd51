// Stabiliser tableaux of n <= 3 qubit Cliffords packed in 64 bits, host and device.
//
// Layout (the reference's, clifford.cu:16-19, 46-58, kept so job semantics and outputs match): row i < n is the
// image of X_i, row n + i the image of Z_i; each row has 2n + 1 bits, x bits | z bits << n | sign << 2n, and
// stands for the Hermitian Pauli (-1)^sign i^(x.z) X^x Z^z. Applying gate G after the Clifford C conjugates
// every row.
//
// B200 choices: a gate updates all 2n rows at once with word-wide masks (one lane bit per row) instead of a loop
// over rows; composing with a fixed Clifford is a 4^n-entry row lookup table; and every group element has a
// perfect index (rank) in [0, |C_n / phase|), so the Clifford table is a plain byte array of distances indexed by
// rank (92,897,280 bytes at n = 3: L2-resident on B200) instead of a hash table of tableaux.
//
// Rank: the symplectic part is ranked by fixing one qubit at a time. With m qubits left, the image A of X_i is any
// nonzero 2m-bit vector (4^m - 1 choices) and the image B of Z_i any vector with <A, B> = 1 (2^(2m-1) choices:
// drop the bit at the pivot of the linear form <A, .>). Symplectic transvections v -> v + <v, h> h then carry
// (A, B) to the standard pair of the first remaining qubit; the other rows land in the complement, lose that
// qubit's two bits, and the next qubit is ranked the same way. The 2n sign bits are the low digits.
#pragma once
#include <cstdint>

#ifndef CZ_HD
#ifdef __CUDACC__
#define CZ_HD __host__ __device__ __forceinline__
#else
#define CZ_HD inline
#endif
#endif

namespace cz {

enum CliffGate : int { CG_H = 0, CG_S = 1, CG_SDG = 2, CG_X = 3, CG_Z = 4, CG_CX = 5, CG_Y = 6 };

CZ_HD int tb_popc(uint32_t v) {
#ifdef __CUDA_ARCH__
  return __popc(v);
#else
  return __builtin_popcount(v);
#endif
}
CZ_HD int tb_ctz(uint32_t v) {
#ifdef __CUDA_ARCH__
  return __ffs((int)v) - 1;
#else
  return __builtin_ctz(v);
#endif
}

// group order up to phase: |Sp(2n, 2)| * 4^n
constexpr long long clifford_order(int n) { return n == 1 ? 24LL : n == 2 ? 11520LL : n == 3 ? 92897280LL : 0LL; }
constexpr uint32_t sp_order(int m) { return m <= 0 ? 1u : m == 1 ? 6u : m == 2 ? 720u : 1451520u; }

template <int N>
struct Tb {
  static constexpr int RB = 2 * N + 1;                 // bits per row
  static constexpr int ROWS = 2 * N;
  static constexpr int SB = 2 * N;                     // sign bit inside a row
  static constexpr uint32_t RMASK = (1u << RB) - 1;
  static constexpr uint32_t SYM = (1u << (2 * N)) - 1; // x | z << n part of a row
  static constexpr uint32_t XM = (1u << N) - 1;
  static constexpr uint64_t lanes() {
    uint64_t m = 0;
    for (int i = 0; i < ROWS; i++) m |= 1ULL << (i * RB);
    return m;
  }
  static constexpr uint64_t L = lanes();               // bit 0 of every row
  static constexpr uint32_t BAD = 0xffffffffu;

  CZ_HD static uint32_t row(uint64_t T, int i) { return (uint32_t)(T >> (i * RB)) & RMASK; }
  CZ_HD static uint64_t with_row(uint64_t T, int i, uint32_t r) {
    const uint64_t m = (uint64_t)RMASK << (i * RB);
    return (T & ~m) | ((uint64_t)r << (i * RB));
  }
  CZ_HD static uint64_t identity() {
    uint64_t T = 0;
    for (int i = 0; i < N; i++) {
      T |= (uint64_t)(1u << i) << (i * RB);
      T |= (uint64_t)(1u << (N + i)) << ((N + i) * RB);
    }
    return T;
  }
  // gate (k, a, b) after T, on every row at once (Aaronson-Gottesman update rules)
  CZ_HD static uint64_t gate(uint64_t T, int k, int a, int b) {
    const uint64_t xa = (T >> a) & L, za = (T >> (N + a)) & L;
    switch (k) {
      case CG_H:
        T ^= (xa & za) << SB;
        return (T & ~((L << a) | (L << (N + a)))) | (za << a) | (xa << (N + a));
      case CG_S: return T ^ ((xa & za) << SB) ^ (xa << (N + a));
      case CG_SDG: return T ^ ((xa & ~za) << SB) ^ (xa << (N + a));
      case CG_X: return T ^ (za << SB);
      case CG_Z: return T ^ (xa << SB);
      case CG_Y: return T ^ ((xa ^ za) << SB);
      default: {
        const uint64_t xb = (T >> b) & L, zb = (T >> (N + b)) & L;
        return T ^ ((xa & zb & ~(xb ^ za)) << SB) ^ (xa << b) ^ (zb << (N + a));
      }
    }
  }
  CZ_HD static int inverse_kind(int k) { return k == CG_S ? CG_SDG : k == CG_SDG ? CG_S : k; }

  // image under T of +i^(x.z) X^x Z^z as a row: product of the selected rows, X rows first, phase in powers of i
  CZ_HD static uint32_t image(uint64_t T, uint32_t x, uint32_t z) {
    int k = tb_popc(x & z);
    uint32_t ax = 0, az = 0, sel = x | (z << N);
    while (sel) {
      const int q = tb_ctz(sel);
      sel &= sel - 1;
      const uint32_t w = row(T, q), bx = w & XM, bz = (w >> N) & XM;
      k += 2 * (int)(w >> SB) + tb_popc(bx & bz) + 2 * tb_popc(az & bx);
      ax ^= bx;
      az ^= bz;
    }
    return ax | (az << N) | ((uint32_t)(((k - tb_popc(ax & az)) & 3) >> 1) << SB);
  }
  // A first, then B
  CZ_HD static uint64_t compose(uint64_t A, uint64_t B) {
    uint64_t C = 0;
    for (int i = 0; i < ROWS; i++) {
      const uint32_t w = row(A, i);
      C |= (uint64_t)(image(B, w & XM, (w >> N) & XM) ^ (w & (1u << SB))) << (i * RB);
    }
    return C;
  }
  // rows of B's action on every Pauli (x, z): tab[x | z << n]
  CZ_HD static void image_table(uint64_t B, uint8_t *tab) {
    for (uint32_t v = 0; v <= SYM; v++) tab[v] = (uint8_t)image(B, v & XM, v >> N);
  }
  template <typename TAB>
  CZ_HD static uint64_t compose_tab(uint64_t A, const TAB &tab) {
    uint64_t C = 0;
    for (int i = 0; i < ROWS; i++) {
      const uint32_t w = row(A, i);
      C |= (uint64_t)((uint32_t)tab[w & SYM] ^ (w & (1u << SB))) << (i * RB);
    }
    return C;
  }
  // inverse: symplectic part from <v, b_j> = <S v, S b_j>, signs from the image of each preimage
  CZ_HD static uint64_t inverse(uint64_t C) {
    uint64_t D = 0;
    for (int i = 0; i < ROWS; i++) {
      const int wi = i < N ? i + N : i - N;            // partner of basis vector i
      uint32_t v = 0;
      for (int j = 0; j < ROWS; j++) {
        const int wj = j < N ? j + N : j - N;
        v |= ((row(C, wj) >> wi) & 1u) << j;
      }
      const uint32_t x = v & XM, z = v >> N;
      D |= (uint64_t)(x | (z << N) | (image(C, x, z) & (1u << SB))) << (i * RB);
    }
    return D;
  }

  // symplectic form of two 2m-bit vectors (x low m bits, z high m bits)
  CZ_HD static uint32_t symp(uint32_t u, uint32_t v, int m) {
    const uint32_t xm = (1u << m) - 1;
    return (uint32_t)tb_popc(((u & xm) & (v >> m)) ^ ((u >> m) & (v & xm))) & 1u;
  }
  // the perfect index of T in [0, clifford_order(N)), or BAD when T is not a valid tableau
  CZ_HD static uint32_t rank(uint64_t T) {
    uint32_t v[ROWS];
    uint32_t signs = 0;
    for (int i = 0; i < N; i++) {
      const uint32_t wx = row(T, i), wz = row(T, N + i);
      v[2 * i] = wx & SYM;
      v[2 * i + 1] = wz & SYM;
      signs |= (wx >> SB) << i;
      signs |= (wz >> SB) << (N + i);
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
      const int m = N - i;
      const uint32_t full = (1u << (2 * m)) - 1, nb = 1u << (2 * m - 1);
      const uint32_t A = v[2 * i], B = v[2 * i + 1];
      if (A == 0 || A > full || B > full || symp(A, B, m) != 1) return BAD;
      const uint32_t u = ((A >> m) | (A << m)) & full;  // <A, w> = parity(u & w)
      const int p = tb_ctz(u);
      const uint32_t ib = ((B >> (p + 1)) << p) | (B & ((1u << p) - 1));
      r = r * (full * nb) + (A - 1) * nb + ib;
      if (m == 1) break;
      const uint32_t e = 1u, f = 1u << m;
      auto tv = [&](uint32_t h) {
#pragma unroll
        for (int j = 2 * i; j < ROWS; j++) v[j] ^= symp(v[j], h, m) ? h : 0u;
      };
      if (A != e) {
        if ((A >> m) & 1u) {
          tv(A ^ e);
        } else {
          uint32_t w = f;
          if (!(A & 1u)) {                               // A lives on the other qubits: pick its lowest one
            const uint32_t supp = ((A | (A >> m)) & ((1u << m) - 1)) & ~1u;
            const int j = tb_ctz(supp);
            w ^= ((A >> j) & 1u) ? (1u << (m + j)) : (1u << j);
          }
          tv(A ^ w);
          tv(w ^ e);
        }
      }
      if (v[2 * i + 1] != f) {
        if (!(v[2 * i + 1] & 1u)) tv(e);
        tv(v[2 * i + 1] ^ f);
      }
      const uint32_t km = (1u << (m - 1)) - 1;
#pragma unroll
      for (int j = 2 * i + 2; j < ROWS; j++) {
        const uint32_t x = v[j];
        if ((x & 1u) || ((x >> m) & 1u)) return BAD;   // not in the complement: not symplectic
        v[j] = ((x >> 1) & km) | (((x >> (m + 1)) & km) << (m - 1));
      }
    }
    return r * (1u << (2 * N)) + signs;
  }
  // the element of rank r (the inverse of rank): the digits give, qubit by qubit from the last, the images A of X_i
  // and B of Z_i in the remaining space; the rows found for the later qubits are put back into that space (a zero
  // inserted for the qubit) and the rank's transvections for (A, B), which are involutions, are undone in reverse.
  CZ_HD static uint64_t unrank(uint32_t r) {
    const uint32_t signs = r & ((1u << (2 * N)) - 1);
    r >>= 2 * N;
    uint32_t d[N];
    for (int i = N - 1; i >= 0; i--) {
      const int m = N - i;
      const uint32_t R = ((1u << (2 * m)) - 1) * (1u << (2 * m - 1));
      d[i] = r % R;
      r /= R;
    }
    uint32_t v[ROWS];
    for (int i = N - 1; i >= 0; i--) {
      const int m = N - i;
      const uint32_t full = (1u << (2 * m)) - 1, nb = 1u << (2 * m - 1), e = 1u, f = 1u << m;
      const uint32_t A = d[i] / nb + 1, ib = d[i] % nb;
      const uint32_t u = ((A >> m) | (A << m)) & full;
      const int p = tb_ctz(u);
      uint32_t B = ((ib >> p) << (p + 1)) | (ib & ((1u << p) - 1));
      if (symp(A, B, m) != 1) B |= 1u << p;            // bit p of B flips <A, B>
      // the transvections the rank applies for (A, B), replayed on (A, B) to find them
      uint32_t h[4];
      int nh = 0;
      uint32_t b = B;
      auto tv = [&](uint32_t x) { b ^= symp(b, x, m) ? x : 0u; h[nh++] = x; };
      if (A != e) {
        if ((A >> m) & 1u) {
          tv(A ^ e);
        } else {
          uint32_t w = f;
          if (!(A & 1u)) {
            const uint32_t supp = ((A | (A >> m)) & ((1u << m) - 1)) & ~1u;
            const int j = tb_ctz(supp);
            w ^= ((A >> j) & 1u) ? (1u << (m + j)) : (1u << j);
          }
          tv(A ^ w);
          tv(w ^ e);
        }
      }
      if (b != f) {
        if (!(b & 1u)) tv(e);
        tv(b ^ f);
      }
      const uint32_t km = (1u << (m - 1)) - 1;
      for (int j = 2 * i + 2; j < ROWS; j++) {
        const uint32_t x = v[j];
        v[j] = ((x & km) << 1) | (((x >> (m - 1)) & km) << (m + 1));
        for (int t = nh - 1; t >= 0; t--) v[j] ^= symp(v[j], h[t], m) ? h[t] : 0u;
      }
      v[2 * i] = A;
      v[2 * i + 1] = B;
    }
    uint64_t T = 0;
    for (int i = 0; i < N; i++) {
      T |= (uint64_t)(v[2 * i] | (((signs >> i) & 1u) << SB)) << (i * RB);
      T |= (uint64_t)(v[2 * i + 1] | (((signs >> (N + i)) & 1u) << SB)) << ((N + i) * RB);
    }
    return T;
  }
};

}  // namespace cz
