// Shared host/device definitions of the B200 gate-count search: limits, status codes, exact Z[w] values.
//
// A residual entry is a + b w + c w^2 + d w^3 (w = e^{i pi/4}); a residual is N x N such entries over one sqrt2
// exponent k (the entries are sqrt2^k times the matrix). Limits and status codes are those of the reference
// (src/cheese.cu:53-57, 647) so per-level counts and exit codes line up one to one.
#pragma once
#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define CZ_HD __host__ __device__ __forceinline__
#else
#define CZ_HD inline
#endif

namespace cz {

constexpr int DMAX = 48;      // longest prefix
constexpr int GMAX = 64;      // most candidates
constexpr int LMAX = 8;       // largest local gate dimension
constexpr int CUTMAX = 16;    // most cuts
constexpr int SYMMAX = 12;    // qubit relabellings x conjugation at 3 qubits
constexpr int NQMAX = 3;      // qubit counts 1..3
constexpr uint32_t PRIME = 998244353u;   // p = 1 mod 8: Z[w] -> F_p for the CX bound's ranks

enum Status : uint8_t { DEAD = 0, ALIVE = 1, FOUND = 2, W2CUT = 3, W3CUT = 4, OVF = 6 };

// exit codes of the drop-in binaries (reference cheese.cu:1023-1026, 1153-1220, 1284, 1848-1891)
enum Rc : int { RC_CIRCUIT = 0, RC_PROOF = 1, RC_SPEC = 2, RC_USAGE = 3, RC_OVERFLOW = 4, RC_CUDA = 5 };

template <typename T> struct Z4 { T a, b, c, d; };
using Zw = Z4<int64_t>;

CZ_HD Zw zadd(Zw x, Zw y) { return {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; }
CZ_HD Zw zsub(Zw x, Zw y) { return {x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d}; }
// (a + b w + c w^2 + d w^3)(a' + ...) with w^4 = -1
CZ_HD Zw zmul(Zw x, Zw y) {
  return {x.a * y.a - x.b * y.d - x.c * y.c - x.d * y.b, x.a * y.b + x.b * y.a - x.c * y.d - x.d * y.c,
          x.a * y.c + x.b * y.b + x.c * y.a - x.d * y.d, x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a};
}
CZ_HD Zw zconj(Zw x) { return {x.a, -x.d, -x.c, -x.b}; }   // w -> w^7
CZ_HD bool zzero(Zw x) { return !(x.a | x.b | x.c | x.d); }
CZ_HD bool zeq(Zw x, Zw y) { return x.a == y.a && x.b == y.b && x.c == y.c && x.d == y.d; }
// divisible by sqrt2 = w - w^3 iff a = c and b = d (mod 2); the quotient
CZ_HD bool zdiv2ok(Zw x) { return !((x.a - x.c) & 1) && !((x.b - x.d) & 1); }
CZ_HD Zw zdown(Zw x) { return {(x.b - x.d) / 2, (x.a + x.c) / 2, (x.b + x.d) / 2, (x.c - x.a) / 2}; }
CZ_HD Zw zwpow(int p) {
  p &= 7;
  Zw r{0, 0, 0, 0};
  const int64_t s = p < 4 ? 1 : -1;
  switch (p & 3) { case 0: r.a = s; break; case 1: r.b = s; break; case 2: r.c = s; break; default: r.d = s; }
  return r;
}
CZ_HD bool fits32(int64_t v) { return v >= INT32_MIN && v <= INT32_MAX; }

// per-gate property bits (derived exactly from the local matrices on the host)
//  GF_CLIFFORD: maps Paulis to Paulis (the T bound of S g^-1 equals that of S)
//  GF_ONEQ:     acts on one qubit (the CX bound of S g^-1 equals that of S)
//  GF_MONAFF:   monomial with an affine permutation (the H-structure bound of S g^-1 equals that of S)
//  GF_TDIAG:    one-qubit diagonal with an odd w-power ratio (all such gates on a qubit give the same T bound:
//               they differ by a power of S, a Clifford)
//  GF_RANK2:    two-qubit gate of operator-Schmidt rank <= 2 over F_p (cx, cz: the CX bound moves by at most 1)
enum GateFlag : uint8_t { GF_CLIFFORD = 1, GF_ONEQ = 2, GF_MONAFF = 4, GF_TDIAG = 8, GF_RANK2 = 16 };

}  // namespace cz
