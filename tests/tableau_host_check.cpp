// Host check of the Clifford tableau rank and unrank (cheese_b200/csrc/cz_tableau.h): unrank is the inverse of rank
// on every rank at 1 and 2 qubits, on seeded sampled ranks at 3 qubits, and rank then unrank returns every tableau
// reached by seeded random gate words. Exit code 0 when all agree.
#include <cstdio>
#include <random>

#include "../cheese_b200/csrc/cz_tableau.h"

using namespace cz;

template <int N>
long long all_ranks() {
  long long bad = 0;
  for (long long r = 0; r < clifford_order(N); r++)
    if (Tb<N>::rank(Tb<N>::unrank((uint32_t)r)) != (uint32_t)r) bad++;
  return bad;
}

int main() {
  long long bad = all_ranks<1>() + all_ranks<2>();
  using T = Tb<3>;
  std::mt19937_64 g(20261203);
  for (int i = 0; i < 2000000; i++) {
    const uint32_t r = (uint32_t)(g() % clifford_order(3));
    if (T::rank(T::unrank(r)) != r) bad++;
  }
  for (int w = 0; w < 100000; w++) {
    uint64_t X = T::identity();
    for (int k = 0; k < 24; k++) {
      const int kind = (int)(g() % 6), a = (int)(g() % 3), b = (a + 1 + (int)(g() % 2)) % 3;
      X = T::gate(X, kind, a, b);
    }
    if (T::unrank(T::rank(X)) != X) bad++;
  }
  std::printf("mismatches: %lld\n", bad);
  return bad != 0;
}
