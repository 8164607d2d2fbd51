// Host side of the spec-file boundary: the reference's text grammar (src/cheese.cu:1149-1226, written by
// python/cheese/spec.py:356-415), the symmetry group of the candidate list (cheese.cu:1379-1429) and the exact
// per-gate properties the B200 kernels use.
#pragma once
#include <array>
#include <string>
#include <vector>

#include "cz_common.h"

namespace cz {

struct HostSpec {
  uint64_t uid = 0;                                 // unique per parse: device copies are cached by it
  int n = 0, depth = 0, standard = 0, lite = 0, tdiv = 1, G = 0, tk = 0;
  int states = 0, m = 0, gk = 0;
  std::vector<std::string> names;
  std::vector<int> gnq, gik;
  std::vector<std::array<int, 3>> gq;
  std::vector<std::array<Zw, LMAX * LMAX>> ginv;   // inverse gate local matrix / sqrt2^ik (row m, column lc)
  std::vector<uint8_t> bad2;                        // G x G
  std::vector<uint32_t> bad3;                       // bitset G^3
  std::vector<Zw> target;                           // N x N, exponent tk (state targets: the start rows)
  std::vector<Zw> goal;                             // state targets: the goal rows (N x N, exponent gk)
  std::vector<int> ginfo;                           // state targets: per pair sde, nullity, Schmidt rank per cut
  std::vector<int> cutmask, cutsize, rad, cxtable;
  std::vector<uint8_t> gflags;                      // GateFlag bits per candidate
};

// returns 0, or the reference's exit code for a bad spec (2) / unsupported qubit count (3); err: one line
int parse_spec(const char *text, size_t len, HostSpec &out, std::string &err);

struct SymGroup {
  int nsym = 0;
  std::vector<std::vector<int>> perm;      // per element: qubit map
  std::vector<uint8_t> conj, bperm;        // bperm: nsym x N basis-index maps
  std::vector<std::vector<int>> gmap;      // per element: candidate -> candidate
};
// the elements (qubit relabelling x optional complex conjugation) that map every candidate to a candidate
SymGroup sym_group(const HostSpec &hs, bool on);

// candidate index of each gate's inverse (t <-> tdg, s <-> sdg), -1 if absent
std::vector<int> inverse_gates(const HostSpec &hs);

}  // namespace cz
