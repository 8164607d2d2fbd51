// cheese-spec: the spec writers of the reference as one native binary.
//   cheese-spec TARGET.qasm DEPTH [--no-w3]   the gate-count spec (python -m cheese.spec, spec.py:420-438)
//   cheese-spec --tcount TARGET.qasm          the T-count spec (python -m cheese.tcount spec, tcount.py:171-174)
// State targets (--ancilla / --inputs) are refused with exit 3: the GPU search does not take them.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cheese_b200.h"

static int usage() {
  std::fprintf(stderr, "usage: cheese-spec TARGET.qasm DEPTH [--no-w3]\n       cheese-spec --tcount TARGET.qasm\n");
  return 2;
}

int main(int argc, char **argv) {
  bool tcount = false, no_w3 = false;
  std::vector<const char *> pos;
  for (int i = 1; i < argc; i++) {
    if (!std::strcmp(argv[i], "--tcount")) tcount = true;
    else if (!std::strcmp(argv[i], "--no-w3")) no_w3 = true;
    else if (!std::strcmp(argv[i], "--ancilla") || !std::strcmp(argv[i], "--inputs")) {
      std::fprintf(stderr, "state targets: not supported by this generator (the GPU search takes unitary targets)\n");
      return 3;
    } else if (argv[i][0] == '-' && argv[i][1] == '-') return usage();
    else pos.push_back(argv[i]);
  }
  if (pos.size() != (tcount ? 1u : 2u)) return usage();
  std::ifstream f(pos[0], std::ios::binary);
  if (!f) { std::fprintf(stderr, "cannot read %s\n", pos[0]); return 2; }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string q = ss.str();
  char err[256] = {0};
  size_t need = 0;
  std::vector<char> out(1 << 16);
  cz_specgen_info info;
  int rc;
  for (int attempt = 0; attempt < 2; attempt++) {
    rc = tcount ? cz_tspec_generate(q.data(), q.size(), 0, 0, nullptr, nullptr, out.data(), out.size(), &need, err,
                                    sizeof err)
                : cz_spec_generate(q.data(), q.size(), 0, 0, nullptr, nullptr, std::atoi(pos[1]), no_w3, out.data(),
                                   out.size(), &need, &info, err, sizeof err);
    if (rc != 3) break;
    out.assign(need + 1, 0);
  }
  if (rc) { std::fprintf(stderr, "%s\n", err); return 2; }
  std::fwrite(out.data(), 1, need, stdout);
  if (!tcount) {
    std::string stem = pos[0];
    const size_t sl = stem.find_last_of('/');
    if (sl != std::string::npos) stem = stem.substr(sl + 1);
    const size_t dot = stem.rfind('.');
    if (dot != std::string::npos && dot > 0) stem = stem.substr(0, dot);
    std::fprintf(stderr, "%s: %d qubits, %d candidates, W2 pairs %d, W3 triples %d\n", stem.c_str(), info.n,
                 info.candidates, info.w2_pairs, info.w3_triples);
  }
  return 0;
}
