// cheese-spec: the spec writers of the reference as one native binary.
//   cheese-spec TARGET.qasm DEPTH [--no-w3] [--ancilla Q ..] [--inputs A,B,..]
//                                             the gate-count spec (python -m cheese.spec, spec.py:427-438); with
//                                             --inputs (or --ancilla: every basis state with those qubits 0) the
//                                             state-target spec (spec.py:418-424)
//   cheese-spec --tcount TARGET.qasm          the T-count spec (python -m cheese.tcount spec, tcount.py:171-174)
//   cheese-spec --rus TARGET.qasm [--outcome K]
//                                             the RUS spec (python -m cheese.rus spec, rus.py:334-342)
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cheese_b200.h"

static int usage() {
  std::fprintf(stderr, "usage: cheese-spec TARGET.qasm DEPTH [--no-w3] [--ancilla Q ..] [--inputs A,B,..]\n"
                       "       cheese-spec --tcount TARGET.qasm\n"
                       "       cheese-spec --rus TARGET.qasm [--outcome K]\n");
  return 2;
}

int main(int argc, char **argv) {
  bool tcount = false, rus = false, no_w3 = false, have_inputs = false;
  int outcome = -1;
  std::vector<const char *> pos;
  std::vector<int> ancilla, inputs;
  auto integer = [](const char *a, int &v) {
    char *e = nullptr;
    const long x = std::strtol(a, &e, 10);
    if (!*a || *e || x < INT_MIN || x > INT_MAX) return false;
    v = (int)x;
    return true;
  };
  for (int i = 1; i < argc; i++) {
    int v;
    if (!std::strcmp(argv[i], "--tcount")) tcount = true;
    else if (!std::strcmp(argv[i], "--rus")) rus = true;
    else if (!std::strcmp(argv[i], "--outcome")) {
      if (++i >= argc || !integer(argv[i], outcome)) return usage();
    }
    else if (!std::strcmp(argv[i], "--no-w3")) no_w3 = true;
    else if (!std::strcmp(argv[i], "--ancilla")) {      // one or more qubit indices
      const size_t before = ancilla.size();
      while (i + 1 < argc && integer(argv[i + 1], v)) { ancilla.push_back(v); i++; }
      if (ancilla.size() == before) return usage();
    } else if (!std::strcmp(argv[i], "--inputs")) {     // comma-separated basis states
      if (++i >= argc) return usage();
      inputs.clear();
      const std::string list = argv[i];
      for (size_t a = 0; !list.empty() && a <= list.size();) {
        size_t b = list.find(',', a);
        if (b == std::string::npos) b = list.size();
        if (!integer(list.substr(a, b - a).c_str(), v)) return usage();
        inputs.push_back(v);
        a = b + 1;
      }
      have_inputs = !inputs.empty();
    } else if (argv[i][0] == '-' && argv[i][1] == '-') return usage();
    else pos.push_back(argv[i]);
  }
  if (tcount && rus) return usage();
  if (pos.size() != (tcount || rus ? 1u : 2u)) return usage();
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
  if (!tcount && !have_inputs && !ancilla.empty()) {
    // every basis state with the ancilla qubits 0 (spec.py state_inputs); the qubit count comes from the circuit
    long long mask = 0;
    for (int a : ancilla) {
      if (a < 0 || a > 61) { std::fprintf(stderr, "ancilla qubit %d out of range\n", a); return 2; }
      mask += 1LL << a;
    }
    rc = cz_spec_generate(q.data(), q.size(), 0, 0, nullptr, nullptr, 1, no_w3, nullptr, 0, &need, &info, err,
                          sizeof err);
    if (rc == 2) { std::fprintf(stderr, "%s\n", err); return 2; }
    for (long long x = 0; x < (1LL << info.n); x++)
      if (!(x & mask)) inputs.push_back((int)x);
  }
  if (rus) {
    cz_rspec_info ri;
    for (int attempt = 0; attempt < 2; attempt++) {
      rc = cz_rspec_generate(q.data(), q.size(), 0, 0, nullptr, nullptr, outcome, out.data(), out.size(), &need, &ri, err,
                             sizeof err);
      if (rc != 3) break;
      out.assign(need + 1, 0);
    }
    if (rc) { std::fprintf(stderr, "%s\n", err); return 2; }
    std::fprintf(stderr, "{\"outcome\": %d, \"roots\": %d, \"p\": [%lld, %lld, %lld], \"rescalings\": %d, "
                         "\"failure_amplitudes\": %d}\n", ri.outcome, ri.roots, (long long)ri.p[0], (long long)ri.p[1],
                 (long long)ri.p[2], ri.rescalings, ri.failure_amplitudes);
    std::fwrite(out.data(), 1, need, stdout);
    return 0;
  }
  for (int attempt = 0; attempt < 2; attempt++) {
    rc = tcount ? cz_tspec_generate(q.data(), q.size(), 0, 0, nullptr, nullptr, out.data(), out.size(), &need, err,
                                    sizeof err)
                : cz_spec_generate_states(q.data(), q.size(), 0, 0, nullptr, nullptr, std::atoi(pos[1]), no_w3,
                                          inputs.data(), (int)inputs.size(), out.data(), out.size(), &need, &info, err,
                                          sizeof err);
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
