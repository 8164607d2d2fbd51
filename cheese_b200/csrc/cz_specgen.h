// Host-side spec generation: the target circuit -> the text spec of the gate-count search (what the reference's
// python/cheese/spec.py writes, unitary targets) and the T-count spec (python/cheese/tcount.py:79-168), in exact
// Z[w] arithmetic. The per-gate-set parts (candidates, window rules, CX table) are cached, so a served request pays
// only for its target.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cz {

struct CircGate {
  std::string g;     // x y z s sdg t tdg h cx cz ccx
  int nq = 0;
  int q[3] = {-1, -1, -1};
};

// OpenQASM subset of the reference's parse_qasm (spec.py:113-123): "qreg name[n];" or "qubit[n];" sets the qubit
// count, "g args;" with g a known gate adds it on the qubits [i] named in args; everything else is skipped
int parse_qasm(const char *text, size_t len, int &n, std::vector<CircGate> &circ, std::string &err);

struct SpecGenInfo { int candidates = 0, bad2 = 0, bad3 = 0; };
// the gate-count spec of the circuit's unitary with budget `depth` (gate set: Clifford+T plus the circuit's own
// gates). With `inputs` (basis states, bit q = qubit q) it is the state-target spec of spec.py:356-415 instead: the
// start rows e_x, the goal rows U e_x and, per goal row, its sde, stabilizer nullity and Schmidt ranks across the
// cuts. Returns 0, or 2 with err (unknown gate, bad qubit, n out of range, bad input, coefficient overflow).
int spec_generate(int n, const std::vector<CircGate> &circ, int depth, bool use_w3, const std::vector<int> &inputs,
                  std::string &out, SpecGenInfo &info, std::string &err);
// the T-count spec (channel representation and Pauli rotation tables) of the circuit's unitary
int tspec_generate(int n, const std::vector<CircGate> &circ, std::string &out, std::string &err);

struct RusSpecInfo { int outcome = 0, roots = 0, rescalings = 0, failure_amplitudes = 0; int64_t p[3] = {0, 0, 0}; };
// the rus-spec of a two-qubit RUS circuit (q0 ancilla, measured; q1 data), as python/cheese/rus.py spec writes it:
// the table root J00, the roots (every valid isometry for this success branch up to left Cliffords), the rotation
// tables and the 11520 Cliffords. outcome: the success outcome, or -1 for the "success outcome K" comment in
// qasm_text, else the branch that is not proportional to a Clifford. Returns 0, or 2 with err.
int rspec_generate(int n, const std::vector<CircGate> &circ, const std::string &qasm_text, int outcome,
                   std::string &out, RusSpecInfo &info, std::string &err);

}  // namespace cz
