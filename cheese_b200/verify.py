"""Exact re-verification of a found circuit (the role of the reference's python/cheese/verify.py:20-45):
multiply the candidate gates out over Z[w] and compare with the target unitary, global phase included."""
from .workloads import gate_matrix, matmul, normalise


def circuit_unitary(n, names):
    N = 1 << n
    U = (0, [[(1, 0, 0, 0) if i == j else (0, 0, 0, 0) for j in range(N)] for i in range(N)])
    for nm in names:                           # L_<gate>_<q>[_<q>...]
        _, g, *qs = nm.split("_")
        U = matmul(gate_matrix(g, tuple(int(q) for q in qs), n), U)
    return U


def spec_target(spec_text):
    """(n, (k, rows)) of a spec's target block"""
    toks = spec_text.split()
    n = int(toks[toks.index("n") + 1])
    i = toks.index("target")
    k = int(toks[i + 1])
    N = 1 << n
    vals = list(map(int, toks[i + 2:i + 2 + 4 * N * N]))
    rows = [[tuple(vals[4 * (r * N + c):4 * (r * N + c) + 4]) for c in range(N)] for r in range(N)]
    return n, normalise(k, rows)


def equivalent(spec_text, names):
    n, T = spec_target(spec_text)
    k, M = circuit_unitary(n, names)
    return (k, [list(r) for r in M]) == (T[0], [list(r) for r in T[1]])


def state_equivalent(spec_text, names):
    """for a state-target spec: the circuit maps every listed input basis state to the target's image exactly
    (global phase included), i.e. its columns at the inputs, as rows, equal the spec's goal rows"""
    toks = spec_text.split()
    n = int(toks[toks.index("n") + 1])
    m = int(toks[toks.index("pairs") + 1])
    N = 1 << n
    i = toks.index("start")
    vals = list(map(int, toks[i + 2:i + 2 + 4 * N * N]))
    inputs = []
    for r in range(m):
        row = [tuple(vals[4 * (r * N + c):4 * (r * N + c) + 4]) for c in range(N)]
        inputs.append(next(c for c in range(N) if row[c] != (0, 0, 0, 0)))
    _, G = spec_target(spec_text)
    k, M = circuit_unitary(n, names)
    rows = [[M[r][x] for r in range(N)] for x in inputs] + [[(0, 0, 0, 0)] * N for _ in range(N - m)]
    kk, R = normalise(k, rows)
    return (kk, [list(r) for r in R]) == (G[0], [list(r) for r in G[1]])


# ---------- RUS circuits (the role of the reference's `python -m cheese.rus verify`, rus.py:306-331) ----------
ZERO4 = (0, 0, 0, 0)


def _pauli(n, p):
    """P_p, digits per qubit (0 I, 1 X, 2 Y, 3 Z) at bits 2q, as (0, rows)"""
    N = 1 << n
    M = [[ZERO4] * N for _ in range(N)]
    for x in range(N):
        flip = ph = 0
        for q in range(n):
            d, bit = (p >> (2 * q)) & 3, (x >> q) & 1
            if d in (1, 2):
                flip |= 1 << q
            ph += (2 + 4 * bit) if d == 2 else (4 * bit if d == 3 else 0)
        M[x ^ flip][x] = _wpow(ph)
    return 0, M


def _wpow(p):
    p &= 7
    out = [0, 0, 0, 0]
    out[p & 3] = 1 if p < 4 else -1
    return tuple(out)


def _adj(A):
    k, a = A
    return k, [[(a[j][i][0], -a[j][i][3], -a[j][i][2], -a[j][i][1]) for j in range(len(a))] for i in range(len(a[0]))]


def _rotation(p, inv):
    """time-ordered gates of R(P_p) on two qubits (R(P)^-1 if inv): basis changes, a CX ladder onto the first
    support qubit, T or Tdg there, the ladder and the basis changes undone"""
    sup = [(q, (p >> (2 * q)) & 3) for q in range(2) if (p >> (2 * q)) & 3]
    q0 = sup[0][0]
    ladder = [("cx", (q, q0)) for q, _ in sup[1:]]
    pre, post = [], []
    for q, d in sup:
        if d == 1:
            pre.append(("h", (q,)))
            post.append(("h", (q,)))
        elif d == 2:
            pre += [("sdg", (q,)), ("h", (q,))]
            post += [("h", (q,)), ("s", (q,))]
    return pre + ladder + [("tdg" if inv else "t", (q0,))] + ladder + post


_GACT = None


def rspec_cliffords(rspec_text):
    """the Clifford list of a rus-spec (its "cliffords" block): per Clifford C, (perm, sign) with
    C^dag P_a C = sign[a] P_perm[a] for the 16 two-qubit Paulis a (digits per qubit 0 I, 1 X, 2 Y, 3 Z at bits 2q)"""
    toks = rspec_text.split()
    i = toks.index("cliffords")
    m = int(toks[i + 1])
    vals = list(map(int, toks[i + 2:i + 2 + 32 * m]))
    return [(tuple(vals[32 * c:32 * c + 32:2]), tuple(vals[32 * c + 1:32 * c + 32:2])) for c in range(m)]


def _gate_actions():
    """conjugation actions (perm, sign) of h q0, h q1, s q0, s q1 and cz on the 16 Paulis, from their matrices"""
    global _GACT
    if _GACT is None:
        P16 = [_pauli(2, p) for p in range(16)]
        _GACT = {}
        for g, qs in (("h", (0,)), ("h", (1,)), ("s", (0,)), ("s", (1,)), ("cz", (0, 1))):
            C = gate_matrix(g, qs, 2)
            Cd = _adj(C)
            perm, sign = [0] * 16, [0] * 16
            for a in range(16):
                k, A = matmul(matmul(Cd, P16[a]), C)
                for b in range(16):
                    for sg in (1, -1):
                        if (k, A) == (0, [[tuple(sg * v for v in x) for x in row] for row in P16[b][1]]):
                            perm[a], sign[a] = b, sg
            _GACT[(g, qs)] = (perm, sign)
    return _GACT


def clifford_word(action):
    """a gate word (time order; gates h, sdg and cz) of the two-qubit Clifford with the given Pauli action
    (perm, sign), up to global phase. The images of X_q and Z_q are reduced to +X_q and +Z_q by conjugation with
    gates g_1 .. g_m, qubit by qubit: Z_q's image made a lone Z on q, then X_q's image a lone X on q with gates that
    keep Z_q, then the signs. So C g_1 .. g_m is the identity up to phase and C = g_m^-1 .. g_1^-1 (g_1^-1 first)."""
    act = _gate_actions()
    X = lambda q: 1 << (2 * q)
    Z = lambda q: 3 << (2 * q)
    img = {P: (action[1][P], action[0][P]) for q in range(2) for P in (X(q), Z(q))}
    word = []

    def apply(*gates):                      # right-multiply the Clifford by each gate: its images conjugated by it
        for g in gates:
            perm, sign = act[g]
            for P, (sg, b) in img.items():
                img[P] = (sg * sign[b], perm[b])
            word.append(g)

    H = lambda q: ("h", (q,))
    S = lambda q: ("s", (q,))
    CZ = ("cz", (0, 1))
    cx = lambda c, t: apply(H(t), CZ, H(t))  # CX(c -> t) = H_t CZ H_t
    digit = lambda b, q: (b >> (2 * q)) & 3
    for q in range(2):
        o = 1 - q
        # Z_q's image: every Y (S: Y -> X) and X (H: X -> Z) digit on qubits >= q turned into Z, then a lone Z on q
        for j in range(q, 2):
            if digit(img[Z(q)][1], j) == 2:
                apply(S(j))
            if digit(img[Z(q)][1], j) == 1:
                apply(H(j))
        if q == 0:
            if digit(img[Z(q)][1], q) == 0:
                cx(q, o)                         # Z_o -> Z_q Z_o: a Z on q
            if digit(img[Z(q)][1], o):
                cx(o, q)                         # Z_q -> Z_o Z_q: the Z on o cleared
            # X_q's image anticommutes with Z_q (an X or Y on q); CX(q -> o), CZ and S_q keep Z_q
            if digit(img[X(q)][1], o) in (1, 2):
                cx(q, o)                         # X_q -> X_q X_o: no X part left on o
            if digit(img[X(q)][1], o) == 3:
                apply(CZ)                        # X_q -> X_q Z_o: the Z on o cleared
        if digit(img[X(q)][1], q) == 2:
            apply(S(q))                          # Y_q -> X_q
    for q in range(2):                           # signs: Z_q = S_q S_q flips X_q's, X_q = H_q Z_q H_q flips Z_q's
        if img[X(q)][0] < 0:
            apply(S(q), S(q))
        if img[Z(q)][0] < 0:
            apply(H(q), S(q), S(q), H(q))
    if any(img[P] != (1, P) for P in img):
        raise ValueError("not a Clifford action")
    inverse = {"h": "h", "cz": "cz", "s": "sdg"}
    return [(inverse[g], qs) for g, qs in word]


def rus_circuit(res, cliffords):
    """the gates (time order) of a `rus` result: W = R(P_1)..R(P_j) C R(Q_c)^-1..R(Q_1)^-1 with fw = (P_1..P_j), the
    Clifford C = entry `cliff` of the rus-spec's Clifford list (rspec_cliffords) and tb = (Q_1..Q_c)"""
    gates = []
    for q in res["tb"]:
        gates += _rotation(q, True)
    for g, qs in clifford_word(cliffords[res["cliff"]]):
        gates += [("h", (1,)), ("cx", (0, 1)), ("h", (1,))] if g == "cz" else [(g, qs)]
    for p in reversed(res["fw"]):
        gates += _rotation(p, False)
    return gates


def _blocks(W):
    k, w = W
    return k, [[[w[o + 2 * i][2 * j] for j in range(2)] for i in range(2)] for o in range(2)]


def _scalar(A):
    k, a = A
    if any(a[i][j] != ZERO4 for i in range(len(a)) for j in range(len(a)) if i != j) or \
            len({a[i][i] for i in range(len(a))}) != 1:
        return None
    kk, m = normalise(k, [[a[0][0]]])
    return kk, m[0][0]


def _clifford_block(k, B):
    """B / sqrt2^k proportional to a one-qubit Clifford: B B^dag = q I and B P B^dag Q = +-q I"""
    Bm = (k, [list(r) for r in B])
    G = _scalar(matmul(Bm, _adj(Bm)))
    if G is None or G[1] == ZERO4:
        return False
    negG = (G[0], tuple(-v for v in G[1]))
    for p in (1, 3):
        A = matmul(matmul(Bm, _pauli(1, p)), _adj(Bm))
        if not any(_scalar(matmul(A, _pauli(1, q))) in (G, negG) for q in (1, 2, 3)):
            return False
    return True


def rus_success_outcome(qasm_text, W):
    """the "success outcome K" comment of the file, else the branch that is not proportional to a Clifford"""
    import re
    m = re.search(r"success outcome (\d)", qasm_text)
    if m:
        return int(m.group(1))
    k, B = _blocks(W)
    cl = [_clifford_block(k, B[o]) for o in range(2)]
    if cl.count(True) != 1:
        raise ValueError("not a RUS circuit: need exactly one branch proportional to a Clifford")
    return cl.index(False)


def parse_qasm(text):
    """(n, [(gate, qubits)]) of the OpenQASM subset the spec writers read (qreg / qubit declaration, one gate per
    statement; measure, creg, comments skipped)"""
    import re
    n, circ = 0, []
    for line in text.splitlines():
        line = line.split("//")[0].strip()
        m = re.match(r"(?:qreg\s+\w+|qubit)\[(\d+)\]", line)
        if m:
            n = int(m.group(1))
            continue
        m = re.match(r"([a-z]+)\s+(.*);", line)
        if m and m.group(1) in ("x", "y", "z", "h", "s", "sdg", "t", "tdg", "cx", "cz", "ccx"):
            circ.append((m.group(1), tuple(int(q) for q in re.findall(r"\[(\d+)\]", m.group(2)))))
    return n, circ


def rus_check(qasm_text, res, cliffords, outcome=None):
    """exact check of a `rus` result against its target circuit: the result's circuit V has the target's success
    branch (outcome 0 of V = a unit times the target's outcome-ks branch, so the same success unitary and
    probability), its failure branch is proportional to a Clifford, and its T-count is the reported one.
    cliffords: the Clifford list of the rus-spec the result came from (rspec_cliffords)"""
    from .workloads import unitary
    n, circ = parse_qasm(qasm_text)
    if n != 2:
        return False
    W = unitary(2, circ)
    ks = outcome if outcome is not None else rus_success_outcome(qasm_text, W)
    gates = rus_circuit(res, cliffords)
    V = unitary(2, gates)
    kW, BW = _blocks(W)
    kV, BV = _blocks(V)
    M = (kW, [list(r) for r in BW[ks]])
    S = (kV, [list(r) for r in BV[0]])
    pM = _scalar(matmul(M, _adj(M)))                      # M M^dag = p I
    mu = _scalar(matmul(S, _adj(M)))                      # S M^dag = mu I, so S = (mu / p) M
    if pM is None or mu is None:
        return False
    from .workloads import zmul
    conj = lambda z: (z[0], -z[3], -z[2], -z[1])
    sq = lambda s, z: normalise(2 * s[0], [[zmul(s[1], z)]])
    tcount = sum(g in ("t", "tdg") for g, _ in gates)
    return sq(mu, conj(mu[1])) == sq(pM, pM[1]) and _clifford_block(kV, BV[1]) and tcount == res["tcount"]
