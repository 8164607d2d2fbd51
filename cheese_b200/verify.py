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
