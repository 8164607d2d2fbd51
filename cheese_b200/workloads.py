"""Synthetic workloads in the reference's input format: seeded random Clifford+T circuits, their exact unitaries,
and their cheese spec files (written by the library's native spec writer).

Exact arithmetic: an entry of Z[w] (w = e^{i pi/4}) is (a, b, c, d) = a + b w + c w^2 + d w^3; a matrix is
(k, rows) meaning rows / sqrt2^k with k as small as possible (the normal form of the reference's spec writer,
python/cheese/spec.py:55-84, so the target block is byte-identical to the one it writes for the same circuit).

Random circuits follow the batched-search workload: n uniform in {2, 3}, length L uniform in [6, 12], each gate
T or Tdg with probability 0.15 each, otherwise uniform over {x, z, h, s, sdg, cx}, qubits uniform (cx: an
ordered pair of distinct qubits), budget L.
"""
import os
import random

ZERO = (0, 0, 0, 0)
ONE = (1, 0, 0, 0)

# gate -> (sqrt2 exponent, local matrix as {(row, col): w-power}); bit j of a local index is qubit qs[j]
_GATES = {
    "x": (0, {(0, 1): 0, (1, 0): 0}),
    "z": (0, {(0, 0): 0, (1, 1): 4}),
    "s": (0, {(0, 0): 0, (1, 1): 2}),
    "sdg": (0, {(0, 0): 0, (1, 1): 6}),
    "t": (0, {(0, 0): 0, (1, 1): 1}),
    "tdg": (0, {(0, 0): 0, (1, 1): 7}),
    "h": (1, {(0, 0): 0, (0, 1): 0, (1, 0): 0, (1, 1): 4}),
    # cx with control = local bit 0, target = local bit 1
    "cx": (0, {(0, 0): 0, (1, 3): 0, (2, 2): 0, (3, 1): 0}),
    "y": (0, {(0, 1): 6, (1, 0): 2}),
    "cz": (0, {(0, 0): 0, (1, 1): 0, (2, 2): 0, (3, 3): 4}),
    # ccx: controls local bits 0 and 1, target bit 2 (local states 3 and 7 swap)
    "ccx": (0, {(l, {3: 7, 7: 3}.get(l, l)): 0 for l in range(8)}),
}
ONE_QUBIT = ["x", "z", "h", "s", "sdg"]


def zmul(x, y):
    out = [0, 0, 0, 0]
    for i, a in enumerate(x):
        if a:
            for j, b in enumerate(y):
                if b:
                    s = i + j
                    out[s & 3] += a * b if s < 4 else -a * b
    return tuple(out)


def zadd(x, y):
    return (x[0] + y[0], x[1] + y[1], x[2] + y[2], x[3] + y[3])


def wpow(p):
    p &= 7
    out = [0, 0, 0, 0]
    out[p & 3] = 1 if p < 4 else -1
    return tuple(out)


def zdown(x):
    a, b, c, d = x
    if (a - c) & 1 or (b - d) & 1:
        return None
    return ((b - d) // 2, (a + c) // 2, (b + d) // 2, (c - a) // 2)


def normalise(k, M):
    while k > 0:
        D = [[zdown(x) for x in row] for row in M]
        if any(x is None for row in D for x in row):
            break
        M, k = D, k - 1
    return k, [list(r) for r in M]


def gate_matrix(g, qs, n):
    gk, loc = _GATES[g]
    N, mask = 1 << n, sum(1 << q for q in qs)
    out = [[ZERO] * N for _ in range(N)]
    for base in range(N):
        if base & mask:
            continue
        idx = [base | sum(((l >> j) & 1) << q for j, q in enumerate(qs)) for l in range(1 << len(qs))]
        for (l, m), p in loc.items():
            out[idx[l]][idx[m]] = zadd(out[idx[l]][idx[m]], wpow(p))
    return gk, out


def matmul(A, B):
    (ka, a), (kb, b) = A, B
    N = len(a)
    out = [[ZERO] * N for _ in range(N)]
    for i in range(N):
        for l in range(N):
            if a[i][l] != ZERO:
                for j in range(N):
                    if b[l][j] != ZERO:
                        out[i][j] = zadd(out[i][j], zmul(a[i][l], b[l][j]))
    return normalise(ka + kb, out)


def unitary(n, circ):
    """exact unitary of a gate list [(gate, qubits)], applied in order (product g_L ... g_1)"""
    N = 1 << n
    U = (0, [[ONE if i == j else ZERO for j in range(N)] for i in range(N)])
    for g, qs in circ:
        U = matmul(gate_matrix(g, tuple(qs), n), U)
    return U


def random_circuit(rng, n=None, L=None):
    n = rng.choice((2, 3)) if n is None else n
    L = rng.randint(6, 12) if L is None else L
    circ = []
    for _ in range(L):
        u = rng.random()
        if u < 0.15:
            g = "t"
        elif u < 0.30:
            g = "tdg"
        else:
            g = rng.choice(ONE_QUBIT + ["cx"])
        if g == "cx":
            a = rng.randrange(n)
            b = rng.randrange(n - 1)
            b += b >= a
            circ.append((g, (a, b)))
        else:
            circ.append((g, (rng.randrange(n),)))
    return n, circ


def batch(seed, count=512):
    """the batched workload: `count` seeded (n, circuit, budget) jobs"""
    rng = random.Random(seed)
    out = []
    for _ in range(count):
        n, circ = random_circuit(rng)
        out.append((n, circ, len(circ)))
    return out


def make_spec(n, circ, depth):
    """spec text for the circuit's unitary with budget `depth`, written by the library's native spec writer
    (cz_spec_generate: the default Clifford+T candidates, window rules, cuts and CX table of n qubits)"""
    from . import spec_generate
    return spec_generate(n, list(circ), depth=depth)[0]


def qasm(n, circ):
    body = "".join(f"{g} " + ",".join(f"q[{q}]" for q in qs) + ";\n" for g, qs in circ)
    return f"OPENQASM 2.0;\ninclude \"qelib1.inc\";\nqreg q[{n}];\n" + body


if __name__ == "__main__":   # print one seeded job's spec: python -m cheese_b200.workloads SEED INDEX
    import sys
    seed, idx = int(sys.argv[1]), int(sys.argv[2])
    n, circ, d = batch(seed, idx + 1)[idx]
    sys.stdout.write(make_spec(n, circ, d))
    print(f"{n} qubits, {d} gates: {circ}", file=sys.stderr)
    os._exit(0)
