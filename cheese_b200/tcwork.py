"""Inputs of the T-count and Clifford-table paths in the reference's formats.

* tspec: channel matrix Uc[a][b] = Tr(P_a U P_b U^dag) / 2^n as (x + y sqrt2) / sqrt2^e with one exponent, and the
  rotation table: for each Pauli P_p (p >= 1) and each Pauli P_c, (-1, 0) if they commute, else (r, s) with
  i P_p P_c = s P_r. The reference writes these with python/cheese/tcount.py (channel :79-101, pauli_tables :104-129,
  write_spec :157-168); this module computes the same normal form with numpy, checked against it byte for byte.
* cliffopt jobs: `n t`, t lines `q dagger`, t + 1 Clifford segments `m (gate q [q2])...` (clifford.cu:213-238).
* the table-driven T-count workload: queries U = C0 T(q1) C1 ... T(qk) Ck with k uniform in [1, 7], Ci random
  Cliffords (seeded random words of 60 gates over h, s, cx: a close approximation of uniform elements), qi uniform.

Pauli digits per qubit: 0 I, 1 X, 2 Y, 3 Z; Pauli index p has digit (p >> 2q) & 3 on qubit q.
"""
import random

import numpy as np

from .workloads import unitary

CLIFFORD_GATES = ["h", "s", "sdg", "x", "z", "cx"]


# ---------- exact Z[w] matrices as 4 int64 arrays (a + b w + c w^2 + d w^3) ----------
def zmat_mul(A, B):
    a0, a1, a2, a3 = A
    b0, b1, b2, b3 = B
    m = np.matmul
    return (m(a0, b0) - m(a1, b3) - m(a2, b2) - m(a3, b1), m(a0, b1) + m(a1, b0) - m(a2, b3) - m(a3, b2),
            m(a0, b2) + m(a1, b1) + m(a2, b0) - m(a3, b3), m(a0, b3) + m(a1, b2) + m(a2, b1) + m(a3, b0))


def zmat_dag(A):
    a0, a1, a2, a3 = A
    return (a0.T.copy(), -a3.T, -a2.T, -a1.T)


def pauli(n, p):
    """P_p as a Z[w] matrix: column x has w^phase at row x ^ flip"""
    N = 1 << n
    out = [np.zeros((N, N), dtype=np.int64) for _ in range(4)]
    for x in range(N):
        flip = ph = 0
        for q in range(n):
            d, bit = (p >> (2 * q)) & 3, (x >> q) & 1
            if d == 1:
                flip |= 1 << q
            elif d == 2:
                flip |= 1 << q
                ph += 2 + 4 * bit
            elif d == 3:
                ph += 4 * bit
        ph &= 7
        out[ph & 3][x ^ flip, x] = 1 if ph < 4 else -1
    return tuple(out)


def channel(n, U):
    """(e, x, y) int arrays: Uc[a][b] = (x + y sqrt2) / sqrt2^e, normalised (e minimal)"""
    k, M = U
    N, P = 1 << n, 4 ** n
    Mz = tuple(np.array([[M[r][c][i] for c in range(N)] for r in range(N)], dtype=np.int64) for i in range(4))
    Md = zmat_dag(Mz)
    paulis = [pauli(n, p) for p in range(P)]
    X = np.zeros((P, P), dtype=np.int64)
    Y = np.zeros((P, P), dtype=np.int64)
    for b in range(P):
        A = zmat_mul(zmat_mul(Mz, paulis[b]), Md)          # sqrt2^2k U P_b U^dag
        for a in range(P):
            T = zmat_mul(paulis[a], A)
            tr = [int(np.trace(t)) for t in T]
            assert tr[2] == 0 and tr[3] == -tr[1], "trace not real"
            X[a, b], Y[a, b] = tr[0], tr[1]                # value (x + y sqrt2) / sqrt2^(2k + 2n)
    e = 2 * k + 2 * n
    while e > 0 and not (X & 1).any():                     # (x + y s) / s = y + (x / 2) s
        X, Y = Y, X // 2
        e -= 1
    return e, X, Y


def pauli_tables(n):
    """per rotation p >= 1 and Pauli c: (-1, 0) if they commute, else (r, s) with i P_p P_c = s P_r"""
    P = 4 ** n
    ps = [pauli(n, p) for p in range(P)]
    iw = tuple(np.eye(1 << n, dtype=np.int64) * v for v in (0, 0, 1, 0))   # i = w^2 as a scalar matrix
    tab = []
    for p in range(1, P):
        row = []
        for c in range(P):
            M1, M2 = zmat_mul(ps[p], ps[c]), zmat_mul(ps[c], ps[p])
            if all((a == b).all() for a, b in zip(M1, M2)):
                row.append((-1, 0))
                continue
            M = zmat_mul(iw, M1)
            hit = None
            for r in range(P):
                for s in (1, -1):
                    if all((m == s * q).all() for m, q in zip(M, ps[r])):
                        hit = (r, s)
                        break
                if hit:
                    break
            assert hit
            row.append(hit)
        tab.append(row)
    return tab


_TABLES = {}


def tspec(n, U):
    """the tcount-spec text of unitary U (k, rows)"""
    e, X, Y = channel(n, U)
    if n not in _TABLES:
        _TABLES[n] = pauli_tables(n)
    tab = _TABLES[n]
    out = [f"tcount-spec 1\nn {n}\nchannel {e}\n"]
    for a in range(X.shape[0]):
        out.append(" ".join(f"{X[a, b]} {Y[a, b]}" for b in range(X.shape[1])) + "\n")
    out.append(f"rotations {len(tab)}\n")
    for row in tab:
        out.append(" ".join(f"{r} {s}" for r, s in row) + "\n")
    out.append("end\n")
    return "".join(out)


# ---------- seeded workloads ----------
def random_clifford_word(rng, n, length=60):
    word = []
    for _ in range(length):
        g = rng.choice(["h", "s", "cx"] if n > 1 else ["h", "s"])
        word.append((g, tuple(rng.sample(range(n), 2)) if g == "cx" else (rng.randrange(n),)))
    return word


def tcount_query(rng, n=3):
    """U = C0 T(q1) C1 ... T(qk) Ck: (gate list, k)"""
    k = rng.randint(1, 7)
    circ = random_clifford_word(rng, n)
    for _ in range(k):
        circ.append(("t", (rng.randrange(n),)))
        circ += random_clifford_word(rng, n)
    return circ, k


def tcount_queries(seed, count=1024, n=3):
    rng = random.Random(seed)
    return [tcount_query(rng, n) for _ in range(count)]


def cliffopt_job(n, tgates, segments):
    """job text: tgates [(q, dagger)], segments [[(gate, qubits)]] (len(tgates) + 1 of them)"""
    out = [f"{n} {len(tgates)}\n"]
    out += [f"{q} {d}\n" for q, d in tgates]
    for seg in segments:
        out.append(f"{len(seg)} " + " ".join(f"{g} " + " ".join(map(str, qs)) for g, qs in seg) + "\n")
    return "".join(out)


def random_clifford_job(rng, n=3, length=40, tcount=0):
    """a cliffopt job: tcount T gates on random qubits between random Clifford segments"""
    gates = ["h", "s", "sdg", "x", "z", "cx"]
    segs = []
    for _ in range(tcount + 1):
        seg = []
        for _ in range(rng.randint(length // 2, length)):
            g = rng.choice(gates)
            seg.append((g, tuple(rng.sample(range(n), 2)) if g == "cx" else (rng.randrange(n),)))
        segs.append(seg)
    ts = [(rng.randrange(n), rng.randrange(2)) for _ in range(tcount)]
    return cliffopt_job(n, ts, segs)


def tspec_of_circuit(n, circ):
    return tspec(n, unitary(n, circ))


# ---------- exact check of a T-count decomposition (the role of tcount.py verify, :171-185) ----------
def _zden(k, M):
    """normalise a (k, Z[w] matrix as 4 arrays) pair: divide by sqrt2 while every entry allows it"""
    a, b, c, d = M
    while k > 0:
        if ((a - c) & 1).any() or ((b - d) & 1).any():
            break
        a, b, c, d = (b - d) // 2, (a + c) // 2, (b + d) // 2, (c - a) // 2
        k -= 1
    return k, (a, b, c, d)


def rotation(n, p):
    """R(P_p) = ((1 + w) I + (1 - w) P_p) / 2 as (k, Z[w] matrix)"""
    N = 1 << n
    P = pauli(n, p)
    I = np.eye(N, dtype=np.int64)
    one_plus_w = (I, I, 0 * I, 0 * I)
    one_minus_w_P = zmat_mul((I, -I, 0 * I, 0 * I), P)
    return _zden(2, tuple(x + y for x, y in zip(one_plus_w, one_minus_w_P)))


def is_clifford(n, k, C):
    """C P C^dag is a Pauli up to a power of w for every Pauli P"""
    P4 = 4 ** n
    Cd = zmat_dag(C)
    paulis = [pauli(n, p) for p in range(P4)]
    for p in range(1, P4):
        kk, A = _zden(2 * k, zmat_mul(zmat_mul(C, paulis[p]), Cd))
        if kk:
            return False
        hit = False
        for r in range(1, P4):
            for ph in range(8):
                w = [0, 0, 0, 0]
                w[ph & 3] = 1 if ph < 4 else -1
                Q = zmat_mul(tuple(np.eye(1 << n, dtype=np.int64) * v for v in w), paulis[r])
                if all((x == y).all() for x, y in zip(A, Q)):
                    hit = True
                    break
            if hit:
                break
        if not hit:
            return False
    return True


def verify_decomposition(n, U, rotations):
    """U = X_1 ... X_t C with X = R(P_p) (inv 0) or R(P_p)^-1 (inv 1) and C a Clifford, exactly"""
    k, M = U
    N = 1 << n
    W = (k, tuple(np.array([[M[r][c][i] for c in range(N)] for r in range(N)], dtype=np.int64) for i in range(4)))
    for p, inv in rotations:
        kr, X = rotation(n, p)
        Xi = X if inv else zmat_dag(X)                        # X_i^-1: R(P)^dag = R(P)^-1
        W = _zden(W[0] + kr, zmat_mul(Xi, W[1]))
    return is_clifford(n, W[0], W[1])
