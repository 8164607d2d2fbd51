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


_MONO = {}


def _monomial(n):
    """per Pauli p: flip[p] (P_p maps column x to row x ^ flip) and ph[p, x] (entry w^ph)"""
    if n not in _MONO:
        P, N = 4 ** n, 1 << n
        flip = np.zeros(P, dtype=np.int64)
        ph = np.zeros((P, N), dtype=np.int64)
        for p in range(P):
            for x in range(N):
                f = k = 0
                for q in range(n):
                    d, bit = (p >> (2 * q)) & 3, (x >> q) & 1
                    if d == 1:
                        f |= 1 << q
                    elif d == 2:
                        f |= 1 << q
                        k += 2 + 4 * bit
                    elif d == 3:
                        k += 4 * bit
                flip[p] = f
                ph[p, x] = k & 7
        _MONO[n] = (flip, ph)
    return _MONO[n]


def _wrot(v, k):
    """w^k v elementwise: v holds Z[w] values as (4, ...) components, k integers shaped like v[0] (w^4 = -1)"""
    if np.ndim(k) == 0:                                       # one power for every element: a signed rotation
        k = int(k) % 8
        out = np.empty_like(v)
        for i in range(4):
            j = (i - k) % 4
            out[i] = -v[j] if ((j + k) // 4) % 2 else v[j]
        return out
    k = np.asarray(k) % 8
    out = np.empty_like(v)
    for i in range(4):
        j = (i - k) % 4                                       # the component that lands on w^i
        neg = ((j + k) // 4) % 2 == 1
        val = np.take_along_axis(v, j[None], axis=0)[0]
        out[i] = np.where(neg, -val, val)
    return out


def channel(n, U):
    """(e, x, y) int arrays: Uc[a][b] = (x + y sqrt2) / sqrt2^e, normalised (e minimal).
    P_b is monomial, so U P_b U^dag is two column gathers and one Z[w] matrix product per b, and Tr(P_a A) is a
    gather of A's entries at (x ^ flip_a, x) times w-powers, for all a at once."""
    k, M = U
    N, P = 1 << n, 4 ** n
    Mz = np.array([[M[r][c] for c in range(N)] for r in range(N)], dtype=np.int64).transpose(2, 0, 1)   # (4, N, N)
    Md = np.stack(zmat_dag(tuple(Mz)))
    flip, ph = _monomial(n)
    xs = np.arange(N)
    X = np.zeros((P, P), dtype=np.int64)
    Y = np.zeros((P, P), dtype=np.int64)
    rows = xs[None, :] ^ flip[:, None]                      # (P, N): row index x ^ flip_a
    phs = ph[np.arange(P)[:, None], rows]                    # Tr(P_a A) = sum_x w^ph_a(x ^ f_a) A[x ^ f_a, x]
    for b in range(P):
        cols = xs ^ flip[b]                                  # (Mz P_b)[r, y] = Mz[r, y ^ flip_b] w^ph_b(y)
        MP = _wrot(Mz[:, :, cols], np.broadcast_to(ph[b][None, :], (N, N)))
        A = np.stack(zmat_mul(tuple(MP), tuple(Md)))        # (4, N, N): sqrt2^2k U P_b U^dag
        G = A[:, rows, xs[None, :]]                          # (4, P, N): A[x ^ flip_a, x]
        T = _wrot(G, phs).sum(axis=2)                        # (4, P): Tr(P_a A)
        assert (T[2] == 0).all() and (T[3] == -T[1]).all(), "trace not real"
        X[:, b], Y[:, b] = T[0], T[1]
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


def unitary_np(n, circ):
    """the exact unitary of a gate list as workloads.unitary gives it (same gates, same normal form), computed with
    numpy row operations: (k, M) with M an N x N nested list of Z[w] 4-tuples"""
    from .workloads import _GATES
    N = 1 << n
    U = np.zeros((4, N, N), dtype=np.int64)
    U[0] = np.eye(N, dtype=np.int64)
    k = 0
    for g, qs in circ:
        gk, loc = _GATES[g]
        mask = sum(1 << q for q in qs)
        bases = np.array([b for b in range(N) if not b & mask], dtype=np.int64)
        rows = {l: bases | sum(((l >> j) & 1) << q for j, q in enumerate(qs)) for l in range(1 << len(qs))}
        new = np.zeros_like(U)
        for (l, m), pw in loc.items():
            new[:, rows[l], :] += _wrot(U[:, rows[m], :], pw)
        U = new
        if gk:                                                # keep the normal form (entries stay small)
            k, U = _zden(k + gk, tuple(U))
            U = np.stack(U)
    return k, [[tuple(int(v) for v in U[:, r, c]) for c in range(N)] for r in range(N)]


def tspec_of_circuit(n, circ):
    return tspec(n, unitary_np(n, circ))


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


# ---------------- table-driven workloads (uniform group elements from the resident Clifford table) ----------------
CLIFFORD_ORDER = {1: 24, 2: 11520, 3: 92897280}


def uniform_clifford_words(engine, n, rng, count):
    """`count` uniform random n-qubit Cliffords (up to phase) as optimal words: a uniform index into the group's
    rank table, that element's optimal word from the distance table"""
    idx = [rng.randrange(CLIFFORD_ORDER[n]) for _ in range(count)]
    return engine.clifford_words(n, engine.clifford_element(n, idx))


def table_queries(engine, seed, count=1024, n=3):
    """the table-driven T-count workload: U = C0 T(q1) C1 ... T(qk) Ck with k uniform in [1, 7], Ci uniform group
    elements, qi uniform qubits: [(circuit, k)]"""
    rng = random.Random(seed)
    ks = [rng.randint(1, 7) for _ in range(count)]
    words = uniform_clifford_words(engine, n, rng, sum(k + 1 for k in ks))
    out, w = [], 0
    for k in ks:
        circ = list(words[w])
        w += 1
        for _ in range(k):
            circ.append(("t", (rng.randrange(n),)))
            circ += words[w]
            w += 1
        out.append((circ, k))
    return out


def serve_requests(engine, seed, count):
    """the serving mix: 60% gate-count searches (random 2-3 qubit circuits as in the batched workload, budgets
    4..11), 30% T-count queries (as table_queries), 10% Clifford-segment minimisations (random 3-qubit Clifford
    words as zero-T cliffopt jobs): [(kind, text, depth, info)] with kind 0 / 1 / 2"""
    from .workloads import make_spec, random_circuit
    rng = random.Random(seed)
    kinds = [0 if u < 0.6 else (1 if u < 0.9 else 2) for u in (rng.random() for _ in range(count))]
    nq = sum(1 for k in kinds if k == 1)
    queries = table_queries(engine, seed + 1, nq) if nq else []
    out, qi = [], 0
    for kind in kinds:
        if kind == 0:
            n, circ = random_circuit(rng, L=rng.randint(4, 11))
            out.append((0, make_spec(n, circ, len(circ)), -1, {"n": n, "circuit": circ}))
        elif kind == 1:
            circ, k = queries[qi]
            qi += 1
            out.append((1, tspec_of_circuit(3, circ), -1, {"n": 3, "circuit": circ, "k": k}))
        else:
            out.append((2, random_clifford_job(rng, 3, 40, 0), -1, {"n": 3}))
    return out


def poisson_arrivals(seed, count, rate):
    rng = random.Random(seed)
    t, out = 0.0, []
    for _ in range(count):
        t += rng.expovariate(rate)
        out.append(t)
    return out
