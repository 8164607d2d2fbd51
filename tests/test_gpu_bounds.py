"""Device bound functions (T bound, CX bound, H structure, support) against the oracle's restatement of the
reference definitions, on random residuals: short circuits (int32 path, k <= 29) and long H-heavy ones (k > 29:
the transform runs mod 2^64)."""
import ctypes as C
import random

import pytest

import cheese_b200 as cz
from cheese_b200 import workloads
from conftest import ORACLE_LIB, spec_text

pytestmark = pytest.mark.gpu


class Zw(C.Structure):
    _fields_ = [("a", C.c_int64), ("b", C.c_int64), ("c", C.c_int64), ("d", C.c_int64)]


@pytest.fixture(scope="module")
def olib(oracle_bin):
    L = C.CDLL(str(ORACLE_LIB))
    for f in ("czo_ptm_t", "czo_ptm_sde"):
        getattr(L, f).argtypes = [C.c_int, C.POINTER(Zw), C.c_int]
    L.czo_cut_rank.argtypes = [C.c_int, C.POINTER(Zw), C.c_int, C.c_int]
    L.czo_h_struct.argtypes = L.czo_support.argtypes = [C.c_int, C.POINTER(Zw)]
    return L


def spec_cuts(text):
    t = text.split()
    i = t.index("cuts")
    m = int(t[i + 1])
    cuts, j = [], i + 2
    for _ in range(m):
        sz = int(t[j])
        cuts.append((sz, sum(1 << int(q) for q in t[j + 1:j + 1 + sz])))
        j += 1 + sz
    i = t.index("cxtable")
    m = int(t[i + 1])
    return cuts, [int(v) for v in t[i + 2:i + 2 + m]]


def oracle_bounds(olib, n, k, M, cuts, table):
    arr = (Zw * (len(M) ** 2))(*[Zw(*x) for row in M for x in row])
    T = olib.czo_ptm_t(n, arr, k)
    idx = mult = mx = 0
    mult = 1
    for sz, mask in cuts:
        rk = olib.czo_cut_rank(n, arr, mask, sz)
        need = 0
        while (1 << need) < rk:
            need += 1
        need = min(need, 2 * sz)
        idx += need * mult
        mult *= 2 * sz + 1
        mx = max(mx, need)
    c2 = table[idx] if table else mx
    ident = k == 0 and all(M[r][c] == ((1, 0, 0, 0) if r == c else (0, 0, 0, 0)) for r in range(len(M)) for c in range(len(M)))
    if ident:                       # the search stops at the goal before the cheap bounds
        return (T, c2, -1, -1)
    return (T, c2, olib.czo_h_struct(n, arr), olib.czo_support(n, arr))


def random_residuals(rng, n, count, lmin, lmax):
    out = []
    for _ in range(count):
        circ = []
        for _ in range(rng.randint(lmin, lmax)):
            g = rng.choice(["h", "t", "tdg", "s", "sdg", "x", "z", "cx"])
            circ.append((g, tuple(rng.sample(range(n), 2)) if g == "cx" else (rng.randrange(n),)))
        out.append(workloads.unitary(n, circ))
    return out


@pytest.mark.parametrize("n,stem", [(3, "toffoli"), (2, "cs")])
def test_bounds_match_oracle(olib, n, stem):
    rng = random.Random(1000 + n)
    e = cz.Engine(0)
    text = spec_text(stem)
    cuts, table = spec_cuts(text)
    res = random_residuals(rng, n, 300, 0, 16)
    got = e.eval_bounds(text, res)
    for (k, M), g in zip(res, got):
        assert g == oracle_bounds(olib, n, k, M, cuts, table), (k, g)
    e.close()


def test_t_bound_uint64_path_matches_oracle(olib):
    # long H-heavy circuits: sqrt2 exponent k > 29, so 2(n + k) > 64 and the transform runs mod 2^64
    rng = random.Random(77)
    e = cz.Engine(0)
    text = spec_text("toffoli")
    cuts, table = spec_cuts(text)
    res = []
    for _ in range(40):                    # (H T)-chains on random qubits with some CX: k between 30 and 50
        circ = []
        for _ in range(rng.randint(60, 90)):
            q = rng.randrange(3)
            circ += [("h", (q,)), (rng.choice(["t", "tdg"]), (q,))]
            if rng.random() < 0.2:
                circ.append(("cx", tuple(rng.sample(range(3), 2))))
        res.append(workloads.unitary(3, circ))
    res = [r for r in res if r[0] > 29]
    assert len(res) > 20
    got = e.eval_bounds(text, res)
    for (k, M), g in zip(res, got):
        assert g == oracle_bounds(olib, 3, k, M, cuts, table), k
    e.close()


def test_t_bound_is_the_direct_ptm_sde(olib):
    rng = random.Random(5)
    e = cz.Engine(0)
    res = random_residuals(rng, 3, 60, 0, 12)
    got = e.eval_bounds(spec_text("toffoli"), res)
    for (k, M), g in zip(res, got):
        arr = (Zw * 64)(*[Zw(*x) for row in M for x in row])
        assert g[0] == olib.czo_ptm_sde(3, arr, k)
    e.close()
