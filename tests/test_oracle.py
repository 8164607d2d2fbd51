"""The CPU restatement (oracle/) pinned against the reference's own outputs (tests/golden, produced by the
reference CPU build compiled from its sources) and against its own definitions of the bounds."""
import ctypes as C
import random

import pytest

from conftest import ORACLE_LIB, SLOW_CPU, golden_cases, run_oracle, spec_path

CASES = [c for c in golden_cases() if c["name"] not in SLOW_CPU and not c["name"].endswith("store64")]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference(oracle_bin, case):
    rc, out = run_oracle(oracle_bin, spec_path(case["spec"]), case["flags"])
    assert rc == case["rc"]
    assert out == case["stdout"]


def test_oracle_store64_matches_reference_store64_build(oracle_bin):
    g = {c["name"]: c for c in golden_cases()}["overflow-4-store64"]
    rc, out = run_oracle(oracle_bin, spec_path("overflow"), ["--store64"])
    assert rc == g["rc"] and out == g["stdout"]


def test_reference_verdicts(oracle_bin):
    """the reference's regression list (its tests/check.sh): exit codes per target and budget"""
    want = {("cs", 4): 1, ("cs", 5): 0, ("toffoli", 8): 1, ("ccz", 7): 1, ("qft_2", 7): 0, ("qft_2", 6): 1,
            ("relative-phase-toffoli", 9): 0}
    for (stem, d), rc0 in want.items():
        rc, _ = run_oracle(oracle_bin, spec_path(stem), ["--depth", str(d)])
        assert rc == rc0, (stem, d)


# ---- single-residual definitions: the Walsh-Hadamard T bound equals the direct PTM sde; the identities the GPU
# kernel relies on (T unchanged by Clifford gates, CX bound unchanged by one-qubit gates) ----

class Zw(C.Structure):
    _fields_ = [("a", C.c_int64), ("b", C.c_int64), ("c", C.c_int64), ("d", C.c_int64)]


@pytest.fixture(scope="module")
def olib(oracle_bin):
    L = C.CDLL(str(ORACLE_LIB))
    L.czo_ptm_t.argtypes = L.czo_ptm_sde.argtypes = [C.c_int, C.POINTER(Zw), C.c_int]
    L.czo_cut_rank.argtypes = [C.c_int, C.POINTER(Zw), C.c_int, C.c_int]
    return L


def _random_unitary(rng, n, length):
    from cheese_b200 import workloads
    circ = []
    for _ in range(length):
        g = rng.choice(["h", "t", "tdg", "s", "x", "cx", "z", "sdg"])
        if g == "cx":
            a, b = rng.sample(range(n), 2)
            circ.append((g, (a, b)))
        else:
            circ.append((g, (rng.randrange(n),)))
    k, M = workloads.unitary(n, circ)
    arr = (Zw * (len(M) * len(M)))()
    for r, row in enumerate(M):
        for c, x in enumerate(row):
            arr[r * len(M) + c] = Zw(*x)
    return k, arr, circ


def test_wht_t_bound_equals_direct_sde(olib):
    rng = random.Random(7)
    for _ in range(60):
        n = rng.choice([2, 3])
        k, arr, _ = _random_unitary(rng, n, rng.randint(0, 14))
        assert olib.czo_ptm_t(n, arr, k) == olib.czo_ptm_sde(n, arr, k)


def test_t_bound_invariant_under_clifford_gates(olib):
    from cheese_b200 import workloads
    rng = random.Random(11)
    for _ in range(40):
        n = rng.choice([2, 3])
        k, arr, circ = _random_unitary(rng, n, rng.randint(2, 12))
        t0 = olib.czo_ptm_t(n, arr, k)
        for g in ["h", "s", "sdg", "x", "z", "cx"]:
            qs = tuple(rng.sample(range(n), 2)) if g == "cx" else (rng.randrange(n),)
            k2, M2 = workloads.unitary(n, circ + [(g, qs)])
            arr2 = (Zw * (len(M2) ** 2))(*[Zw(*x) for row in M2 for x in row])
            assert olib.czo_ptm_t(n, arr2, k2) == t0


def test_cut_rank_invariant_under_one_qubit_gates(olib):
    from cheese_b200 import workloads
    rng = random.Random(13)
    for _ in range(40):
        n = 3
        k, arr, circ = _random_unitary(rng, n, rng.randint(2, 12))
        r0 = [olib.czo_cut_rank(n, arr, 1 << q, 1) for q in range(n)]
        for g in ["h", "s", "t", "tdg", "x", "z", "sdg"]:
            k2, M2 = workloads.unitary(n, circ + [(g, (rng.randrange(n),))])
            arr2 = (Zw * 64)(*[Zw(*x) for row in M2 for x in row])
            assert [olib.czo_cut_rank(n, arr2, 1 << q, 1) for q in range(n)] == r0
