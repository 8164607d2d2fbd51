"""T-count and Clifford-table paths on the CPU: tcount-spec generation, host parsing through the C ABI, and the C
restatements (oracle/tc_oracle.c, oracle/clifford_oracle.c) pinned against the reference's own outputs."""
import json
import random
import subprocess
from pathlib import Path

import pytest

from conftest import GOLD, ORACLE_DIR, strip_seconds

from cheese_b200 import SpecError, lib, tcwork, tspec_check
import ctypes as C

TC_ORACLE = ORACLE_DIR / "_ref" / "tc-oracle"
CL_ORACLE = ORACLE_DIR / "_ref" / "clifford-oracle"
TC_GOLD = GOLD / "tcount_cases.json"
CL_GOLD = GOLD / "cliffopt_cases.json"


@pytest.fixture(scope="session")
def oracles():
    if not TC_ORACLE.exists() or not CL_ORACLE.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "oracle"], check=True, capture_output=True)
    return TC_ORACLE, CL_ORACLE


def _perm(n, p):
    N = 1 << n
    M = [[(0, 0, 0, 0)] * N for _ in range(N)]
    for c in range(N):
        M[p(c)][c] = (1, 0, 0, 0)
    return (0, M)


def _diag(n, phase):
    N = 1 << n
    M = [[(0, 0, 0, 0)] * N for _ in range(N)]
    for c in range(N):
        e = [0, 0, 0, 0]
        k = phase(c) % 8
        e[k % 4] = 1 if k < 4 else -1
        M[c][c] = tuple(e)
    return (0, M)


def _fredkin(x):
    return 1 | (((x >> 2) & 1) << 1) | (((x >> 1) & 1) << 2) if x & 1 else x


# targets by their unitaries (basis index bit q = qubit q): the tcount-spec fixtures were written by the
# reference's tcount.py from its qasm files; the same text must come out of tcwork
TARGETS = {
    "toffoli": (3, _perm(3, lambda x: x ^ 4 if (x & 3) == 3 else x)),
    "ccz": (3, _diag(3, lambda x: 4 if x == 7 else 0)),
    "cs": (2, _diag(2, lambda x: 2 if x == 3 else 0)),
    "fredkin": (3, _perm(3, _fredkin)),
}


@pytest.mark.parametrize("name", sorted(TARGETS))
def test_tspec_matches_reference_writer(name):
    n, U = TARGETS[name]
    assert tcwork.tspec(n, U) == (GOLD / "tcount" / f"{name}.tspec").read_text()


def test_query_fixtures_regenerate():
    rng = random.Random(4096)
    for i in range(8):
        circ, k = tcwork.tcount_query(rng, 3)
        assert 1 <= k <= 7
        assert tcwork.tspec_of_circuit(3, circ) == (GOLD / "tcount" / f"q3-{i}.tspec").read_text()
    for i in range(4):
        circ, _ = tcwork.tcount_query(rng, 2)
        assert tcwork.tspec_of_circuit(2, circ) == (GOLD / "tcount" / f"q2-{i}.tspec").read_text()


def test_verify_decomposition_of_published_optima():
    """the reference's benchmarks/optimal decompositions verify exactly; dropping a rotation breaks them"""
    opt = {c["name"]: json.loads(c["stdout"][-1]) for c in json.loads((GOLD / "tcount" / "optimal.json").read_text())}
    for name, (n, U) in TARGETS.items():
        rots = opt[name]["rotations"]
        assert len(rots) == opt[name]["tcount"]
        assert tcwork.verify_decomposition(n, U, rots), name
        assert not tcwork.verify_decomposition(n, U, rots[1:]), name


def test_tspec_check_errors():
    assert tspec_check((GOLD / "tcount" / "cs.tspec").read_text()) == 2
    with pytest.raises(SpecError) as e:
        tspec_check("foo")
    assert e.value.rc == 2 and "not a tcount spec" in str(e.value)
    with pytest.raises(SpecError) as e:
        tspec_check("tcount-spec 1\nn 4\nend\n")
    assert e.value.rc == 3
    with pytest.raises(SpecError) as e:
        tspec_check("tcount-spec 1\nn 1\nbogus 3\nend\n")
    assert e.value.rc == 2 and "unknown field bogus" in str(e.value)
    with pytest.raises(SpecError) as e:
        tspec_check("tcount-spec 1\nn 1\nchannel 0\n1 0\nend\n")
    assert e.value.rc == 2


def test_cliffjob_check():
    n, t = C.c_int(), C.c_int()
    err = C.create_string_buffer(256)
    job = (GOLD / "cliffopt" / "t3-0.job").read_bytes()
    assert lib().cz_cliffjob_check(job, len(job), C.byref(n), C.byref(t), err, 256) == 0
    assert (n.value, t.value) == (3, 2)
    for bad, msg in [(b"4 0\n0\n", "bad job file"), (b"2 0\n1 q 0\n", "unknown Clifford gate q"),
                     (b"2 1\n0 0\n0\n", "bad job file"), (b"2 0\n1 h 5\n", "bad job file"),
                     (b"2 0\n1 cx 1 1\n", "bad job file")]:
        assert lib().cz_cliffjob_check(bad, len(bad), C.byref(n), C.byref(t), err, 256) == 2
        assert err.value.decode() == msg


def _run(exe, args, timeout=300):
    p = subprocess.run([str(exe)] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    return p.returncode, strip_seconds(p.stdout.splitlines()), p.stderr.splitlines()


def test_tc_oracle_published_small_targets(oracles):
    """2-qubit published optima (found in the table, split [0, 3]) from the restatement"""
    opt = {c["name"]: c["stdout"] for c in json.loads((GOLD / "tcount" / "optimal.json").read_text())}
    for name in ("cs", "qft_2"):
        rc, out, _ = _run(oracles[0], [GOLD / "tcount" / f"{name}.tspec", "--table", "4"])
        assert rc == 0
        assert out[-1] == opt[name][-1]


def _golden(path):
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    return json.loads(path.read_text())


# reference runs the restatement reproduces in seconds (2 qubits; 3 qubits with the table cut to K <= 2)
SMALL_TC = ["cs-k2", "cs-k4", "qft_2-k2", "qft_2-k4", "toffoli-k1-max3", "toffoli-k2-max4"]


@pytest.mark.parametrize("name", SMALL_TC)
def test_tc_oracle_matches_reference(oracles, name):
    case = {c["name"]: c for c in _golden(TC_GOLD)}[name]
    args = [GOLD / "tcount" / Path(case["args"][0]).name] + case["args"][1:]
    rc, out, _ = _run(oracles[0], args)
    assert rc == case["rc"]
    if not any('"dir": "table"' in l for l in case["stdout"]):   # the reference loaded that table from its cache
        out = [l for l in out if '"dir": "table"' not in l]
    assert out == case["stdout"]


@pytest.mark.parametrize("job", ["c2-0", "c2-1"])
def test_clifford_oracle_matches_reference_2q(oracles, job):
    case = {c["name"]: c for c in _golden(CL_GOLD)}[job]
    rc, out, err = _run(oracles[1], [GOLD / "cliffopt" / f"{job}.job"])
    assert rc == case["rc"] == 0
    assert out == case["stdout"]
    assert [l for l in err if "clifford gates" in l] == [l for l in case["stderr"] if "clifford gates" in l]


def test_clifford_oracle_output_is_equivalent(oracles):
    """the oracle's 2-qubit output circuits implement the job's circuit up to global phase"""
    for job in ("c2-0", "c2-1"):
        text = (GOLD / "cliffopt" / f"{job}.job").read_text()
        rc, out, _ = _run(CL_ORACLE, [GOLD / "cliffopt" / f"{job}.job"])
        assert rc == 0
        assert _same_up_to_phase(2, _job_circuit(text), _lines_circuit(out[1:]))


def _job_circuit(text):
    tok = text.split()
    pos = 0

    def nxt():
        nonlocal pos
        pos += 1
        return tok[pos - 1]
    n, t = int(nxt()), int(nxt())
    ts = [(int(nxt()), int(nxt())) for _ in range(t)]
    circ = []
    for j in range(t + 1):
        m = int(nxt())
        for _ in range(m):
            g = nxt()
            qs = (int(nxt()), int(nxt())) if g == "cx" else (int(nxt()),)
            circ.append((g, qs))
        if j < t:
            circ.append(("tdg" if ts[j][1] else "t", (ts[j][0],)))
    return circ


def _lines_circuit(lines):
    out = []
    for l in lines:
        f = l.split()
        out.append((f[0], tuple(int(x) for x in f[1:])))
    return out


def _same_up_to_phase(n, c1, c2):
    from cheese_b200 import workloads
    k1, A = workloads.unitary(n, _expand_y(c1))
    k2, B = workloads.unitary(n, _expand_y(c2))
    for ph in range(8):
        w = [0, 0, 0, 0]
        w[ph % 4] = 1 if ph < 4 else -1
        if k1 == k2 and all(workloads.zmul(tuple(w), B[r][c]) == A[r][c] for r in range(1 << n) for c in range(1 << n)):
            return True
    return False


def _expand_y(circ):
    out = []
    for g, q in circ:
        if g == "y":                       # Y = i X Z: X then Z up to phase
            out += [("z", q), ("x", q)]
        else:
            out.append((g, q))
    return out
