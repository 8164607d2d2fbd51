"""The C++ spec generators (host code, no GPU) against the reference's own writers: every spec file the reference's
python/cheese/spec.py wrote for a fixture circuit is reproduced line for line, except that the W3 triples of one
(first, second) pair may come in another order (the reference lists them in Python set order; the set is the same),
every T-count spec its tcount.py wrote is reproduced byte for byte, and so is every state-target spec (mode states)."""
import json
import random
import subprocess

import pytest

from conftest import GOLD, spec_path

CASES = json.loads((GOLD / "spec_circuits.json").read_text())


def parts(text):
    """(lines up to the bad3 header, the bad3 lines sorted, the lines after them)"""
    L = text.splitlines()
    i = next(j for j, l in enumerate(L) if l.startswith("bad3 "))
    n = int(L[i].split()[1])
    return L[:i + 1], sorted(L[i + 1:i + 1 + n]), L[i + 1 + n:]


def circ_of(c):
    return [(g, tuple(q)) for g, q in c["circuit"]]


@pytest.mark.parametrize("name", sorted(CASES))
def test_spec_matches_reference_writer(name):
    import cheese_b200 as cz
    c = CASES[name]
    text, info = cz.spec_generate(c["n"], circ_of(c), depth=c["depth"], w3=c.get("w3", True))
    want = spec_path(name).read_text()
    assert parts(text) == parts(want)
    assert info["candidates"] == int(want.split("\ngates ")[1].split()[0])
    if "qasm" in c:
        text2, _ = cz.spec_generate(qasm=c["qasm"], depth=c["depth"])
        assert text2 == text


def test_random_targets_match_reference_writer():
    """the seeded random targets of the golden cases (2 and 3 qubits) and the distance-table cases"""
    import cheese_b200 as cz
    cases = [c for c in json.loads((GOLD / "cases.json").read_text()) if "circuit" in c]
    cases += [c for c in json.loads((GOLD / "table_cases.json").read_text()) if "circuit" in c]
    assert len(cases) >= 30
    for c in cases:
        want = spec_path(c["spec"]).read_text()
        n = int(want.split("\nn ")[1].split()[0])
        depth = int(want.split("\ndepth ")[1].split()[0])
        text, _ = cz.spec_generate(n, circ_of(c), depth=depth)
        assert parts(text) == parts(want), c["name"]


def test_same_as_reference_base_spec_with_python_target():
    """the native writer against the reference-written base spec of each qubit count with the target block that the
    Python exact arithmetic (workloads.unitary) gives: the same candidates, rules, cuts, CX table and target"""
    from cheese_b200 import workloads
    base = {n: spec_path(f"base-n{n}").read_text() for n in (2, 3)}
    for n, circ, d in workloads.batch(3, 40):
        k, M = workloads.unitary(n, circ)
        head, rest = base[n].split("target ", 1)
        head = "".join(f"depth {d}\n" if ln.startswith("depth ") else ln for ln in head.splitlines(keepends=True))
        target = f"target {k}\n" + "".join(" ".join(" ".join(map(str, x)) for x in row) + "\n" for row in M)
        want = head + target + rest[rest.index("cuts "):]
        assert parts(workloads.make_spec(n, circ, d)) == parts(want)


@pytest.mark.parametrize("name", ["cs", "qft_2", "toffoli", "ccz", "fredkin", "peres", "relative-phase-toffoli"])
def test_tspec_matches_reference_writer(name):
    import cheese_b200 as cz
    c = CASES[name]
    assert cz.tspec_generate(c["n"], circ_of(c)) == (GOLD / "tcount" / f"{name}.tspec").read_text()
    assert cz.tspec_generate(qasm=c["qasm"]) == (GOLD / "tcount" / f"{name}.tspec").read_text()


def test_tspec_of_seeded_queries():
    """the seeded T-count queries of the golden cases (circuits re-drawn from their seed)"""
    import cheese_b200 as cz
    from cheese_b200 import tcwork
    rng = random.Random(4096)
    for i in range(8):
        circ, _ = tcwork.tcount_query(rng, 3)
        assert cz.tspec_generate(3, circ) == (GOLD / "tcount" / f"q3-{i}.tspec").read_text()
    for i in range(4):
        circ, _ = tcwork.tcount_query(rng, 2)
        assert cz.tspec_generate(2, circ) == (GOLD / "tcount" / f"q2-{i}.tspec").read_text()


def test_errors():
    import cheese_b200 as cz
    with pytest.raises(cz.SpecError) as e:
        cz.spec_generate(3, [("u3", (0,))], depth=4)
    assert e.value.rc == 2 and "unknown gate u3" in str(e.value)
    with pytest.raises(cz.SpecError) as e:
        cz.spec_generate(2, [("cx", (0, 2))], depth=4)
    assert e.value.rc == 2 and "out of range" in str(e.value)
    with pytest.raises(cz.SpecError) as e:
        cz.spec_generate(qasm="OPENQASM 2.0;\nh q[0];\n", depth=4)
    assert e.value.rc == 2 and "no qubit register" in str(e.value)


def test_cli(tmp_path):
    import cheese_b200 as cz
    c = CASES["toffoli"]
    q = tmp_path / "toffoli.qasm"
    q.write_text(c["qasm"])
    p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), str(q), str(c["depth"])], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    want = spec_path("toffoli").read_text()
    assert parts(p.stdout) == parts(want)
    nb2 = int(want.split("\nbad2 ")[1].split()[0])
    nb3 = int(want.split("\nbad3 ")[1].split()[0])
    assert p.stderr.strip() == f"toffoli: 3 qubits, 27 candidates, W2 pairs {nb2}, W3 triples {nb3}"
    p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), "--tcount", str(q)], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout == (GOLD / "tcount" / "toffoli.tspec").read_text()
    # state targets: --ancilla (every basis state with qubit 2 in |0>) and the same inputs listed with --inputs
    st = next(c for c in STATE_CASES if c["name"] == "toffoli-anc2")
    for flags in (["--ancilla", "2"], ["--inputs", ",".join(map(str, st["inputs"]))]):
        p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), str(q), str(st["depth"]), "--no-w3"] + flags,
                           capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        assert p.stdout == st["spec"]
    p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), str(q), "5", "--inputs", "0,8"], capture_output=True,
                       text=True)
    assert p.returncode == 2 and "input 8 out of range" in p.stderr
    p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), str(q), "5", "--ancilla"], capture_output=True, text=True)
    assert p.returncode == 2 and p.stderr.startswith("usage")


STATE_CASES = json.loads((GOLD / "state_spec_cases.json").read_text())


@pytest.mark.parametrize("case", STATE_CASES, ids=[c["name"] for c in STATE_CASES])
def test_state_spec_matches_reference_writer(case):
    """state-target specs (start and goal rows, per goal row its sde, stabilizer nullity and Schmidt ranks) byte for
    byte as the reference's generator wrote them"""
    import cheese_b200 as cz
    circ = [(g, tuple(q)) for g, q in case["circuit"]]
    text, info = cz.spec_generate(case["n"], circ, depth=case["depth"], w3=False, inputs=case["inputs"])
    assert text == case["spec"]
    if case["ancilla"]:
        assert cz.state_inputs(case["n"], case["ancilla"]) == case["inputs"]


def test_state_specs_of_search_fixtures():
    """the state-target specs that the GPU search fixtures use (reference-written, W3 on): the seeded random
    circuits on random input sets, and CS with its ancilla in |0>"""
    import cheese_b200 as cz
    cases = [c for c in json.loads((GOLD / "state_cases.json").read_text()) if "inputs" in c]
    assert len(cases) == 6
    for c in cases:
        want = spec_path(c["spec"]).read_text()
        n = int(want.split("\nn ")[1].split()[0])
        depth = int(want.split("\ndepth ")[1].split()[0])
        text, _ = cz.spec_generate(n, circ_of(c), depth=depth, inputs=c["inputs"])
        assert parts(text) == parts(want), c["name"]
    cs = CASES["cs"]
    text, _ = cz.spec_generate(cs["n"], circ_of(cs), depth=5, inputs=[0, 1])
    assert parts(text) == parts(spec_path("cs-states").read_text())


def test_state_spec_errors():
    import cheese_b200 as cz
    with pytest.raises(cz.SpecError) as e:
        cz.spec_generate(2, [("h", (0,))], depth=3, inputs=[0, 4])
    assert e.value.rc == 2 and "input 4 out of range" in str(e.value)
    with pytest.raises(cz.SpecError) as e:
        cz.spec_generate(1, [("h", (0,))], depth=3, inputs=[0, 1, 0])
    assert e.value.rc == 2 and "3 inputs for 2 basis states" in str(e.value)
