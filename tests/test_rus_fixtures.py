"""RUS T-count fixtures (the reference's build/rus, src/rus.cu) on the CPU: the C restatement reproduces every
committed case, the case set holds the reference's own pins (tests/rus_check.sh optima, the 692 cosets of table level
4 published in its docs), the per-node arithmetic of the sm_100a path (cz_rus_node.h, compiled for the host) driven
through the GPU path's level flow gives the same lines, and the library parses rus-specs like the reference's
read_spec."""
import json
import subprocess

import pytest

from conftest import GOLD, ORACLE_DIR, ROOT, rus_cases, rus_spec_text

CASES = rus_cases()
RUS_ORACLE = ORACLE_DIR / "_ref" / "rus-oracle"


@pytest.fixture(scope="module")
def specs(tmp_path_factory):
    d = tmp_path_factory.mktemp("rspec")
    out = {}
    for t in {c["target"] for c in CASES}:
        out[t] = d / f"{t}.rspec"
        out[t].write_text(rus_spec_text(t))
    return out


@pytest.fixture(scope="module")
def rus_oracle():
    if not RUS_ORACLE.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "_ref/rus-oracle"], check=True, capture_output=True)
    return RUS_ORACLE


def test_reference_pins():
    """the reference's regression verdicts (tests/rus_check.sh) and its level-4 table size"""
    by = {c["name"]: c for c in CASES}
    assert json.loads(by["ricotta-rus-0003-k4-max3"]["stdout"][-1]) == {"tcount_above": 3, "seconds": 0.0}
    assert json.loads(by["ricotta-rus-0003-k1-max3"]["stdout"][-1]) == {"tcount_above": 3, "seconds": 0.0}
    assert json.loads(by["ricotta-rus-0229-k7-max11"]["stdout"][-1])["tcount"] == 10
    assert json.loads(by["ricotta-rus-0229-k5-max11"]["stdout"][-1])["tcount"] == 10
    lvl4 = [json.loads(l) for l in by["ricotta-rus-0003-k4-max3"]["stdout"] if '"dir": "table", "t": 4' in l][0]
    assert lvl4["new"] == 692
    assert all(c["verified"] for c in CASES if c["rc"] == 0)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_reproduces(case, specs, rus_oracle):
    p = subprocess.run([str(rus_oracle), str(specs[case["target"]])] + case["flags"], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == case["rc"]
    assert p.stdout.splitlines() == case["stdout"]


def test_host_compiled_node_arithmetic(specs, tmp_path):
    exe = tmp_path / "rus-host-check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", str(exe), str(ROOT / "tests" / "rus_host_check.cpp")], check=True)
    for case in CASES:
        if case["name"] == "ricotta-rus-0229-k5-max11":
            continue                         # the slowest case (2.2M children at search level 5): GPU tests only
        p = subprocess.run([str(exe), str(specs[case["target"]])] + case["flags"], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == case["rc"], case["name"]
        assert p.stdout.splitlines() == case["stdout"], case["name"]


def test_spec_check():
    import ctypes as C
    import cheese_b200 as cz
    L = cz.lib()
    n, err = C.c_int(), C.create_string_buffer(256)
    text = rus_spec_text("ricotta-rus-0229").encode()
    assert L.cz_rspec_check(text, len(text), C.byref(n), err, 256) == 0 and n.value == 12
    bad = [(b"tcount-spec 1\nend\n", "not a rus spec"), (b"rus-spec 1\nroots 0\nend\n", "incomplete spec"),
           (b"rus-spec 1\nfoo 3\nend\n", "unknown field foo"),
           (text.replace(b"cliffords 11520", b"cliffords 11519"), "expected 11520 Cliffords")]
    for t, msg in bad:
        assert L.cz_rspec_check(t, len(t), C.byref(n), err, 256) == 2, msg
        assert err.value.decode() == msg


def test_bench_reads_the_same_specs():
    import bench
    for t in {c["target"] for c in CASES}:
        assert bench.rus_spec(t) == rus_spec_text(t)


SPEC_CASES = json.loads((GOLD / "rus_spec_cases.json").read_text())


@pytest.mark.parametrize("case", SPEC_CASES, ids=[c["name"] for c in SPEC_CASES])
def test_rspec_writer_matches_reference(case):
    """the C++ writer of rus-specs (roots, table root, rotation tables, Clifford list) byte for byte as the
    reference's rus.py writes them, with the same summary (success outcome, roots, Pr[success], rescalings)"""
    import gzip
    import cheese_b200 as cz
    with gzip.open(GOLD / "rus" / "common.rspec.gz", "rt") as f:
        root, rest = f.read().split("\n@@\n")
    text, info = cz.rspec_generate(qasm=case["qasm"])
    assert text == "rus-spec 1\n" + root + case["roots"] + rest + "end\n"
    assert info == case["info"]


def test_rspec_writer_cli_and_errors(tmp_path):
    import cheese_b200 as cz
    case = next(c for c in SPEC_CASES if c["name"] == "ricotta-rus-0229-v2")
    q = tmp_path / "v.qasm"
    q.write_text(case["qasm"])
    p = subprocess.run([str(cz.BIN_DIR / "cheese-spec"), "--rus", str(q)], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout == cz.rspec_generate(qasm=case["qasm"])[0]
    assert json.loads(p.stderr) == case["info"]
    with pytest.raises(cz.SpecError) as e:
        cz.rspec_generate(3, [("h", (0,))])
    assert e.value.rc == 2 and "two qubits" in str(e.value)
    with pytest.raises(cz.SpecError) as e:
        cz.rspec_generate(2, [("h", (0,)), ("t", (1,))])
    assert e.value.rc == 2 and "not a RUS circuit" in str(e.value)


def test_variants_keep_the_optimum(tmp_path, rus_oracle):
    """Cliffords on either side are free: the C restatement finds the targets' optima for the derived circuits"""
    import cheese_b200 as cz
    for name, flags, last in (("ricotta-rus-0003-v1", ["--table", "4", "--max", "3"], {"tcount_above": 3}),
                              ("ricotta-rus-0003-v2", ["--table", "3", "--max", "4"], {"tcount": 4}),
                              ("ricotta-rus-0229-v3", ["--table", "7", "--max", "11"], {"tcount": 10})):
        case = next(c for c in SPEC_CASES if c["name"] == name)
        spec = tmp_path / f"{name}.rspec"
        spec.write_text(cz.rspec_generate(qasm=case["qasm"])[0])
        p = subprocess.run([str(rus_oracle), str(spec)] + flags, capture_output=True, text=True, timeout=600)
        got = json.loads(p.stdout.splitlines()[-1])
        assert {k: got[k] for k in last} == last, name


def test_drop_in_rejects_before_the_device(tmp_path):
    """usage and spec errors are reported before any device work (the reference reads its spec before CUDA setup),
    so they behave the same on a host without a GPU"""
    import cheese_b200 as cz
    p = subprocess.run([str(cz.BIN_DIR / "rus")], capture_output=True, text=True)
    assert p.returncode == 3 and p.stderr.startswith("usage: rus SPEC")
    for text, msg in (("rus-spec 1\nroots 0\nend\n", "incomplete spec"), ("cheese-spec 1\n", "not a rus spec"),
                      ("rus-spec 1\nmystery 1\nend\n", "unknown field mystery")):
        f = tmp_path / "bad.rspec"
        f.write_text(text)
        p = subprocess.run([str(cz.BIN_DIR / "rus"), str(f)], capture_output=True, text=True)
        assert p.returncode == 2 and p.stderr.strip() == msg


def test_found_circuits_verify_exactly():
    """every found circuit of the fixtures passes the exact RUS check of cheese_b200.verify (the role of the
    reference's `rus.py verify`), and damaged results do not"""
    from cheese_b200 import verify
    from conftest import rus_spec_text
    qasm = {c["name"]: c["qasm"] for c in SPEC_CASES}
    found = [c for c in CASES if c["rc"] == 0]
    assert len(found) == 7
    for c in found:
        cl = verify.rspec_cliffords(rus_spec_text(c["target"]))
        assert verify.rus_check(qasm[c["target"]], json.loads(c["stdout"][-1]), cl), c["name"]
    res = json.loads(found[-1]["stdout"][-1])
    cl = verify.rspec_cliffords(rus_spec_text(found[-1]["target"]))
    for damage in ({"cliff": (res["cliff"] + 1) % 11520}, {"tb": res["tb"][:-1]}, {"fw": res["fw"][1:] + [1]},
                   {"tcount": res["tcount"] - 1}):
        assert not verify.rus_check(qasm[found[-1]["target"]], {**res, **damage}, cl), damage


def test_clifford_words_realise_the_spec_list():
    """the gate word built for an entry of a rus-spec's Clifford list has that entry's Pauli action exactly"""
    import random
    from conftest import rus_spec_text
    from cheese_b200.workloads import matmul, unitary
    cl = verify_mod().rspec_cliffords(rus_spec_text(CASES[0]["target"]))
    assert len(cl) == 11520
    P = [verify_mod()._pauli(2, p) for p in range(16)]
    for i in list(range(40)) + random.Random(3).sample(range(11520), 200):
        U = unitary(2, verify_mod().clifford_word(cl[i]))
        Ud = verify_mod()._adj(U)
        for a in range(16):
            b, s = cl[i][0][a], cl[i][1][a]
            assert matmul(matmul(Ud, P[a]), U) == (0, [[tuple(s * v for v in x) for x in r] for r in P[b][1]]), i


def verify_mod():
    from cheese_b200 import verify
    return verify
