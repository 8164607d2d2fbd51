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
