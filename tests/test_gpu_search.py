"""Parity of the sm_100a search with the reference (golden outputs of its CPU build) and with the CPU restatement
(oracle/) on fresh seeded targets. Every call goes through the C ABI (libcheese_b200.so) or the drop-in binary."""
import json
import random
import subprocess

import pytest

import cheese_b200 as cz
from cheese_b200 import verify, workloads
from conftest import (ROOT, case_depth, golden_cases, run_oracle, spec_path, spec_text, strip_seconds)

pytestmark = pytest.mark.gpu
GOLD = {c["name"]: c for c in golden_cases()}
CASES = [c for c in golden_cases() if not c["name"].endswith("store64")]


@pytest.fixture(scope="module")
def engine():
    e = cz.Engine(0)
    yield e
    e.close()


def _flags(case):
    f = case["flags"]
    return dict(depth=case_depth(case), dedupe="--no-dedupe" not in f, sym="--no-sym" not in f)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_matches_reference(engine, case):
    want = case
    if case["name"] == "overflow-4":
        # the reference's default build aborts (exit 4: int32 limbs); this build promotes to int64 limbs and must
        # agree with the reference's -DSTORE64 build
        want = GOLD["overflow-4-store64"]
    out = engine.search(spec_text(case["spec"]), **_flags(case))
    assert out.rc == want["rc"], out.error
    assert out.lines() == want["stdout"]
    if out.rc == 0 and out.circuit:
        assert verify.equivalent(spec_text(case["spec"]), out.circuit)
    if case["name"] == "overflow-4":
        assert out.raw.store64 == 1


def test_forced_int64_limbs_identical(engine):
    for name in ["toffoli-9", "ccz-8", "cs-5", "rand-02", "qft_2-7"]:
        c = GOLD[name]
        a = engine.search(spec_text(c["spec"]), **_flags(c))
        b = engine.search(spec_text(c["spec"]), store64=True, **_flags(c))
        assert b.raw.store64 == 1
        assert (a.rc, a.lines()) == (b.rc, b.lines()) == (c["rc"], c["stdout"])


def test_state_target_met_by_the_empty_circuit(engine):
    """the CS target on inputs |00>, |01> (control 0) is already met: the reference CPU build's depth-0 answer"""
    out = engine.search(spec_text("cs-states"))
    assert out.rc == 0 and out.depth0 and out.lines() == ['{"found": 0, "circuit": []}']


def test_depth_above_limit_is_usage_error(engine):
    out = engine.search(spec_text("toffoli"), depth=49)
    assert out.rc == 3


def _random_specs(seed, count, Lmax):
    rng = random.Random(seed)
    for i in range(count):
        n, circ = workloads.random_circuit(rng, L=rng.randint(4, Lmax))
        yield i, n, circ, workloads.make_spec(n, circ, len(circ))


@pytest.mark.parametrize("sym", [True, False])
def test_random_targets_match_oracle(engine, oracle_bin, tmp_path, sym):
    for i, n, circ, text in _random_specs(4242 + sym, 24, 9):
        p = tmp_path / f"r{i}.spec"
        p.write_text(text)
        rc, lines = run_oracle(oracle_bin, p, [] if sym else ["--no-sym"])
        out = engine.search(text, sym=sym)
        assert out.rc == rc, (i, circ)
        assert out.lines() == lines, (i, circ)
        assert out.rc == 0 and verify.equivalent(text, out.circuit)


def test_tight_budgets_prove_and_loose_budgets_find(engine, oracle_bin, tmp_path):
    # budgets below and above the optimum on the same targets: proofs and circuits agree with the oracle
    for i, n, circ, text in _random_specs(99, 10, 8):
        found = engine.search(text)
        opt = len(found.circuit)
        for d in sorted({max(1, opt - 1), opt, opt + 2}):
            p = tmp_path / f"b{i}.spec"
            p.write_text(text)
            rc, lines = run_oracle(oracle_bin, p, ["--depth", str(d)])
            out = engine.search(text, depth=d)
            assert (out.rc, out.lines()) == (rc, lines), (i, d)


def test_drop_in_binary(tmp_path):
    exe = cz.BIN_DIR / "cheese"
    for name in ["toffoli-9", "cs-5", "relative-phase-toffoli-9", "ccz-8-nosym"]:
        c = GOLD[name]
        p = subprocess.run([str(exe), str(spec_path(c["spec"]))] + c["flags"], capture_output=True, text=True,
                           timeout=300)
        assert p.returncode == c["rc"], p.stderr
        assert strip_seconds(p.stdout.splitlines()) == c["stdout"]
        assert "cheese: n" in p.stderr and "symmetry classes" in p.stderr
    p = subprocess.run([str(exe)], capture_output=True, text=True)
    assert p.returncode == 3 and "usage" in p.stderr
    bad = tmp_path / "bad.spec"
    bad.write_text("cheese-spec 1\nn 3\nwhat 1\n")
    p = subprocess.run([str(exe), str(bad)], capture_output=True, text=True)
    assert p.returncode == 2 and "unknown spec field what" in p.stderr
    p = subprocess.run([str(exe), str(spec_path("toffoli")), "--depth", "60"], capture_output=True, text=True)
    assert p.returncode == 3 and "depth > 48" in p.stderr
    p = subprocess.run([str(exe), str(spec_path("cs-states"))], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout == '{"found": 0, "circuit": []}\n'
    assert "symmetry classes: 1 group elements" in p.stderr


def test_trim_releases_and_search_repeats(engine):
    """trim() frees the cached work buffers; the next search allocates again and answers the same"""
    c = GOLD["toffoli-10"]
    a = engine.search(spec_text(c["spec"]), depth=10)
    assert engine.trim() > 0
    assert engine.trim() == 0
    b = engine.search(spec_text(c["spec"]), depth=10)
    assert (a.rc, a.lines()) == (b.rc, b.lines()) == (c["rc"], c["stdout"])
