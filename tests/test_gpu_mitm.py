"""Meet-in-the-middle mode (`cheese SPEC --mitm`, reference src/cheese.cu:1595-1760) on the GPU.

The golden cases were made by the reference CPU build: forward and backward levels ("dir": "fwd" / "bwd"), the join
line, and the circuit with its "mitm" split or the proof line. Through the C ABI and through the drop-in binary the
same stdout lines and exit codes come out; every circuit is verified exactly."""
import json
import re
import subprocess

import pytest

from conftest import GOLD, spec_path, spec_text

pytestmark = pytest.mark.gpu

SECONDS = re.compile(r'"seconds": [0-9.]+')
CASES = json.loads((GOLD / "mitm_cases.json").read_text())


def _flag(case, name, default=None):
    f = case["flags"]
    return int(f[f.index(name) + 1]) if name in f else default


@pytest.fixture(scope="module")
def engine():
    from cheese_b200 import Engine
    return Engine()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_api_matches_reference(engine, case):
    from cheese_b200 import Spec, verify
    sp = Spec(spec_text(case["spec"]))
    d = _flag(case, "--depth", -1)
    out = engine.search(sp, depth=d, dedupe="--no-dedupe" not in case["flags"], mitm=True,
                        table_k=_flag(case, "--table", 0), cache_dir=None)
    assert out.rc == case["rc"], (out.error, out.lines(depth=d if d >= 0 else sp.depth))
    assert out.lines(depth=d if d >= 0 else sp.depth) == case["stdout"]
    if out.rc == 0 and out.circuit:
        assert verify.equivalent(spec_text(case["spec"]), out.circuit)
    assert out.raw.nsym == 1


def test_drop_in_binary(tmp_path):
    import cheese_b200 as cz
    for name in ("toffoli-9-mitm", "cs-5-mitm", "relative-phase-toffoli-9-mitm", "rand-01-mitm", "table-rand-6-mitm",
                 "toffoli-6-mitm", "toffoli-9-mitm-table4"):
        c = next(x for x in CASES if x["name"] == name)
        p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(c["spec"]))] + c["flags"], capture_output=True,
                           text=True, cwd=tmp_path, timeout=300)
        assert p.returncode == c["rc"], p.stderr
        assert [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()] == c["stdout"]
        assert "symmetry classes: 1 group elements" in p.stderr


def test_mitm_agrees_with_plain_search(engine):
    """the verdict and the optimal length equal the plain search's on seeded random targets"""
    from cheese_b200 import workloads
    import random
    rng = random.Random(41)
    for i in range(12):
        n, circ = workloads.random_circuit(rng, L=rng.randint(5, 9))
        text = workloads.make_spec(n, circ, len(circ))
        for d in (len(circ) - 2, len(circ)):
            a = engine.search(text, depth=d)
            b = engine.search(text, depth=d, mitm=True)
            assert a.rc == b.rc, (i, d)
            if a.rc == 0:
                assert len(a.circuit) == len(b.circuit)
