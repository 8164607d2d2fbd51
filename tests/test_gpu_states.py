"""State targets (RUS without measurement: the circuit must map every listed input basis state to the target's image,
reference src/cheese.cu:451-583) on the GPU. The reference's GPU binary refuses them; its CPU build searches them,
and the golden cases are that build's output: the reference's RUS targets with their ancillas in |0> and seeded
random circuits on random input sets. Level lines, exit codes and circuits are the same; every circuit is checked
exactly on the inputs."""
import json
import re
import subprocess

import pytest

from conftest import GOLD, spec_path, spec_text

pytestmark = pytest.mark.gpu

SECONDS = re.compile(r'"seconds": [0-9.]+')
CASES = json.loads((GOLD / "state_cases.json").read_text())


@pytest.fixture(scope="module")
def engine():
    from cheese_b200 import Engine
    return Engine()


def _depth(case):
    return int(case["flags"][case["flags"].index("--depth") + 1])


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_matches_reference_cpu_build(engine, case):
    from cheese_b200 import verify
    text = spec_text(case["spec"])
    out = engine.search(text, depth=_depth(case))
    assert out.rc == case["rc"], out.error
    assert out.lines() == case["stdout"]
    assert out.raw.nsym == 1
    if out.rc == 0 and out.circuit:
        assert verify.state_equivalent(text, out.circuit)


def test_drop_in_binary(tmp_path):
    import cheese_b200 as cz
    for name in ("rus2-states-7", "rus1-states-9", "states-rand-4-5", "rus7-states-5"):
        c = next(x for x in CASES if x["name"] == name)
        p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(c["spec"]))] + c["flags"], capture_output=True,
                           text=True, cwd=tmp_path, timeout=300)
        assert p.returncode == c["rc"], p.stderr
        assert [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()] == c["stdout"]
        assert "symmetry classes: 1 group elements" in p.stderr


def test_mitm_refused_for_state_targets(tmp_path):
    """the reference's --mitm takes unitary targets only (exit 3); --table is ignored for state targets"""
    import cheese_b200 as cz
    c = next(x for x in CASES if x["name"] == "rus2-states-7")
    p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(c["spec"])), "--depth", "7", "--mitm"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert p.returncode == 3 and "--mitm: unitary targets only" in p.stderr
    p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(c["spec"])), "--depth", "7", "--table", "3"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert p.returncode == c["rc"]
    assert [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()] == c["stdout"]
