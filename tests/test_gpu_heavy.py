"""The large-frontier regime against the reference itself (tests/golden/heavy_cases.json, made by
tests/golden/make_golden_heavy.py): seeded random 3-qubit targets of 12 gates at budget 12 whose levels reach 1e7 to
4.4e7 prefixes and 1e6 to 8.4e6 survivors, Toffoli budget 12 without symmetry classes, and --table 8 runs (Fredkin
budgets 15 and 16, whose deepest levels hold 1e8 prefixes and 7e7 survivors, and the Toffoli optimum 15). Every
case was run by the reference's own sm_100a build (some also by its CPU build, which agrees line for line); the
library must print the same lines and exit the same way, and every circuit it finds is verified exactly."""
import json
import re
import subprocess

import pytest

from conftest import GOLD, spec_path, spec_text

SECONDS = re.compile(r'"seconds": [0-9.]+')
CASES = json.loads((GOLD / "heavy_cases.json").read_text())
SEARCH = [c for c in CASES if "--table" not in c["flags"]]
TABLE = [c for c in CASES if "--table" in c["flags"]]


def depth(c):
    return int(c["flags"][c["flags"].index("--depth") + 1])


def test_fixtures_cover_the_large_frontier_regime():
    """the committed cases reach the sizes the dedupe is built for, and their circuits are exact"""
    from cheese_b200 import verify
    levels = [json.loads(l) for c in CASES for l in c["stdout"] if '"prefixes"' in l]
    assert max(l["prefixes"] for l in levels) >= 1e8
    assert sum(l["prefixes"] >= 1e7 for l in levels) >= 10
    assert max(l["survivors"] for l in levels if l.get("dir") != "table") >= 5e6
    found = 0
    for c in CASES:
        last = json.loads(c["stdout"][-1])
        if c["rc"] == 0:
            assert verify.equivalent(spec_text(c["spec"]), last["circuit"]), c["name"]
            found += 1
    assert found >= 10


@pytest.fixture(scope="module")
def engine():
    import cheese_b200 as cz
    e = cz.Engine(0)
    yield e
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", SEARCH, ids=[c["name"] for c in SEARCH])
def test_search_matches_reference(engine, case):
    from cheese_b200 import verify
    out = engine.search(spec_text(case["spec"]), depth=depth(case), sym="--no-sym" not in case["flags"])
    assert out.rc == case["rc"], out.error
    assert out.lines() == case["stdout"]
    if out.rc == 0:
        assert verify.equivalent(spec_text(case["spec"]), out.circuit)
    engine.trim()


@pytest.mark.gpu
@pytest.mark.parametrize("case", TABLE, ids=[c["name"] for c in TABLE])
def test_table_drop_in_matches_reference(case, tmp_path):
    import cheese_b200 as cz
    from cheese_b200 import verify
    p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(case["spec"]))] + case["flags"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=900)
    assert p.returncode == case["rc"], p.stderr
    assert [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()] == case["stdout"]
    tab = [l for l in p.stderr.splitlines() if l.startswith("table")]
    assert (re.sub(r"(\(|, )([0-9.]+) s\)", r"\g<1>0.0 s)", tab[0]) if tab else "") == case["stderr_table"]
    if case["rc"] == 0:
        assert verify.equivalent(spec_text(case["spec"]), json.loads(case["stdout"][-1])["circuit"])
