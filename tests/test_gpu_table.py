"""Distance-table mode (`cheese SPEC --table K`, reference src/cheese.cu:1431-1593 and 1804-1838) on the GPU.

Every golden case was made by the reference CPU build in an empty working directory, so it built its table: the
drop-in binary, run the same way, prints the same stdout lines (the "dir": "table" build levels, the search levels,
the circuit with its "table" split or the table proof line), exits the same way and names the same cache file. A
second run in the same directory loads the cache instead (no table lines), and a cache file written by the reference
itself loads too. Every circuit found through the table is verified exactly."""
import json
import re
import shutil
import subprocess

import pytest

from conftest import GOLD, spec_path, spec_text

pytestmark = pytest.mark.gpu

SECONDS = re.compile(r'"seconds": [0-9.]+')
CASES = json.loads((GOLD / "table_cases.json").read_text())


def strip(lines):
    return [SECONDS.sub('"seconds": 0.00', l) for l in lines]


def table_line(stderr):
    tab = [l for l in stderr.splitlines() if l.startswith("table")]
    return re.sub(r"(\(|, )([0-9.]+) s\)", r"\g<1>0.0 s)", tab[0]) if tab else ""


def run_cli(case, cwd):
    import cheese_b200 as cz
    p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(spec_path(case["spec"]))] + case["flags"],
                       capture_output=True, text=True, cwd=cwd, timeout=600)
    return p


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_drop_in_matches_reference(case, tmp_path):
    p = run_cli(case, tmp_path)
    assert p.returncode == case["rc"], p.stderr
    assert strip(p.stdout.splitlines()) == case["stdout"]
    assert table_line(p.stderr) == case["stderr_table"]
    last = json.loads(case["stdout"][-1])
    if case["rc"] == 0:
        from cheese_b200 import verify
        assert verify.equivalent(spec_text(case["spec"]), last["circuit"])
        assert sum(last["table"]) == last["t"]


@pytest.fixture(scope="module")
def engine():
    from cheese_b200 import Engine
    return Engine()


def _depth(case):
    f = case["flags"]
    return int(f[f.index("--depth") + 1]) if "--depth" in f else -1


def test_api_matches_reference(engine):
    """through the C ABI without a cache file: the table is built by the first search that needs it and stays
    resident on the engine, so later searches print no table levels (like a reference run that loaded its cache)"""
    for case in CASES:
        k = int(case["flags"][case["flags"].index("--table") + 1])
        out = engine.search(spec_text(case["spec"]), depth=_depth(case), sym="--no-sym" not in case["flags"],
                            table_k=k, cache_dir=None)
        assert out.rc == case["rc"], (case["name"], out.error)
        d = _depth(case) if _depth(case) >= 0 else None
        want = case["stdout"] if out.table["table_built"] else [l for l in case["stdout"]
                                                                 if not l.startswith('{"dir": "table"')]
        if d is None:
            d = json.loads(case["stdout"][-1]).get("depth")
        assert out.lines(depth=d) == want, case["name"]


def test_cache_roundtrip(tmp_path):
    """a second run in the same directory loads the cache: no table levels, the same answer (the cache directory
    must exist, as for the reference, which writes its table only into an existing build/)"""
    (tmp_path / "build").mkdir()
    for name in ("toffoli-9-table4", "cs-5-table3", "table-rand-5-table4"):
        case = next(c for c in CASES if c["name"] == name)
        first = run_cli(case, tmp_path)
        assert first.returncode == case["rc"]
        second = run_cli(case, tmp_path)
        assert second.returncode == case["rc"], second.stderr
        want = [l for l in case["stdout"] if not l.startswith('{"dir": "table"')]
        assert strip(second.stdout.splitlines()) == want
        assert "(loaded" in table_line(second.stderr)
        built = case["stderr_table"]
        classes = re.search(r"table: (\d+) classes", built).group(1)
        path = re.search(r"cached in (\S+)", built).group(1)
        assert table_line(second.stderr) == f"table {path}: {classes} classes (loaded, 0.0 s)"


def test_reference_cache_file_loads(tmp_path):
    """a table file written by the reference CPU build is read (its keys recomputed) and answers the same"""
    for f in (GOLD / "table").glob("*.bin"):
        (tmp_path / "build").mkdir(exist_ok=True)
        shutil.copy(f, tmp_path / "build" / f.name)
    for name in ("toffoli-7-table3", "ccz-7-table3", "table-rand-0-table3", "cs-5-table3", "table-rand-6-table3"):
        case = next(c for c in CASES if c["name"] == name)
        p = run_cli(case, tmp_path)
        assert p.returncode == case["rc"], p.stderr
        want = [l for l in case["stdout"] if not l.startswith('{"dir": "table"')]
        assert strip(p.stdout.splitlines()) == want
        assert "(loaded" in table_line(p.stderr)
