"""T-count path on the GPU through the C ABI: bit-exact against the reference's own outputs (its published optimal
decompositions and its runs on the same tcount-specs), every decomposition verified exactly, and the drop-in
binary's table cache."""
import json
import os
import random
import re
import subprocess

import pytest

from conftest import GOLD, ROOT, strip_seconds
from test_tcount import TARGETS, TC_GOLD

pytestmark = pytest.mark.gpu

BIN = ROOT / "cheese_b200" / "bin" / "tcount"


@pytest.fixture(scope="module")
def eng():
    from cheese_b200 import Engine
    return Engine()


def lines(levels, rc, res):
    out = []
    for l in levels:
        out.append(f'{{"dir": "{"table" if l["table"] else "search"}", "t": {l["t"]}, "parents": {l["parents"]}, '
                   f'"children": {l["children"]}, "cosets": {l["cosets"]}, "new": {l["fresh"]}, "seconds": 0.00}}')
    if rc == 0:
        rot = ", ".join(f"[{p}, {i}]" for p, i in res["rotations"])
        out.append(f'{{"tcount": {res["tcount"]}, "rotations": [{rot}], "split": [{res["split_j"]}, '
                   f'{res["split_c"]}], "seconds": 0.00}}')
    elif rc == 1:
        out.append(f'{{"tcount_above": {res["maxt"]}, "seconds": 0.00}}')
    return out


def unitary_of(name):
    """the exact unitary behind a tcount-spec fixture, when this test file knows it"""
    from cheese_b200 import tcwork
    if name in TARGETS:
        return TARGETS[name]
    m = re.fullmatch(r"q([23])-(\d)", name)
    if not m:
        return None
    rng = random.Random(4096)
    qs = [tcwork.tcount_query(rng, 3) for _ in range(8)] + [tcwork.tcount_query(rng, 2) for _ in range(4)]
    from cheese_b200 import workloads
    n, i = int(m.group(1)), int(m.group(2))
    circ, _ = qs[i] if n == 3 else qs[8 + i]
    return n, workloads.unitary(n, circ)


def spec_text(name):
    return (GOLD / "tcount" / f"{name}.tspec").read_text()


@pytest.mark.parametrize("name", ["cs", "qft_2", "toffoli", "ccz", "fredkin", "peres", "relative-phase-toffoli"])
def test_published_optimum(eng, name):
    """the reference's benchmarks/optimal output (K = 4 table loaded): same search levels, same decomposition"""
    want = {c["name"]: c["stdout"] for c in json.loads((GOLD / "tcount" / "optimal.json").read_text())}[name]
    rc, levels, res = eng.tcount(spec_text(name), table_k=4, cache_dir=None)
    assert rc == 0, res["error"]
    got = lines([l for l in levels if not l["table"]], rc, res)
    assert got == want
    u = unitary_of(name)
    if u:
        from cheese_b200 import tcwork
        assert tcwork.verify_decomposition(u[0], u[1], res["rotations"])


def _cases():
    if not TC_GOLD.exists():
        return []
    return [c for c in json.loads(TC_GOLD.read_text()) if c["rc"] in (0, 1)]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_reference_runs(eng, case):
    """the reference's own runs on these specs: every search level, the result line, the table size; table levels
    too where both this run and the reference's built the table"""
    args = case["args"]
    name = os.path.basename(args[0])[:-len(".tspec")]
    K = int(args[args.index("--table") + 1]) if "--table" in args else 4
    maxt = int(args[args.index("--max") + 1]) if "--max" in args else 16
    rc, levels, res = eng.tcount(spec_text(name), table_k=K, maxt=maxt, cache_dir=None)
    assert rc == case["rc"], res["error"]
    want = case["stdout"]
    want_table = [l for l in want if l.startswith('{"dir": "table"')]
    got = lines(levels, rc, res)
    if res["table_built"] and want_table:
        assert got == want
    else:
        assert [l for l in got if not l.startswith('{"dir": "table"')] == \
               [l for l in want if not l.startswith('{"dir": "table"')]
    for l in case["stderr"]:
        m = re.search(r"table: (\d+) cosets", l) or re.search(r"table \S+: (\d+) cosets", l)
        if m:
            assert res["table_cosets"] == int(m.group(1))
    if rc == 0:
        u = unitary_of(name)
        if u:
            from cheese_b200 import tcwork
            assert tcwork.verify_decomposition(u[0], u[1], res["rotations"])
            assert not tcwork.verify_decomposition(u[0], u[1], res["rotations"][:-1])


def test_resident_table_same_answers(eng):
    """a second query against the resident table answers exactly like the first"""
    a = eng.tcount(spec_text("cs"), table_k=4, cache_dir=None)
    b = eng.tcount(spec_text("cs"), table_k=4, cache_dir=None)
    assert b[2]["table_resident"] == 1
    assert lines(a[1], a[0], a[2])[-1] == lines(b[1], b[0], b[2])[-1]


def test_cli_cache_roundtrip(tmp_path):
    """build/tcount-table-n2-k4.cz.bin is written by the first run and read by the second; same stdout"""
    (tmp_path / "build").mkdir()
    spec = GOLD / "tcount" / "q2-1.tspec"
    p1 = subprocess.run([str(BIN), str(spec), "--table", "4"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert p1.returncode in (0, 1), p1.stderr
    assert "cached in" in p1.stderr
    assert (tmp_path / "build" / "tcount-table-n2-k4.cz.bin").exists()
    p2 = subprocess.run([str(BIN), str(spec), "--table", "4"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert p2.returncode == p1.returncode
    assert "loaded" in p2.stderr
    search = lambda out: [l for l in strip_seconds(out.splitlines()) if '"dir": "table"' not in l]
    assert search(p2.stdout) == search(p1.stdout)


def test_cli_errors(tmp_path):
    bad = tmp_path / "bad.tspec"
    bad.write_text("tcount-spec 1\nn 5\nend\n")
    p = subprocess.run([str(BIN), str(bad)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 3
    p = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 3 and "usage" in p.stderr
