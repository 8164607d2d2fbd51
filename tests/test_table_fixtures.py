"""The --table K golden fixtures (made by the reference CPU build) on the CPU: every circuit found through the table
implements its target exactly, its "table" split adds up, the build levels count the classes of the stderr line, and
the committed reference cache files hold the class counts of those lines."""
import json
import re
import struct

from conftest import GOLD, spec_text

CASES = json.loads((GOLD / "table_cases.json").read_text())


def test_found_circuits_are_exact():
    from cheese_b200 import verify
    found = [c for c in CASES if c["rc"] == 0]
    assert len(found) >= 8
    for c in found:
        last = json.loads(c["stdout"][-1])
        assert verify.equivalent(spec_text(c["spec"]), last["circuit"]), c["name"]
        assert sum(last["table"]) == last["t"] == len(last["circuit"])


def test_build_levels_count_the_table():
    for c in CASES:
        tab = [json.loads(l) for l in c["stdout"] if l.startswith('{"dir": "table"')]
        classes = int(re.search(r"table: (\d+) classes within (\d+) gates", c["stderr_table"]).group(1))
        k = int(c["flags"][c["flags"].index("--table") + 1])
        assert [t["t"] for t in tab] == list(range(1, k + 1))
        assert 1 + sum(t["distinct"] for t in tab) == classes, c["name"]


def test_proof_lines():
    for c in CASES:
        last = json.loads(c["stdout"][-1])
        if "table" in last and "depth" in last:
            assert c["rc"] == 1 and last["proved_unsat"] is True
            assert last["depth"] == int(c["flags"][c["flags"].index("--depth") + 1])


def test_reference_cache_files():
    """the key count of each committed reference table file equals the classes the reference reported building it"""
    built = {re.search(r"cached in build/(\S+)", c["stderr_table"]).group(1):
             int(re.search(r"table: (\d+) classes", c["stderr_table"]).group(1)) for c in CASES}
    files = sorted((GOLD / "table").glob("*.bin"))
    assert files
    for f in files:
        b = f.read_bytes()
        assert f.name in built
        assert built[f.name] * 24 < len(b)
