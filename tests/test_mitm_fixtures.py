"""The --mitm golden fixtures (made by the reference CPU build) on the CPU: circuits implement their targets exactly,
the "mitm" split adds up to the circuit length, and the join's forward count is the last forward level's."""
import json

from conftest import GOLD, spec_text

CASES = json.loads((GOLD / "mitm_cases.json").read_text())


def test_found_circuits_are_exact():
    from cheese_b200 import verify
    found = [c for c in CASES if c["rc"] == 0]
    assert len(found) >= 30
    for c in found:
        last = json.loads(c["stdout"][-1])
        if last.get("circuit"):
            assert verify.equivalent(spec_text(c["spec"]), last["circuit"]), c["name"]
        if "mitm" in last:
            assert sum(last["mitm"]) == last["t"] == len(last["circuit"])


def test_join_counts():
    for c in CASES:
        lines = [json.loads(l) for l in c["stdout"]]
        join = [l for l in lines if l.get("dir") == "join"]
        if not join:
            continue
        fwd = [l for l in lines if l.get("dir") == "fwd"]
        bwd = [l for l in lines if l.get("dir") == "bwd"]
        assert join[0]["forward"] == fwd[-1]["distinct"]
        assert join[0]["backward"] == sum(l["distinct"] for l in bwd)
