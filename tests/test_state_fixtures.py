"""The state-target fixtures on the CPU: every circuit the reference CPU build found maps the spec's inputs to the
goal rows exactly (this pins the verifier the GPU tests use), and the random cases' own circuits do too."""
import json

from conftest import GOLD, spec_text

CASES = json.loads((GOLD / "state_cases.json").read_text())


def test_reference_circuits_verify():
    from cheese_b200 import verify
    found = [c for c in CASES if c["rc"] == 0 and json.loads(c["stdout"][-1]).get("circuit")]
    assert len(found) >= 8
    for c in found:
        assert verify.state_equivalent(spec_text(c["spec"]), json.loads(c["stdout"][-1])["circuit"]), c["name"]


def test_generating_circuits_verify():
    from cheese_b200 import verify
    for c in CASES:
        if "circuit" in c:
            names = [f"L_{g}_" + "_".join(map(str, qs)) for g, qs in c["circuit"]]
            assert verify.state_equivalent(spec_text(c["spec"]), names), c["name"]
