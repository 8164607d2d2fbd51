"""Host-side workload generation and exact verification (no GPU)."""
import json
import random

from cheese_b200 import verify, workloads
from conftest import golden_cases, spec_text


def test_spec_assembly_matches_reference_writer():
    # the golden random specs were written by the reference's spec generator for these circuits; the W3 triples are
    # the same set (the reference lists them in the iteration order of a Python set)
    from test_specgen import parts
    for c in golden_cases():
        if "circuit" not in c:
            continue
        circ = [(g, tuple(q)) for g, q in c["circuit"]]
        n = 3 if "L_cx_0_2" in spec_text(c["spec"]) else 2
        assert parts(workloads.make_spec(n, circ, len(circ))) == parts(spec_text(c["spec"])), c["name"]


def test_found_circuits_in_golden_outputs_verify_exactly():
    seen = 0
    for c in golden_cases():
        if c["rc"] != 0:
            continue
        line = json.loads(c["stdout"][-1])
        if not line["circuit"]:
            continue
        assert verify.equivalent(spec_text(c["spec"]), line["circuit"]), c["name"]
        seen += 1
    assert seen >= 20


def test_wrong_circuit_does_not_verify():
    c = next(c for c in golden_cases() if c["name"] == "cs-5")
    circ = json.loads(c["stdout"][-1])["circuit"]
    assert not verify.equivalent(spec_text("cs"), circ[:-1])
    assert not verify.equivalent(spec_text("cs"), circ[1:] + circ[:1])


def test_batch_is_seeded_and_in_range():
    a, b = workloads.batch(5, 64), workloads.batch(5, 64)
    assert a == b
    for n, circ, d in a:
        assert n in (2, 3) and 6 <= d <= 12 and len(circ) == d
        for g, qs in circ:
            assert all(0 <= q < n for q in qs)
            if g == "cx":
                assert qs[0] != qs[1]
    frac_t = sum(g in ("t", "tdg") for _, c, _ in a for g, _ in c) / sum(len(c) for _, c, _ in a)
    assert 0.2 < frac_t < 0.4
