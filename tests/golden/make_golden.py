"""Generate the golden fixtures of the gate-count search from the reference itself.

Run in a container that has the reference source tree (read-only is fine) and the reference CPU build
(`make -C oracle`, which compiles it from the reference's own sources into oracle/_ref/):

    python tests/golden/make_golden.py --ref /path/to/reference [--quick]

Writes
  tests/golden/specs/<name>.spec        spec files written by the reference's spec generator (python/cheese/spec.py)
  tests/golden/cases.json               per case: spec, flags, exit code and the reference's stdout with every
                                        "seconds" value replaced by 0.00 (machine dependent, never compared)
  tests/golden/mitm_cases.json          the same for --mitm runs
  tests/golden/state_cases.json         the same for state targets (RUS without measurement), reference CPU build
  tests/golden/state_spec_cases.json    state-target specs written by the reference's generator (circuit, inputs,
                                        spec text) for the C++ generator
  tests/golden/spec_circuits.json       the reference's qasm targets (circuit, budget) and extra reference-written
                                        specs (W3 off, ccx, cz / y gate sets) for the C++ spec generator
  tests/golden/table_cases.json         the same for --table K runs, each in a fresh working directory (so the
                                        reference builds its distance table and prints the "dir": "table" lines),
                                        plus the reference's stderr table line
The reference is used only here, to produce data; nothing at test time reads the reference tree.
"""
import argparse
import io
import json
import random
import re
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
GOLD = ROOT / "tests" / "golden"
SECONDS = re.compile(r'"seconds": [0-9.]+')

# (case name, target qasm stem, budget, extra flags): the reference's own regression verdicts (tests/check.sh),
# its bench list (tests/bench.sh) and the deep proofs of the benchmark configuration
CASES = [
    ("cs-4", "cs", 4, []), ("cs-5", "cs", 5, []),
    ("ccz-7", "ccz", 7, []), ("ccz-8", "ccz", 8, []), ("ccz-8-nosym", "ccz", 8, ["--no-sym"]),
    ("qft_2-6", "qft_2", 6, []), ("qft_2-7", "qft_2", 7, []),
    ("relative-phase-toffoli-9", "relative-phase-toffoli", 9, []),
    ("toffoli-7-nodedupe", "toffoli", 7, ["--no-dedupe"]),
    ("toffoli-9-nosym", "toffoli", 9, ["--no-sym"]),
    ("fredkin-9", "fredkin", 9, []), ("peres-9", "peres", 9, []), ("half_adder_3-9", "half_adder_3", 9, []),
] + [(f"toffoli-{d}", "toffoli", d, []) for d in range(1, 11)]
SLOW = [("grover_3-10", "grover_3", 10, []), ("toffoli-11", "toffoli", 11, []), ("toffoli-12", "toffoli", 12, []),
        ("toffoli-11-nosym", "toffoli", 11, ["--no-sym"])]


# --table K cases (reference cheese.cu:1804-1838): proofs through the table, proofs by a level, and circuits found
# in the table; (case name, target stem, budget, K, extra flags)
TABLE_CASES = [
    ("toffoli-7-table3", "toffoli", 7, 3, []), ("toffoli-9-table4", "toffoli", 9, 4, []),
    ("toffoli-10-table5", "toffoli", 10, 5, []), ("ccz-8-table4", "ccz", 8, 4, []),
    ("ccz-7-table3", "ccz", 7, 3, []), ("toffoli-9-table4-nosym", "toffoli", 9, 4, ["--no-sym"]),
    ("cs-5-table3", "cs", 5, 3, []), ("qft_2-7-table3", "qft_2", 7, 3, []),
]


# --mitm cases (reference cheese.cu:1595-1760): proofs through the join, proofs by a forward level, circuits found by
# the join or by a tree level; (case name, spec stem, flags)
MITM_CASES = [(f"toffoli-{d}-mitm", "toffoli", ["--depth", str(d), "--mitm"]) for d in range(4, 11)] + [
    ("ccz-7-mitm", "ccz", ["--depth", "7", "--mitm"]), ("ccz-8-mitm", "ccz", ["--depth", "8", "--mitm"]),
    ("cs-4-mitm", "cs", ["--depth", "4", "--mitm"]), ("cs-5-mitm", "cs", ["--depth", "5", "--mitm"]),
    ("qft_2-6-mitm", "qft_2", ["--depth", "6", "--mitm"]), ("qft_2-7-mitm", "qft_2", ["--depth", "7", "--mitm"]),
    ("relative-phase-toffoli-9-mitm", "relative-phase-toffoli", ["--depth", "9", "--mitm"]),
    ("peres-9-mitm", "peres", ["--depth", "9", "--mitm"]), ("fredkin-9-mitm", "fredkin", ["--depth", "9", "--mitm"]),
    ("half_adder_3-9-mitm", "half_adder_3", ["--depth", "9", "--mitm"]),
    ("toffoli-7-mitm-nodedupe", "toffoli", ["--depth", "7", "--mitm", "--no-dedupe"]),
    ("toffoli-9-mitm-table4", "toffoli", ["--depth", "9", "--mitm", "--table", "4"]),
] + [(f"rand-{i:02d}-mitm", f"rand-{i:02d}", ["--mitm"]) for i in range(24)] + [
    (f"table-rand-{i}-mitm", f"table-rand-{i}", ["--mitm"]) for i in range(8)]


# targets whose reference-written spec files the C++ spec generator is checked against
SPECGEN_TARGETS = ["cs", "ccz", "qft_2", "toffoli", "fredkin", "peres", "half_adder_3", "relative-phase-toffoli",
                   "grover_3"]


def specgen_cases(ref, write_spec):
    """circuits of the reference's own qasm targets (parsed by its parse_qasm) with the budget of their committed
    spec files, and a few specs the reference's generator writes for other gate sets (W3 off; with ccx, the "lite"
    bounds; with cz and y)"""
    from cheese import spec as refspec
    out = {}
    qdir = Path(ref) / "tests" / "qasm"
    for stem in SPECGEN_TARGETS:
        n, circ = refspec.parse_qasm(qdir / f"{stem}.qasm")
        text = (GOLD / "specs" / f"{stem}.spec").read_text()
        depth = int(text.split("\ndepth ")[1].split()[0])
        out[stem] = {"n": n, "circuit": [[g, list(qs)] for g, qs in circ], "depth": depth,
                     "qasm": (qdir / f"{stem}.qasm").read_text()}
    extra = {
        "toffoli-now3": (3, out["toffoli"]["circuit"], 9, False),
        "ccx-lite": (3, [["ccx", [0, 1, 2]], ["h", [2]], ["t", [1]]], 5, True),
        "cz-y": (2, [["cz", [0, 1]], ["y", [1]], ["h", [0]], ["t", [0]]], 5, True),
        "ccx-lite-n4": (4, [["ccx", [0, 2, 3]], ["cx", [1, 0]]], 3, True),
    }
    for name, (n, circ, d, use3) in extra.items():
        buf = io.StringIO()
        refspec.write_spec(buf, n, [(g, tuple(q)) for g, q in circ], d, use3=use3)
        (GOLD / "specs" / f"{name}.spec").write_text(buf.getvalue())
        out[name] = {"n": n, "circuit": circ, "depth": d, "w3": use3}
    (GOLD / "spec_circuits.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} spec-generation cases written", file=sys.stderr)


# state targets (RUS without measurement, reference cheese.cu:451-583, run by its CPU build): the reference's own RUS
# targets with their ancilla qubits starting in |0>, and seeded random circuits with random input sets
# (case stem, rus id or None, ancillas, budgets)
STATE_CASES = [("rus28-states", 28, [1], [2, 3, 4]), ("rus2-states", 2, [1], [5, 6, 7]),
               ("rus12-states", 12, [1], [5, 6, 7, 8]), ("rus20-states", 20, [2], [5, 6, 7, 8, 9]),
               ("rus1-states", 1, [1], [7, 8, 9, 10, 11]), ("rus3-states", 3, [1], [7, 8, 9, 10, 11]),
               ("rus7-states", 7, [1, 2], [3, 4, 5, 6, 7]), ("rus8-states", 8, [1, 2], [6, 7, 8, 9, 10])]


def state_cases(ref, binp):
    from cheese import spec as refspec
    sys.path.insert(0, str(ROOT))
    from cheese_b200 import workloads
    out = []

    def run(name, stem, d):
        t0 = time.time()
        try:
            p = subprocess.run([str(binp), str(GOLD / "specs" / f"{stem}.spec"), "--depth", str(d)],
                               capture_output=True, text=True, timeout=300)
        except subprocess.TimeoutExpired:
            print(f"{name}: timed out, left out", file=sys.stderr)
            return
        lines = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
        print(f"{name}: rc {p.returncode}, {len(lines)} lines, {time.time() - t0:.1f} s", file=sys.stderr)
        out.append({"name": name, "spec": stem, "flags": ["--depth", str(d)], "rc": p.returncode, "stdout": lines})

    for stem, rid, anc, budgets in STATE_CASES:
        n, circ = refspec.parse_qasm(Path(ref) / "benchmarks" / "rus" / str(rid) / "spec.qasm")
        mask = sum(1 << q for q in anc)
        inputs = [x for x in range(1 << n) if not x & mask]
        buf = io.StringIO()
        refspec.write_spec(buf, n, circ, budgets[0], inputs=inputs)
        (GOLD / "specs" / f"{stem}.spec").write_text(buf.getvalue())
        for d in budgets:
            run(f"{stem}-{d}", stem, d)
    rng = random.Random(4242)
    for i in range(6):
        n, circ = workloads.random_circuit(rng, n=2 if i < 3 else 3, L=rng.randint(4, 7))
        inputs = sorted(rng.sample(range(1 << n), rng.randint(1, (1 << n) - 1)))
        stem = f"states-rand-{i}"
        buf = io.StringIO()
        refspec.write_spec(buf, n, circ, len(circ), inputs=inputs)
        (GOLD / "specs" / f"{stem}.spec").write_text(buf.getvalue())
        run(f"{stem}-{len(circ)}", stem, len(circ))
        out[-1]["circuit"] = [[g, list(qs)] for g, qs in circ]
        out[-1]["inputs"] = inputs
    (GOLD / "state_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} state cases written", file=sys.stderr)


def state_specgen_cases():
    """state-target specs written by the reference's generator (spec.py:229-325, 356-424) for the C++ generator: the
    qasm targets of the spec-generation cases with ancillas in |0>, and seeded random circuits of 2-4 qubits (some
    with y / cz / ccx) on random input sets. W3 is off so that the fixture stays small: the W3 rules do not depend on
    the target and are checked on the unitary specs."""
    from cheese import spec as refspec
    from cheese_b200 import workloads
    named = json.loads((GOLD / "spec_circuits.json").read_text())
    out = []

    def add(name, n, circ, depth, inputs, ancilla=None):
        buf = io.StringIO()
        refspec.write_spec(buf, n, [(g, tuple(q)) for g, q in circ], depth, use3=False, inputs=inputs)
        out.append({"name": name, "n": n, "circuit": [[g, list(q)] for g, q in circ], "depth": depth,
                    "inputs": inputs, "ancilla": ancilla, "spec": buf.getvalue()})

    for stem, anc in [("toffoli", [2]), ("ccz", [2]), ("fredkin", [0]), ("peres", [1, 2]), ("cs", [1]),
                      ("qft_2", [0]), ("relative-phase-toffoli", [2]), ("half_adder_3", [2]), ("grover_3", [0])]:
        c = named[stem]
        mask = sum(1 << a for a in anc)
        add(f"{stem}-anc{''.join(map(str, anc))}", c["n"], c["circuit"], c["depth"],
            [x for x in range(1 << c["n"]) if not x & mask], anc)
    rng = random.Random(5150)
    for i in range(12):
        n = 2 + i % 3
        _, circ = workloads.random_circuit(rng, n=n, L=rng.randint(3, 8))
        if i % 4 == 3:                                  # other gate sets: y, cz and (3+ qubits) ccx
            circ += [("y", (rng.randrange(n),)), ("cz", (0, 1))] + ([("ccx", (0, 1, 2))] if n >= 3 else [])
        inputs = sorted(rng.sample(range(1 << n), rng.randint(1, 1 << n)))
        add(f"rand-{i}", n, circ, len(circ), inputs)
    (GOLD / "state_spec_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} state spec-generation cases written", file=sys.stderr)


def mitm_cases(binp):
    out = []
    for name, stem, flags in MITM_CASES:
        t0 = time.time()
        p = subprocess.run([str(binp), str(GOLD / "specs" / f"{stem}.spec")] + flags, capture_output=True, text=True,
                           timeout=3600)
        lines = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
        print(f"{name}: rc {p.returncode}, {len(lines)} lines, {time.time() - t0:.1f} s", file=sys.stderr)
        out.append({"name": name, "spec": stem, "flags": flags, "rc": p.returncode, "stdout": lines})
    (GOLD / "mitm_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} mitm cases written", file=sys.stderr)


def table_cases(binp, write_spec):
    """--table K golden cases: named targets plus seeded random ones (found circuits), each run in its own empty
    working directory so that the reference builds (and prints) its distance table"""
    import tempfile
    from cheese_b200 import workloads
    out = []

    def run(case, spec, flags):
        with tempfile.TemporaryDirectory() as cwd:
            t0 = time.time()
            p = subprocess.run([str(binp), str(GOLD / "specs" / f"{spec}.spec")] + flags, capture_output=True,
                               text=True, cwd=cwd)
        lines = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
        tab = [l for l in p.stderr.splitlines() if l.startswith("table")]
        print(f"{case}: rc {p.returncode}, {len(lines)} lines, {time.time() - t0:.1f} s", file=sys.stderr)
        return {"name": case, "spec": spec, "flags": flags, "rc": p.returncode, "stdout": lines,
                "stderr_table": re.sub(r"\(([0-9.]+) s\)", "(0.0 s)", tab[0]) if tab else ""}

    for name, stem, d, k, flags in TABLE_CASES:
        out.append(run(name, stem, ["--depth", str(d), "--table", str(k)] + flags))
    rng = random.Random(77)
    for i in range(8):
        n, circ = workloads.random_circuit(rng, n=3 if i < 6 else 2, L=rng.randint(6, 9))
        name = f"table-rand-{i}"
        write_spec(name, n, circ, len(circ))
        k = 3 if i % 2 == 0 else 4
        out.append(run(f"{name}-table{k}", name, ["--table", str(k)]))
        out[-1]["circuit"] = [[g, list(qs)] for g, qs in circ]
    # budgets below the table depth: only the target's own class is looked up
    for name, stem, d, k in [("table-rand-4-depth2-table3", "table-rand-4", 2, 3),
                             ("table-rand-4-depth3-table4", "table-rand-4", 3, 4)]:
        out.append(run(name, stem, ["--depth", str(d), "--table", str(k)]))
    (GOLD / "table_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} table cases written", file=sys.stderr)


def parts(text):
    """(lines up to the bad3 header, the bad3 lines sorted, the lines after them): the reference lists its W3
    triples in the iteration order of a Python set, so two writers agree on them as a set"""
    L = text.splitlines()
    i = next(j for j, l in enumerate(L) if l.startswith("bad3 "))
    n = int(L[i].split()[1])
    return L[:i + 1], sorted(L[i + 1:i + 1 + n]), L[i + 1 + n:]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's source tree (read only)")
    ap.add_argument("--quick", action="store_true", help="skip the cases that take more than a few seconds")
    ap.add_argument("--table-only", action="store_true", help="write only the --table K cases")
    ap.add_argument("--mitm-only", action="store_true", help="write only the --mitm cases")
    ap.add_argument("--specgen-only", action="store_true", help="write only the spec-generation cases")
    ap.add_argument("--states-only", action="store_true", help="write only the state-target cases")
    ap.add_argument("--state-specgen-only", action="store_true",
                    help="write only the state-target spec-generation cases (no reference binary needed)")
    o = ap.parse_args()
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(o.ref) / "python"))
    from cheese import spec as refspec            # the reference's spec writer
    sys.path.insert(0, str(ROOT))
    from cheese_b200 import workloads

    if o.state_specgen_only:
        state_specgen_cases()
        return
    binp = ROOT / "oracle" / "_ref" / "cheese-cpu"
    b64 = ROOT / "oracle" / "_ref" / "cheese-cpu-store64"
    assert binp.exists(), "build the reference CPU binary first: make -C oracle"
    (GOLD / "specs").mkdir(parents=True, exist_ok=True)

    def write_spec(name, n, circ, depth):
        buf = io.StringIO()
        refspec.write_spec(buf, n, circ, depth)
        (GOLD / "specs" / f"{name}.spec").write_text(buf.getvalue())
        return buf.getvalue()

    def run(case, spec, flags, exe=binp):
        t0 = time.time()
        p = subprocess.run([str(exe), str(GOLD / "specs" / f"{spec}.spec")] + flags, capture_output=True, text=True)
        out = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
        print(f"{case}: rc {p.returncode}, {len(out)} lines, {time.time() - t0:.1f} s", file=sys.stderr)
        return {"name": case, "spec": spec, "flags": flags, "rc": p.returncode, "stdout": out}

    if o.table_only:
        table_cases(binp, write_spec)
        return
    if o.mitm_only:
        mitm_cases(binp)
        return
    if o.specgen_only:
        specgen_cases(o.ref, write_spec)
        return
    if o.states_only:
        state_cases(o.ref, binp)
        return
    # target specs written by the reference generator (budget line = the first budget used)
    qdir = Path(o.ref) / "tests" / "qasm"
    cases = []
    written = set()
    for name, stem, d, flags in CASES + ([] if o.quick else SLOW):
        if stem not in written:
            n, circ = refspec.parse_qasm(qdir / f"{stem}.qasm")
            write_spec(stem, n, circ, d)
            written.add(stem)
        cases.append(run(name, stem, ["--depth", str(d)] + flags))

    # base specs: identity target, default Clifford+T candidates, per qubit count
    for n in (2, 3):
        write_spec(f"base-n{n}", n, [], 1)

    # seeded random circuits (the batched workload's generator): reference spec, checked against ours
    rng = random.Random(20261203)
    for i in range(24):
        n, circ = workloads.random_circuit(rng, L=rng.randint(6, 9))
        name = f"rand-{i:02d}"
        text = write_spec(name, n, circ, len(circ))
        assert parts(text) == parts(workloads.make_spec(n, circ, len(circ))), f"{name}: spec differs from the reference"
        cases.append(run(name, name, []))
        cases[-1]["circuit"] = [[g, list(qs)] for g, qs in circ]

    # a state-target spec (RUS without measurement, ancilla qubit 1 of CS): the GPU binaries refuse it (exit 3)
    n, circ = refspec.parse_qasm(qdir / "cs.qasm")
    buf = io.StringIO()
    refspec.write_spec(buf, n, circ, 5, inputs=[0, 1])
    (GOLD / "specs" / "cs-states.spec").write_text(buf.getvalue())

    # int32 overflow: a 2-qubit target (HT)^140 with sqrt2 exponent 72 (coefficients ~2^36); default build exits 4,
    # the -DSTORE64 build runs the search
    circ = [("h", (0,)), ("t", (0,))] * 140
    write_spec("overflow", 2, circ, 4)
    cases.append(run("overflow-4", "overflow", []))
    c64 = run("overflow-4-store64", "overflow", [], exe=b64)
    cases.append(c64)

    (GOLD / "cases.json").write_text(json.dumps(cases, indent=1) + "\n")
    print(f"{len(cases)} cases written", file=sys.stderr)
    table_cases(binp, write_spec)
    mitm_cases(binp)
    specgen_cases(o.ref, write_spec)
    state_cases(o.ref, binp)


if __name__ == "__main__":
    main()
