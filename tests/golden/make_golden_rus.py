"""Generate the golden fixtures of the RUS T-count search (the reference's build/rus, src/rus.cu).

Run in a container that has the reference source tree (read-only is fine) and the C restatement built
(`make -C oracle`):

    python tests/golden/make_golden_rus.py --ref /path/to/reference

The rus-specs are written by the reference's own writer (python -m cheese.rus spec) for its RUS regression targets
(tests/qasm/ricotta-rus-*.qasm). Every spec shares its table root, rotation tables and Clifford list, so those are
stored once (rus/common.rspec.gz) and the roots per target (rus/<target>.roots); tests join them back into the
reference's file layout. The expected output of each (target, --table K, --max T) case is the C restatement's
(oracle/rus_oracle.c), pinned by the reference's own known optima (tests/rus_check.sh: 0003 -> 4 at K = 4 and 1,
0229 -> 10 at K = 7 and 5), its published level-4 table size (692 cosets) and, for every found circuit, the
reference's exact verifier (python -m cheese.rus verify).

Writes
  tests/golden/rus/common.rspec.gz     table-root, rotations and cliffords blocks
  tests/golden/rus/<target>.roots      the roots block of each target
  tests/golden/rus_cases.json          per case: target, flags, exit code, stdout ("seconds" 0.00), verified
  tests/golden/rus_spec_cases.json     (--specgen-only) variant RUS circuits with the reference writer's roots
                                       block and its info line, for the C++ writer
"""
import argparse
import gzip
import json
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
GOLD = ROOT / "tests" / "golden"
ORACLE = ROOT / "oracle" / "_ref" / "rus-oracle"

# (target stem, table depth, max T-count)
CASES = [("ricotta-rus-0003", k, 3) for k in (0, 1, 2, 3, 4, 5)] + [("ricotta-rus-0003", k, 4) for k in (1, 3, 4)] + [
    ("ricotta-rus-0229", k, 11) for k in (5, 6, 7)] + [("ricotta-rus-0229", 6, 9), ("ricotta-rus-0229", 7, 10),
                                                      ("ricotta-rus-0229", 4, 8)]


def split_spec(text):
    """(table-root block, roots block, rotations + cliffords blocks) of a rus-spec"""
    a, b = text.index("table-root"), text.index("roots ")
    c, d = text.index("rotations "), text.index("\nend")
    return text[a:b], text[b:c], text[c:d + 1]


def join_spec(common, roots):
    root, rest = common.split("\n@@\n")
    return "rus-spec 1\n" + root + roots + rest + "end\n"


def variants(ref):
    """The regression targets themselves, and RUS circuits derived from them: seeded Clifford gates on the data qubit before and after
    (and a CZ after: a Pauli correction per outcome), some with the outcomes swapped by an X on the ancilla; comments
    dropped, so the writer detects the success outcome. Their optimal RUS T-counts equal the targets' (Cliffords
    are free on either side)."""
    import random
    rng = random.Random(7301)
    out = []
    for stem in ("ricotta-rus-0003", "ricotta-rus-0229"):
        text = (Path(ref) / "tests" / "qasm" / f"{stem}.qasm").read_text()
        out.append((stem, stem, text))              # as is: its "success outcome" comment names the outcome
        lines = text.splitlines()
        head = [l for l in lines if l.startswith(("OPENQASM", "include", "qreg", "creg"))]
        body = [l for l in lines if l and not l.startswith(("OPENQASM", "include", "qreg", "creg", "//", "measure"))]
        for i in range(4):
            pre = [f"{rng.choice(['h', 's', 'sdg', 'x', 'y', 'z'])} q[1];" for _ in range(rng.randint(1, 3))]
            post = [f"{rng.choice(['h', 's', 'sdg', 'x', 'y', 'z'])} q[1];" for _ in range(rng.randint(1, 3))]
            if i % 2:
                post.append("cz q[0],q[1];")
            if i >= 2:
                post.append("x q[0];")
            text = "\n".join(head + pre + body + post + ["measure q[0] -> c[0];"]) + "\n"
            out.append((f"{stem}-v{i}", stem, text))
    return out


def specgen_cases(ref, common):
    """the reference writer's rus-specs of the variant circuits, for the C++ writer"""
    cases = []
    with tempfile.TemporaryDirectory() as td:
        for name, stem, text in variants(ref):
            q = Path(td) / f"{name}.qasm"
            q.write_text(text)
            p = subprocess.run([sys.executable, "-m", "cheese.rus", "spec", str(q)], capture_output=True, text=True,
                               cwd=Path(ref) / "python", check=True)
            root, roots, rest = split_spec(p.stdout)
            assert root + "\n@@\n" + rest == common, "the shared spec blocks differ"
            cases.append({"name": name, "base": stem, "qasm": text, "roots": roots,
                          "info": json.loads(p.stderr.strip().splitlines()[-1])})
            print(f"{name}: {cases[-1]['info']}", file=sys.stderr)
    (GOLD / "rus_spec_cases.json").write_text(json.dumps(cases, indent=1) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's source tree (read only)")
    ap.add_argument("--specgen-only", action="store_true", help="write only the spec-writer cases (variants)")
    o = ap.parse_args()
    if o.specgen_only:
        with gzip.open(GOLD / "rus" / "common.rspec.gz", "rt") as f:
            specgen_cases(o.ref, f.read())
        return
    assert ORACLE.exists(), "build the C restatement first: make -C oracle"
    (GOLD / "rus").mkdir(parents=True, exist_ok=True)
    common = None
    for stem in sorted({c[0] for c in CASES}):
        p = subprocess.run([sys.executable, "-m", "cheese.rus", "spec", str(Path(o.ref) / "tests" / "qasm" / f"{stem}.qasm")],
                           capture_output=True, text=True, cwd=Path(o.ref) / "python", check=True)
        root, roots, rest = split_spec(p.stdout)
        c = root + "\n@@\n" + rest
        assert common is None or c == common, "the shared spec blocks differ between targets"
        common = c
        (GOLD / "rus" / f"{stem}.roots").write_text(roots)
        assert join_spec(common, roots) == p.stdout
    with gzip.open(GOLD / "rus" / "common.rspec.gz", "wt") as f:
        f.write(common)
    out = []
    with tempfile.TemporaryDirectory() as td:
        for stem, k, mx in CASES:
            spec = Path(td) / f"{stem}.rspec"
            spec.write_text(join_spec(common, (GOLD / "rus" / f"{stem}.roots").read_text()))
            flags = ["--table", str(k), "--max", str(mx)]
            p = subprocess.run([str(ORACLE), str(spec)] + flags, capture_output=True, text=True, timeout=3600)
            lines = p.stdout.splitlines()
            verified = None
            if p.returncode == 0:
                log = Path(td) / "out.log"
                log.write_text(p.stdout)
                v = subprocess.run([sys.executable, "-m", "cheese.rus", "verify",
                                    str(Path(o.ref) / "tests" / "qasm" / f"{stem}.qasm"), str(log), str(Path(td) / "w.qasm")],
                                   capture_output=True, text=True, cwd=Path(o.ref) / "python")
                verified = v.returncode == 0 and v.stdout.startswith("verified")
                assert verified, v.stdout + v.stderr
            name = f"{stem}-k{k}-max{mx}"
            print(f"{name}: rc {p.returncode}, {lines[-1]}", file=sys.stderr)
            out.append({"name": name, "target": stem, "flags": flags, "rc": p.returncode, "stdout": lines,
                        "verified": verified})
    (GOLD / "rus_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} RUS cases written", file=sys.stderr)


if __name__ == "__main__":
    main()
