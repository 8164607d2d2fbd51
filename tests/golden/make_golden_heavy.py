"""Golden fixtures of the large-frontier regime: seeded random 3-qubit targets of 12 gates at budget 12 (the
batched workload's generator at its heaviest setting) and Toffoli budget 12 without symmetry classes, whose levels
reach 1e7 prefixes and 1e6-1e7 survivors, run by the reference itself.

Step 1 (a machine with the reference source tree; its spec writer python/cheese/spec.py writes the specs):
    python tests/golden/make_golden_heavy.py specs --ref /path/to/reference --seeds 0:48
  writes tests/golden/specs/heavy-<seed>.spec and tests/golden/heavy_circuits.json (seed -> circuit).

Step 2 (any machine with a reference build under oracle/_ref: the CPU build cheese-cpu, or the GPU build
cheese-gpu-ref on a CUDA machine; `make -C oracle REF=/path/to/reference`):
    python tests/golden/make_golden_heavy.py run OUT.json --exe oracle/_ref/cheese-gpu-ref [--seeds 0:48] [--timeout S]
  runs the reference program on every heavy spec, on toffoli.spec --no-sym at budget 12 and on the --table 8 cases
  (TABLE_HEAVY, unless --no-table), each in an empty working directory, and writes per case the spec, flags, exit
  code, stdout with every "seconds" value replaced by 0.00, the table line of stderr and the program that ran it.

Step 3 (any machine): merge the chosen cases into tests/golden/heavy_cases.json:
    python tests/golden/make_golden_heavy.py merge OUT.json [OUT2.json ...] --keep heavy-5,heavy-9,...
  A case present in several inputs (CPU and GPU build of the reference) must agree line for line; the merged case
  lists every program that produced it.
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
L, N_QUBITS = 12, 3


def heavy_circuit(seed):
    """the target of seed: a random 3-qubit Clifford+T circuit of 12 gates (the batched workload's generator)"""
    sys.path.insert(0, str(ROOT))
    from cheese_b200 import workloads
    return workloads.random_circuit(random.Random(seed), n=N_QUBITS, L=L)[1]


def seeds_of(arg):
    a, b = (int(x) for x in arg.split(":"))
    return range(a, b)


def write_specs(ref, seeds):
    sys.path.insert(0, str(Path(ref) / "python"))
    from cheese import spec as refspec            # the reference's spec writer
    circ = {}
    for s in seeds:
        c = heavy_circuit(s)
        buf = io.StringIO()
        refspec.write_spec(buf, N_QUBITS, c, L)
        (GOLD / "specs" / f"heavy-{s}.spec").write_text(buf.getvalue())
        circ[str(s)] = [[g, list(q)] for g, q in c]
    p = GOLD / "heavy_circuits.json"
    old = json.loads(p.read_text()) if p.exists() else {}
    old.update(circ)
    p.write_text(json.dumps(old, indent=1, sort_keys=True) + "\n")


# --table 8 runs past the sizes of the table golden cases: Fredkin 15 and 16 (proofs whose levels after the table
# reach tens of millions of prefixes) and the Toffoli optimum 15 (a circuit found through the table), each in an
# empty working directory so the reference builds its K = 8 table and prints its table line
TABLE_HEAVY = [("fredkin-15-table8", "fredkin", 15), ("fredkin-16-table8", "fredkin", 16),
               ("toffoli-15-table8", "toffoli", 15)]


def run_cases(out, exe, seeds, timeout, with_table=True):
    import tempfile
    exe = Path(exe).resolve()
    cases = [("toffoli-12-nosym", "toffoli", ["--depth", "12", "--no-sym"])]
    if with_table:
        cases += [(name, stem, ["--depth", str(d), "--table", "8"]) for name, stem, d in TABLE_HEAVY]
    cases += [(f"heavy-{s}", f"heavy-{s}", ["--depth", str(L)]) for s in seeds
              if (GOLD / "specs" / f"heavy-{s}.spec").exists()]
    res = []
    for name, spec, flags in cases:
        t0 = time.time()
        with tempfile.TemporaryDirectory() as cwd:
            try:
                p = subprocess.run([str(exe), str(GOLD / "specs" / f"{spec}.spec")] + flags, capture_output=True,
                                   text=True, timeout=timeout, cwd=cwd)
            except subprocess.TimeoutExpired:
                print(f"{name}: timeout after {timeout} s", file=sys.stderr, flush=True)
                continue
        lines = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
        peak = max((json.loads(l).get("prefixes", 0) for l in lines if '"prefixes"' in l), default=0)
        dt = time.time() - t0
        print(f"{name}: rc {p.returncode}, {len(lines)} lines, peak level {peak} prefixes, {dt:.1f} s",
              file=sys.stderr, flush=True)
        rec = {"name": name, "spec": spec, "flags": flags, "rc": p.returncode, "stdout": lines,
               "by": [exe.name], "peak_prefixes": peak, "seconds": round(dt, 1)}
        if "--table" in flags:
            tab = [l for l in p.stderr.splitlines() if l.startswith("table")]
            rec["stderr_table"] = re.sub(r"\(([0-9.]+) s\)", "(0.0 s)", tab[0]) if tab else ""
        res.append(rec)
        Path(out).write_text(json.dumps(res, indent=1) + "\n")


def merge(inputs, keep):
    merged = {}
    for f in inputs:
        for c in json.loads(Path(f).read_text()):
            if keep and c["name"] not in keep:
                continue
            c = dict(c)
            c.pop("seconds", None)
            if c["name"] in merged:
                m = merged[c["name"]]
                assert (m["rc"], m["stdout"]) == (c["rc"], c["stdout"]), f"{c['name']}: reference builds disagree"
                m["by"] = sorted(set(m["by"]) | set(c["by"]))
            else:
                merged[c["name"]] = c
    circ = json.loads((GOLD / "heavy_circuits.json").read_text())
    out = []
    for name in sorted(merged, key=lambda n: (not n.startswith("toffoli"), len(n), n)):
        c = merged[name]
        if name.startswith("heavy-"):
            c["circuit"] = circ[name.split("-")[1]]
        out.append(c)
    (GOLD / "heavy_cases.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out)} cases written", file=sys.stderr)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["specs", "run", "merge"])
    ap.add_argument("files", nargs="*")
    ap.add_argument("--ref", help="the reference's source tree (step specs)")
    ap.add_argument("--exe", help="the reference program (step run)")
    ap.add_argument("--seeds", default="0:48")
    ap.add_argument("--timeout", type=float, default=1800)
    ap.add_argument("--keep", default="", help="comma-separated case names (step merge)")
    ap.add_argument("--no-table", action="store_true", help="step run: skip the --table 8 cases")
    o = ap.parse_args()
    sys.dont_write_bytecode = True
    if o.step == "specs":
        if not o.ref:
            sys.exit("specs: --ref /path/to/reference is required")
        write_specs(o.ref, seeds_of(o.seeds))
    elif o.step == "run":
        run_cases(o.files[0], o.exe, seeds_of(o.seeds), o.timeout, not o.no_table)
    else:
        merge(o.files, set(filter(None, o.keep.split(","))))


if __name__ == "__main__":
    main()
