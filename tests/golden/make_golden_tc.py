"""Golden fixtures of the T-count and Clifford-table paths.

Step 1 (any machine with the reference tree, which provides the qasm targets):
    python tests/golden/make_golden_tc.py inputs --ref /path/to/reference
  writes tests/golden/tcount/*.tspec (the reference's targets and seeded table-driven queries, in the reference's
  tcount-spec format, checked against its tcount.py where it exists) and tests/golden/cliffopt/*.job.

Step 2 (a CUDA machine with oracle/_ref/tcount-ref and oracle/_ref/cliffopt-ref, the reference's own programs built
by `make -C oracle refgpu`):
    python tests/golden/make_golden_tc.py outputs OUTDIR
  runs the reference programs on every input (fresh table caches) and writes OUTDIR/tcount_cases.json and
  OUTDIR/cliffopt_cases.json: arguments, exit code, stdout ("seconds" values replaced by 0.00) and the stderr lines
  that carry results (table sizes, BFS counts per distance). The JSON files are committed under tests/golden/.

Step 3 (any machine, after `make -C oracle oracle`):
    python tests/golden/make_golden_tc.py oracle
  writes tests/golden/cliffopt_oracle.json: the C restatement's cliffopt outputs for the jobs with T gates, whose
  beam ties the reference leaves to an atomic counter (see oracle/clifford_oracle.c).
"""
import json
import os
import random
import re
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
GOLD = ROOT / "tests" / "golden"
SECONDS = re.compile(r'"seconds": [0-9.]+')
TARGETS = ["cs", "qft_2", "toffoli", "ccz", "fredkin", "peres", "relative-phase-toffoli"]


def inputs(ref):
    sys.path.insert(0, str(ROOT))
    from cheese_b200 import tcwork, workloads
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref) / "python"))
    from cheese import spec as refspec
    from cheese import tcount as reftc
    import io
    (GOLD / "tcount").mkdir(exist_ok=True)
    (GOLD / "cliffopt").mkdir(exist_ok=True)
    for t in TARGETS:
        n, circ = refspec.parse_qasm(Path(ref) / "tests" / "qasm" / f"{t}.qasm")
        buf = io.StringIO()
        reftc.write_spec(buf, n, refspec.unitary(n, circ))
        assert buf.getvalue() == tcwork.tspec(n, workloads.unitary(n, circ)), t
        (GOLD / "tcount" / f"{t}.tspec").write_text(buf.getvalue())
    # the reference's published optimal decompositions (benchmarks/optimal/<t>-tcount.json: search levels with the
    # K = 4 table loaded, then the result line), seconds stripped
    opt = []
    for t in TARGETS:
        lines = (Path(ref) / "benchmarks" / "optimal" / f"{t}-tcount.json").read_text().splitlines()
        opt.append({"name": t, "stdout": [SECONDS.sub('"seconds": 0.00', l) for l in lines if l.strip()]})
    (GOLD / "tcount" / "optimal.json").write_text(json.dumps(opt, indent=1) + "\n")
    rng = random.Random(4096)
    for i in range(8):
        circ, k = tcwork.tcount_query(rng, 3)
        (GOLD / "tcount" / f"q3-{i}.tspec").write_text(tcwork.tspec_of_circuit(3, circ))
    for i in range(4):
        circ, k = tcwork.tcount_query(rng, 2)
        (GOLD / "tcount" / f"q2-{i}.tspec").write_text(tcwork.tspec_of_circuit(2, circ))
    rng = random.Random(8192)
    for i in range(6):
        (GOLD / "cliffopt" / f"c3-{i}.job").write_text(tcwork.random_clifford_job(rng, 3, 40, 0))
    for i in range(2):
        (GOLD / "cliffopt" / f"c2-{i}.job").write_text(tcwork.random_clifford_job(rng, 2, 20, 0))
    for i in range(3):
        (GOLD / "cliffopt" / f"t3-{i}.job").write_text(tcwork.random_clifford_job(rng, 3, 12, 2 + i))


def run(exe, args, cwd, timeout=600):
    p = subprocess.run([str(exe)] + args, capture_output=True, text=True, cwd=cwd, timeout=timeout)
    out = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
    err = [re.sub(r"\(([0-9.]+) s\)|, [0-9.]+ s$|\(loaded, [0-9.]+ s\)", "", l) for l in p.stderr.splitlines()]
    return {"args": args, "rc": p.returncode, "stdout": out, "stderr": err}


def outputs(outdir):
    """every case is bounded (a few minutes at most on a B200); the JSON files are rewritten after each case"""
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    tc = ROOT / "oracle" / "_ref" / "tcount-ref"
    co = ROOT / "oracle" / "_ref" / "cliffopt-ref"
    work = Path(tempfile.mkdtemp())
    (work / "build").mkdir()
    cases = []
    spec = lambda name: str(GOLD / "tcount" / f"{name}.tspec")

    def case(name, args):
        try:
            r = run(tc, args, work)
        except subprocess.TimeoutExpired:
            print(name, "timed out", file=sys.stderr, flush=True)
            return
        r["name"] = name
        r["args"] = [str(Path(args[0]).relative_to(ROOT))] + args[1:]
        cases.append(r)
        (outdir / "tcount_cases.json").write_text(json.dumps(cases, indent=1) + "\n")
        print(name, r["rc"], r["stdout"][-1] if r["stdout"] else "", file=sys.stderr, flush=True)

    # 3 qubits: the default table (K = 4) is built by the first run, loaded by the others
    case("toffoli-k4", [spec("toffoli"), "--table", "4"])
    for t in ["ccz", "fredkin", "peres", "relative-phase-toffoli"]:
        case(f"{t}-k4", [spec(t), "--table", "4"])
    for i in range(8):
        case(f"q3-{i}-k4", [spec(f"q3-{i}"), "--table", "4"])
    case("toffoli-k4-max5", [spec("toffoli"), "--table", "4", "--max", "5"])
    # smaller tables: K = 3 needs four search levels for the Toffoli (K = 1, 2 need far more: not run)
    case("toffoli-k3", [spec("toffoli"), "--table", "3"])
    case("toffoli-k2-max4", [spec("toffoli"), "--table", "2", "--max", "4"])
    case("toffoli-k1-max3", [spec("toffoli"), "--table", "1", "--max", "3"])
    # 2 qubits: K = 6 and smaller tables
    case("cs-k6", [spec("cs"), "--table", "6"])
    case("qft_2-k6", [spec("qft_2"), "--table", "6"])
    for i in range(4):
        case(f"q2-{i}-k6", [spec(f"q2-{i}"), "--table", "6"])
    for K in (2, 4):
        case(f"cs-k{K}", [spec("cs"), "--table", str(K)])
        case(f"qft_2-k{K}", [spec("qft_2"), "--table", str(K)])

    jobs = []
    for j in sorted((GOLD / "cliffopt").glob("*.job")):
        try:
            r = run(co, [str(j)], work)
        except subprocess.TimeoutExpired:
            print(j.stem, "timed out", file=sys.stderr, flush=True)
            continue
        r["name"] = j.stem
        r["args"] = [str(j.relative_to(ROOT))]
        jobs.append(r)
        (outdir / "cliffopt_cases.json").write_text(json.dumps(jobs, indent=1) + "\n")
        print(j.stem, r["rc"], r["stdout"][:1], file=sys.stderr, flush=True)
    shutil.rmtree(work, ignore_errors=True)


def oracle_outputs():
    """the C restatement's outputs for the cliffopt jobs with T gates (3 qubits: about a minute of table build plus
    minutes of beam per job on a few CPU cores), at beams 16 and 4 -> tests/golden/cliffopt_oracle.json. Its
    candidate order is the product's, so these are exact expectations for the GPU path."""
    exe = ROOT / "oracle" / "_ref" / "clifford-oracle"
    jobs = sorted((GOLD / "cliffopt").glob("t3-*.job"))
    out = []
    for beam in (16, 4):
        p = subprocess.run([str(exe)] + [str(j) for j in jobs] + ["--beam", str(beam)], capture_output=True, text=True,
                           timeout=7200)
        blocks = p.stdout.split("### ")[1:]
        for j, blk in zip(jobs, [b for b in blocks if not b.startswith("rc ")]):
            lines = blk.splitlines()[1:]
            out.append({"name": j.stem, "beam": beam, "stdout": lines})
        print("beam", beam, "done", file=sys.stderr, flush=True)
    (GOLD / "cliffopt_oracle.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    if sys.argv[1] == "oracle":
        oracle_outputs()
    elif sys.argv[1] == "inputs":
        if "--ref" not in sys.argv:
            sys.exit("inputs: --ref /path/to/reference is required (the reference's source tree)")
        inputs(sys.argv[sys.argv.index("--ref") + 1])
    else:
        outputs(sys.argv[2])
