"""Golden fixtures of the T-count and Clifford-table paths.

Step 1 (any machine with the reference tree, which provides the qasm targets):
    python tests/golden/make_golden_tc.py inputs [--ref /path/to/reference]
  writes tests/golden/tcount/*.tspec (the reference's targets and seeded table-driven queries, in the reference's
  tcount-spec format, checked against its tcount.py where it exists) and tests/golden/cliffopt/*.job.

Step 2 (a CUDA machine with oracle/_ref/tcount-ref and oracle/_ref/cliffopt-ref, the reference's own programs built
by `make -C oracle refgpu`):
    python tests/golden/make_golden_tc.py outputs OUTDIR
  runs the reference programs on every input (fresh table caches) and writes OUTDIR/tcount_cases.json and
  OUTDIR/cliffopt_cases.json: arguments, exit code, stdout ("seconds" values replaced by 0.00) and the stderr lines
  that carry results (table sizes, BFS counts per distance). The JSON files are committed under tests/golden/.
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


def run(exe, args, cwd):
    p = subprocess.run([str(exe)] + args, capture_output=True, text=True, cwd=cwd, timeout=1800)
    out = [SECONDS.sub('"seconds": 0.00', l) for l in p.stdout.splitlines()]
    err = [re.sub(r"\(([0-9.]+) s\)|, [0-9.]+ s$|\(loaded, [0-9.]+ s\)", "", l) for l in p.stderr.splitlines()]
    return {"args": args, "rc": p.returncode, "stdout": out, "stderr": err}


def outputs(outdir):
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    tc = ROOT / "oracle" / "_ref" / "tcount-ref"
    co = ROOT / "oracle" / "_ref" / "cliffopt-ref"
    work = Path(tempfile.mkdtemp())
    (work / "build").mkdir()
    cases = []
    spec = lambda name: str(GOLD / "tcount" / f"{name}.tspec")

    def case(name, args):
        r = run(tc, args, work)
        r["name"] = name
        cases.append(r)
        print(name, r["rc"], r["stdout"][-1] if r["stdout"] else "", file=sys.stderr, flush=True)

    # 3 qubits: the default table (K = 4) is built by the first run, loaded by the others
    case("toffoli-k4", [spec("toffoli"), "--table", "4"])
    for t in ["ccz", "fredkin", "peres", "relative-phase-toffoli"]:
        case(f"{t}-k4", [spec(t), "--table", "4"])
    for i in range(8):
        case(f"q3-{i}-k4", [spec(f"q3-{i}"), "--table", "4"])
    case("toffoli-k4-max5", [spec("toffoli"), "--table", "4", "--max", "5"])
    for K in (1, 2, 3):
        case(f"toffoli-k{K}", [spec("toffoli"), "--table", str(K)])
    # 2 qubits: K = 6 (the driver's default for n <= 2) and smaller tables
    case("cs-k6", [spec("cs"), "--table", "6"])
    case("qft_2-k6", [spec("qft_2"), "--table", "6"])
    for i in range(4):
        case(f"q2-{i}-k6", [spec(f"q2-{i}"), "--table", "6"])
    for K in (2, 4):
        case(f"cs-k{K}", [spec("cs"), "--table", str(K)])
        case(f"qft_2-k{K}", [spec("qft_2"), "--table", str(K)])
    (outdir / "tcount_cases.json").write_text(json.dumps(cases, indent=1) + "\n")

    jobs = []
    for j in sorted((GOLD / "cliffopt").glob("*.job")):
        r = run(co, [str(j)], work)
        r["name"] = j.stem
        jobs.append(r)
        print(j.stem, r["rc"], r["stdout"][:1], file=sys.stderr, flush=True)
    (outdir / "cliffopt_cases.json").write_text(json.dumps(jobs, indent=1) + "\n")
    shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    if sys.argv[1] == "inputs":
        ref = sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv else "/root/reference"
        inputs(ref)
    else:
        outputs(sys.argv[2])
