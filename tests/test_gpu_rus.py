"""RUS T-count with measurement (`rus SPEC --table K --max T`, the reference's build/rus, src/rus.cu) on the GPU.

Every committed case (the reference's RUS regression targets at several table depths and budgets) is reproduced by
the drop-in binary (stdout lines, exit code, stderr table line) in a fresh working directory, a second run loads the
table from its cache file, the C ABI gives the same lines with the table resident on the engine, and the reference's
own sm_100a build, where it was compiled (oracle/_ref/rus-ref), prints the same lines on the same specs."""
import re
import subprocess

import pytest

from conftest import ORACLE_DIR, rus_cases, rus_spec_text, strip_seconds

pytestmark = pytest.mark.gpu

CASES = rus_cases()
REF_GPU = ORACLE_DIR / "_ref" / "rus-ref"


@pytest.fixture(scope="module")
def specs(tmp_path_factory):
    d = tmp_path_factory.mktemp("rspec")
    out = {}
    for t in {c["target"] for c in CASES}:
        out[t] = d / f"{t}.rspec"
        out[t].write_text(rus_spec_text(t))
    return out


def run(exe, spec, flags, cwd):
    return subprocess.run([str(exe), str(spec)] + flags, capture_output=True, text=True, cwd=cwd, timeout=900)


def table_classes(case):
    return 1 + sum(int(re.search(r'"new": (\d+)', l).group(1)) for l in case["stdout"] if '"dir": "table"' in l)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_drop_in_matches(case, specs, tmp_path):
    import cheese_b200 as cz
    (tmp_path / "build").mkdir()
    p = run(cz.BIN_DIR / "rus", specs[case["target"]], case["flags"], tmp_path)
    assert p.returncode == case["rc"], p.stderr
    assert strip_seconds(p.stdout.splitlines()) == case["stdout"]
    k = int(case["flags"][1])
    tab = [l for l in p.stderr.splitlines() if l.startswith("table")][0]
    assert re.sub(r"\(([0-9.]+) s\)", "(0.0 s)", tab) == (
        f"table: {table_classes(case)} cosets with T-count <= {k} (0.0 s), cached in build/rus-table-k{k}.cz.bin")


def test_cache_roundtrip(specs, tmp_path):
    import cheese_b200 as cz
    (tmp_path / "build").mkdir()
    for name in ("ricotta-rus-0003-k4-max4", "ricotta-rus-0229-k7-max11", "ricotta-rus-0229-k7-max10"):
        case = next(c for c in CASES if c["name"] == name)
        p = run(cz.BIN_DIR / "rus", specs[case["target"]], case["flags"], tmp_path)
        assert p.returncode == case["rc"]
        p = run(cz.BIN_DIR / "rus", specs[case["target"]], case["flags"], tmp_path)
        assert p.returncode == case["rc"], p.stderr
        assert strip_seconds(p.stdout.splitlines()) == [l for l in case["stdout"] if '"dir": "table"' not in l]
        assert "(loaded" in p.stderr


def test_api_matches(specs):
    import json
    import cheese_b200 as cz
    from cheese_b200 import verify
    from conftest import GOLD
    qasm = {c["name"]: c["qasm"] for c in json.loads((GOLD / "rus_spec_cases.json").read_text())}
    eng = cz.Engine()
    for case in CASES:
        k, mx = int(case["flags"][1]), int(case["flags"][3])
        rc, levels, out = eng.rus(specs[case["target"]].read_text(), table_k=k, maxt=mx, cache_dir=None)
        assert rc == case["rc"], (case["name"], out["error"])
        want = case["stdout"] if out["table_built"] else [l for l in case["stdout"] if '"dir": "table"' not in l]
        assert eng.rus_lines(rc, levels, out) == want, case["name"]
        assert out["kernel_launches"] > 0
        if rc == 0:                                   # the found circuit, checked exactly against its target
            cl = verify.rspec_cliffords(specs[case["target"]].read_text())
            assert verify.rus_check(qasm[case["target"]], out, cl), case["name"]
    eng.trim()


def test_spec_errors(tmp_path):
    import cheese_b200 as cz
    bad = tmp_path / "bad.rspec"
    bad.write_text("rus-spec 1\nroots 0\nend\n")
    p = run(cz.BIN_DIR / "rus", bad, [], tmp_path)
    assert p.returncode == 2 and p.stderr.strip() == "incomplete spec"
    p = subprocess.run([str(cz.BIN_DIR / "rus")], capture_output=True, text=True)
    assert p.returncode == 3 and p.stderr.startswith("usage: rus SPEC")


@pytest.mark.skipif(not REF_GPU.exists(), reason="the reference's sm_100a build of rus.cu was not compiled here")
def test_reference_gpu_build_agrees(specs, tmp_path):
    for name in ("ricotta-rus-0003-k4-max3", "ricotta-rus-0003-k1-max4", "ricotta-rus-0229-k7-max11",
                 "ricotta-rus-0229-k6-max9"):
        case = next(c for c in CASES if c["name"] == name)
        d = tmp_path / name
        (d / "build").mkdir(parents=True)
        p = run(REF_GPU, specs[case["target"]], case["flags"], d)
        assert p.returncode == case["rc"], p.stderr
        assert strip_seconds(p.stdout.splitlines()) == case["stdout"], name
