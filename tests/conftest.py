import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"
ORACLE_DIR = ROOT / "oracle"
ORACLE_BIN = ORACLE_DIR / "_ref" / "cz-oracle"
ORACLE_LIB = ORACLE_DIR / "_ref" / "libcz_oracle.so"
REF_CPU = ORACLE_DIR / "_ref" / "cheese-cpu"
sys.path.insert(0, str(ROOT))

# cases whose reference run takes tens of seconds on a few CPU cores: GPU tests only
SLOW_CPU = {"toffoli-11", "toffoli-12", "toffoli-11-nosym"}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_cases():
    return json.loads((GOLD / "cases.json").read_text())


def spec_path(name):
    return GOLD / "specs" / f"{name}.spec"


def spec_text(name):
    return spec_path(name).read_text()


def case_depth(case):
    f = case["flags"]
    return int(f[f.index("--depth") + 1]) if "--depth" in f else -1


@pytest.fixture(scope="session")
def oracle_bin():
    """the C restatement (checker); built from oracle/ with gcc when the prebuilt binary is absent"""
    if not ORACLE_BIN.exists() or not ORACLE_LIB.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "oracle"], check=True, capture_output=True)
    return ORACLE_BIN


def run_oracle(oracle, spec, flags, timeout=600):
    p = subprocess.run([str(oracle), str(spec)] + list(flags), capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout.splitlines()


def strip_seconds(lines):
    import re
    pat = re.compile(r'"seconds": [0-9.]+')
    return [pat.sub('"seconds": 0.00', l) for l in lines]


def rus_cases():
    return json.loads((GOLD / "rus_cases.json").read_text())


def rus_spec_text(target):
    """a rus-spec as the reference's writer prints it: the shared blocks (table root, rotations, Cliffords, stored
    once) joined with the target's roots"""
    import gzip
    with gzip.open(GOLD / "rus" / "common.rspec.gz", "rt") as f:
        common = f.read()
    root, rest = common.split("\n@@\n")
    return "rus-spec 1\n" + root + (GOLD / "rus" / f"{target}.roots").read_text() + rest + "end\n"
