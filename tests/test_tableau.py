"""Host checks of the Clifford-table path's tableau ranking (no GPU): the table stores only a distance per rank and
recomputes the element of a rank when it needs one, so unrank must invert rank exactly."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_unrank_inverts_rank(tmp_path):
    exe = tmp_path / "tableau_host_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", str(exe), str(ROOT / "tests" / "tableau_host_check.cpp")],
                   check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip() == "mismatches: 0"
