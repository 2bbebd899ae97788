"""CPU: compile the real host runtime (plan.cpp, acceptance.cpp, capi.cpp) against the fake
device seam and run its guard / fault-injection / autotuner checks (no GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "ascend-fft_b200" / "csrc"


@pytest.mark.skipif(not shutil.which("g++"), reason="g++ required")
def test_host_runtime_guards(tmp_path):
    exe = tmp_path / "guards"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", str(ROOT / "include"), "-I", str(CSRC),
           str(ROOT / "tests" / "host" / "test_runtime_guards.cpp"),
           str(ROOT / "tests" / "host" / "fake_backend.cpp"),
           str(CSRC / "plan.cpp"), str(CSRC / "acceptance.cpp"), str(CSRC / "capi.cpp"),
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(ROOT / "ascend-fft_b200" / "config"), str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
