"""CPU: bench.py's reference arm (the reference's own CPU FFT compiled from its sources, or the C
restatement when that library is absent) prints one parseable JSON line with the keys the
benchmark contract names, and ranks other than 0 print nothing and exit 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_line():
    r = _run()
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e", "same_config"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "GB/s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert len(r.stdout.strip().splitlines()[-1]) < 2048


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_clock_summary_uses_the_timed_window():
    """Clock samples outside the timed window do not count toward the median or the reasons."""
    sys.path.insert(0, str(ROOT))
    import bench
    c = bench.ClockSampler(0)
    c.samples = [1000, 1965, 1965, 1400]
    c.times = [0.0, 1.0, 1.5, 3.0]
    c.masks = [0x4, 0, 0, 0x40]          # sw_power_cap before, hw_thermal_slowdown after the window
    c.max_mhz = 1965
    c.window = (0.9, 2.0)
    s = c.summary()
    assert s["sm_mhz"] == 1965 and s["reasons"] == [] and s["samples_in_timed_region"] == 2
    c.window = (5.0, 6.0)                # no sample inside: every sample stands in
    s = c.summary()
    assert s["samples_in_timed_region"] == 0 and "hw_thermal_slowdown" in s["reasons"]
