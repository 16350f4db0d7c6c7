"""bench.py's command line and dispatch (CPU): every configuration and arm
resolves to a function, and --help runs."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_every_arm_has_its_function():
    for name in ("run_own", "run_c5", "run_reference", "reference_program", "reference_gpu", "cpu_baseline",
                 "safe_reference_threads", "run_reference_program", "timed_epochs", "single_job_epochs"):
        assert callable(getattr(bench, name)), name


def test_help_runs():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "--impl" in r.stdout and "--per-epoch" in r.stdout


def test_clock_summary_reads_median_clock_and_active_reasons():
    c = bench.ClockSampler(0)
    c.lines = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 800.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 1.0, 0x0, Not Active, Active, Not Active, Not Active",
    ]
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["hw_thermal_slowdown", "sw_power_cap"],
                 "samples": 3}


def test_clock_summary_without_samples_is_none():
    assert bench.ClockSampler(0).summary() is None


def test_peaks_come_from_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6552.3}')
    assert bench.peaks() == (6552.3, "measured")
