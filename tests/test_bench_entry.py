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
