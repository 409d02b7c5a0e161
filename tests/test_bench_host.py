"""Host-side arithmetic of bench.py's checkpointed variant (CPU only): the
number of time steps one G G^T application runs, with and without stage-A
history windows, which is the divisor of the roofline's average step time."""
import importlib.util
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("daw_bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _count(nt, k):
    """Steps counted window by window, as the engine runs them: stage A over
    every window (each with its history flush step), stage A again over every
    window but the last, then stage B over the whole record."""
    if k <= 0 or k >= nt:
        return nt + 1 + nt
    wins = [min(k, nt - s0) for s0 in range(0, nt, k)]
    first_pass = sum(n + 1 for n in wins)
    recompute = sum(n + 1 for n in wins[:-1])
    return first_pass + recompute + nt


def test_op_steps_match_window_schedule():
    b = _bench()
    for nt in (1, 2, 50, 400, 7500, 10000):
        for k in (0, 1, 2, 7, 64, 750, 1673, nt - 1, nt, nt + 5):
            assert b.op_steps_per_application(nt, k) == _count(nt, k), (nt, k)


def test_checkpoint_needs_one_shot_per_launch():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--checkpoint", "10",
                        "--batch", "2"], capture_output=True, text=True, cwd=ROOT, timeout=120)
    assert r.returncode == 2
    assert "--batch 1" in r.stderr
