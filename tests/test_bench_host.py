"""Host-side arithmetic of bench.py (CPU only): the number of time steps one
G G^T application runs, with and without stage-A history windows (the
divisor of the roofline's average step time), the roofline's algorithmic
bytes with and without a density, and the Gardner density of its density
switch."""
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


def test_roofline_bytes_with_density():
    """Algorithmic bytes per shot step: 36 B per extended point + 6 B of FP16
    history per interior point; a density adds the two buoyancy coefficient
    fields (8 B per extended point) and stage B's buoyancy weight (4 B per
    interior point of a stage-B step, here half the shot steps)."""
    from types import SimpleNamespace
    b = _bench()
    w = SimpleNamespace(n1=751, n2=2301, npml=40)
    tim = dict(shot_steps_a=100, shot_steps_b=100, sim_a_ms=2.0, sim_b_ms=2.0, steps_a=50,
               steps_b=50)
    ne, ni = 831 * 2381, 751 * 2301
    r1 = b.roofline(tim, w)
    r2 = b.roofline(tim, w, rho=True)
    assert r1["bytes_per_shot_step"] == 36 * ne + 6 * ni
    assert r2["bytes_per_shot_step"] == 36 * ne + 6 * ni + 8 * ne + 2 * ni
    assert r2["traffic"] is None  # the committed traffic capture ran density 1
    assert abs(r2["achieved"] / r1["achieved"] - r2["bytes_per_shot_step"] / r1["bytes_per_shot_step"]) < 1e-12


def test_gardner_density():
    import numpy as np
    b = _bench()
    b.entry.load_package()
    from daw_b200 import synthetic
    rho = synthetic.gardner(np.array([[1500.0, 2000.0], [4000.0, 5500.0]]))
    assert rho.dtype == np.float32 and rho.flags.f_contiguous
    assert np.allclose(rho, 0.31 * np.array([[1500.0, 2000.0], [4000.0, 5500.0]]) ** 0.25, rtol=1e-6)
    from types import SimpleNamespace
    w = SimpleNamespace(vtrue=np.full((3, 4), 2000.0), c0=np.full((3, 4), 1500.0))
    rt, r0 = b.densities(w, SimpleNamespace(density="gardner"))
    assert rt.shape == (3, 4) and abs(float(rt[0, 0]) - 0.31 * 2000.0 ** 0.25) < 1e-5
    assert abs(float(r0[0, 0]) - 0.31 * 1500.0 ** 0.25) < 1e-5
    assert b.densities(w, SimpleNamespace(density="1")) == (None, None)


def test_reference_arm_prints_the_same_config():
    """Both arms describe the workload with one dict (bench_config), so the
    reference arm's line carries exactly the config of the measured arm."""
    import json
    from types import SimpleNamespace
    b = _bench()
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0", "--ref-sample-nt", "2", "--cpu-procs", "2"],
                       capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    args = SimpleNamespace(config=4, batch=2, density="1", checkpoint=0)
    assert line["config"] == b.bench_config(b.make_workload(4), args, 1)
    assert line["impl"] == "reference" and line["steps"] == 1
