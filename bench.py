"""Benchmark: shots/hour of batched mixed-precision DAW redatuming on the
751x2301 (h = 4 m) model.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 4|2] [--batch B] [--checkpoint K] [--nt NT --maxiter M]

Workload (--config 4, the default: the metric's own configuration): the
751x2301 model, npml 40, dt = 0.4 ms, 15 Hz Ricker, 20 MINRES iterations,
datum receivers every 16 m at 1200 m, and the seeded 256-shot set with record
lengths nt ~ U[3000, 7500] and receiver spreads of 100-576 channels (split
offsets).  Mixed precision: FP32 stencils, FP16 wavefield histories with one
power-of-two scale per shot, step and field, FP64 MINRES scalars.  One step =
the next batch of this rank's shots, as many as HBM admits (each shot's own
nt and spread), through the whole hot path: forward modelling, the MINRES
solve (2 + 1 + 20 G G^T applications), the final extended-source simulation,
the on-the-fly datum extraction and the band-pass filter.  --config 2 runs
the uniform 50-shot variant instead (nt 7500, 576 receivers, batches of
--batch shots).  Inputs are seeded synthetic data of those shapes (the
reference publishes no data set); observed data are modelled in the true
model on the GPU before timing.  Density is 1 as in the reference
(src/submodeling2.f90:93).

`value`: device time of the batches with their inputs staged in HBM (the
stage-in is untimed).  `e2e`: the same shots through daw_shots with host
buffers, host-device copies included.  Denominators on the first timed
batch's shots: `plain_fp32` (kernel per reference loop, FP32 histories and
scalars) and `fused_fp32` (the same one-kernel-per-step kernels with FP32
histories and FP32 scalars).  `accuracy`: the mixed path against the FP64
oracle on the whole 151x461 single-shot configuration, and against the
FP32-history kernels on the timed batch.  The reference arm (--impl
reference) times the CPU restatement of the reference (FP32, one
single-threaded process per core as the reference's MPI ranks run) on a
truncated sample scaled by point updates.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as entry  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per shot time step of the pressure + velocity kernels, measured
# by ncu on the same grid
TRAFFIC = os.path.join(ROOT, "profiles", "k_tma_751x2301_traffic.json")
METRIC = "shots/hour redatumed at <=1e-3 rel err vs FP64: batched mixed vs plain FP32"


def env_int(k, d):
    return int(os.environ.get(k, d))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def make_workload(config=4, nt=None, maxiter=None):
    """The workload of --config (4: the 256-shot uneven set; 2: the uniform
    50-shot set; 5: the 2001x8001 grid, reduced to nt 1000 and 2 MINRES
    iterations unless given)."""
    w = _workload(config, nt)
    if maxiter is not None:
        w.maxiter = maxiter
    elif config == 5:
        w.maxiter = 2
    return w


def _workload(config, nt):
    entry.load_package()
    from daw_b200 import synthetic
    if config == 4:
        w = synthetic.config3(3, nshot=256)
        w.name = "cfg4"
    elif config == 5:
        w = synthetic.config5()
        w.nt = nt or 1000
        w.nts = [w.nt] * len(w.nts)
    else:
        w = synthetic.config2(2, nshot=50, nt=nt or 7500)
    return w


def workload_text(w, args):
    if w.name == "cfg5":
        return (f"2001x8001 h=5 m, npml 50, nt {w.nt} @ 0.4 ms (reduced from 10000), 1200 "
                f"receivers, 20 Hz, {w.maxiter} MINRES iterations (reduced from 30), datum at "
                f"2500 m, FP16 histories / FP64 MINRES scalars; a reduced variant, not the "
                f"benchmark")
    if w.name == "cfg4":
        return ("751x2301 h=4 m, npml 40, 256 shots with nt U[3000,7500] @ 0.4 ms and 100-576 "
                "receivers (seeded split offsets), 15 Hz, 20 MINRES iterations, datum at 1200 m, "
                "FP16 histories / FP64 MINRES scalars")
    txt = (f"751x2301 h=4 m, npml 40, nt {w.nt} @ 0.4 ms, 576 receivers, 15 Hz, {w.maxiter} MINRES "
           f"iterations, datum at 1200 m")
    if w.nt != 7500 or w.maxiter != 20:
        txt += " (reduced profiling variant with dobs = 0, not the benchmark)"
    return txt


def densities(w, args):
    """(rho of the true model, rho of the background model): None for the
    reference's rho = 1, or Gardner's relation of each velocity model."""
    if getattr(args, "density", "1") != "gardner":
        return None, None
    from daw_b200 import synthetic
    return synthetic.gardner(w.vtrue), synthetic.gardner(w.c0)


def bench_config(w, args, world):
    """The workload the line was measured on; both arms print the same."""
    return {"workload": workload_text(w, args),
            "batching": ("shots sorted by record length, as many per batch as HBM admits, "
                         "batches in seeded shuffled order"
                         if args.config == 4 else f"{args.batch} shots per batch"),
            "density": ("Gardner, rho = 0.31 vp^0.25 of each velocity model (the "
                        "configuration's; the reference runs rho = 1)"
                        if args.density == "gardner" else
                        "1 (the reference's rho = 1, src/submodeling2.f90:93)"),
            "parallelism": f"shots x{world} (para_range, no collective)",
            "stage_a_history": (f"windows of {args.checkpoint} steps (checkpointed)"
                                if args.checkpoint > 0 else "whole record"),
            "l2": "working set (30-78 GB of FP16 history per shot) far exceeds L2"}


def shot_dicts(pkg, h, w, ids, model_dobs=True, rho=(None, None)):
    """The shots `ids` of the workload; observed data modelled in the true
    model (mode 0, batched) on the GPU.  Reduced profiling variants use dobs =
    0: their records are too short for a reflection to separate the models,
    and a zero residual would stop MINRES at once, so it is not used there."""
    shots = []
    for i in ids:
        nt = w.nts[i]
        rec = pkg.subacqui(w.rec_pos[i], w.h, w.npml, w.ofs)
        src = pkg.subacqui(w.src_pos[i:i + 1], w.h, w.npml, w.ofs)[0]
        shots.append(dict(s=w.wavelet(nt), nt=nt, src=src, rec=rec, mu=w.mu, maxiter=w.maxiter,
                          rtol=0.0, band=w.band, shot=i + 1))
    if model_dobs:
        h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs, rho=rho[0])
        data = h.submodeling_shots(shots)
        for sh, d in zip(shots, data):
            sh["dobs"] = d
    else:
        for sh in shots:
            sh["dobs"] = np.zeros((sh["nt"], sh["rec"].shape[0]), np.float32, order="F")
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs, rho=rho[1])
    h.set_datum(pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs))
    return shots


def stage_batch(pkg, h, shots, start, cap):
    """Stages the longest run of shots from `start` (at most `cap`) that HBM
    admits as one batch; returns its length."""
    k = min(cap, len(shots) - start)
    while k >= 1:
        try:
            h.stage_shots(shots[start:start + k])
            return k
        except pkg.DawError as e:
            if e.code != -2 or k == 1:
                raise
            k -= 1
    raise RuntimeError("no shot admitted")


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.path = os.path.join(tempfile.mkdtemp(prefix="daw_clocks_"), f"clocks_{device}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device),
                                       f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.send_signal(signal.SIGTERM)
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline (the oracle restatement of the reference, FP32)
# ---------------------------------------------------------------------------
SAMPLE_NT = 100


def _cpu_worker(args):
    import __graft_entry__ as e
    O = e.load_oracle()
    sample_nt, shot = args
    w = make_workload(2)
    rec = O.acqui_table(w.rec_pos[0], w.h, w.npml, w.ofs)
    src = O.acqui_table(w.src_pos[shot:shot + 1], w.h, w.npml, w.ofs)[0]
    s = w.wavelet(w.nt)[:sample_nt]
    dobs = np.zeros((sample_nt, rec.shape[0]), np.float32, order="F")
    t0 = time.perf_counter()
    upd = O.baseline_sample(w.c0, w.npml, w.h, w.ofs, sample_nt, w.dt, s, src, rec, dobs, w.mu, 1)
    return time.perf_counter() - t0, upd


def cpu_baseline(w, max_procs=None, sample_nt=SAMPLE_NT):
    """The FP32 CPU restatement on every host core (one single-threaded
    process per core), each process one 751x2301 shot truncated to sample_nt
    steps and one MINRES iteration; scaled by point updates to the workload's
    mean shot."""
    ne = (w.n1 + 2 * w.npml) * (w.n2 + 2 * w.npml)
    mean_nt = float(np.mean(w.nts))
    full = (7 + 2 * w.maxiter) * mean_nt * ne  # point updates of the mean shot
    ncpu = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 16 << 30
    per_proc = 3 * w.n1 * w.n2 * sample_nt * 4 + 12 * ne * 4 + (256 << 20)
    procs = max(1, min(ncpu, int(avail * 0.6 // per_proc), max_procs or ncpu))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(sample_nt, i % 50) for i in range(procs)])
    wall = time.perf_counter() - t0
    t_sample = max(r[0] for r in res)
    upd = res[0][1]
    t_shot = t_sample * full / upd
    value = procs * 3600.0 / t_shot
    return dict(value=value, unit="shots/hour", cores=procs, kind="port",
                sample=(f"{procs} single-threaded processes (one per core), each one 751x2301 "
                        f"shot truncated to nt={sample_nt} with 1 MINRES iteration "
                        f"({upd:.3g} point updates, {t_sample:.1f} s), scaled by point updates "
                        f"to the workload's mean shot ({full:.3g}); FP32 CPU restatement of the "
                        f"reference"),
                wall_s=wall, ns_per_update=t_sample / upd * 1e9)


class Cfg1Oracle:
    """The whole 151x461 single-shot configuration (nt 2000, 10 MINRES
    iterations) on the CPU oracle in background threads (ctypes releases the
    GIL): in FP64 as the accuracy reference of the mixed path, and in FP32
    timed, a full CPU shot that checks the point-update scaling of the CPU
    baseline's truncated samples."""

    def __init__(self, pkg):
        self.O = entry.load_oracle()
        from daw_b200 import synthetic
        w = synthetic.config1()
        self.w = w
        self.src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
        self.rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
        self.ird = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
        self.s = w.wavelet()
        self.dobs, _ = self.O.submodeling(w.vtrue, w.npml, w.h, w.ofs, w.nt, w.dt, self.s,
                                          self.src, self.rec)
        self.res = {}
        self.threads = [threading.Thread(target=self._run, args=(p,)) for p in ("f64", "f32")]
        for t in self.threads:
            t.start()

    def _run(self, prec):
        w = self.w
        t0 = time.perf_counter()
        out = self.O.daw_shot(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, self.s, self.src, self.rec,
                              self.dobs, w.mu, w.maxiter, 0.0, self.ird, w.band, prec=prec)
        self.res[prec] = (out, time.perf_counter() - t0)

    def gpu_shot(self, pkg, local):
        w = self.w
        with pkg.Handle(local, preset="mixed") as h:
            h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
            h.set_datum(self.ird)
            return h.shot(s=self.s, nt=w.nt, src=self.src, rec=self.rec, dobs=self.dobs, mu=w.mu,
                          maxiter=w.maxiter, rtol=0.0, band=w.band)

    def join(self):
        for t in self.threads:
            t.join()


# ---------------------------------------------------------------------------
def op_steps_per_application(nt, window):
    """Time steps of one G G^T application with the split kernels: stage A
    (nt steps + the history flush step) and stage B (nt steps); with history
    windows of `window` steps, stage A also re-runs every window but the last,
    each with its own flush step."""
    if window <= 0 or window >= nt:
        return 2 * nt + 1
    nwin = -(-nt // window)
    last = nt - (nwin - 1) * window
    return nt + (nt - last) + (2 * nwin - 1) + nt


def roofline(tim, w, fp16=True, rho=False):
    """The step kernels of the G G^T stages (stage A and stage B, one launch
    per time step): algorithmic bytes per shot step = 36 B per extended point
    (px, pz, vx, vz read and written, kappa read) + 3 history fields per
    interior point (written in stage A, read in stage B: 2 B each in FP16),
    over the device time of those time loops.  With a density, the two
    buoyancy coefficient fields add 8 B per extended point, and the buoyancy
    weight of stage B's velocity sources 4 B per interior point of a stage-B
    step."""
    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    ne = (w.n1 + 2 * w.npml) * (w.n2 + 2 * w.npml)
    ni = w.n1 * w.n2
    per_shot_step = 36.0 * ne + 3 * (2 if fp16 else 4) * ni + (8.0 * ne if rho else 0.0)
    shot_steps = tim["shot_steps_a"] + tim["shot_steps_b"]
    if rho:  # averaged over the stage-A and stage-B shot steps
        per_shot_step += 4.0 * ni * tim["shot_steps_b"] / max(shot_steps, 1)
    ms = tim["sim_a_ms"] + tim["sim_b_ms"]
    launches = tim["steps_a"] + tim["steps_b"]
    achieved = per_shot_step * shot_steps / (ms * 1e-3) / 1e9
    avg_ms = ms / max(launches, 1)
    bytes_per_launch = per_shot_step * shot_steps / max(launches, 1)
    traffic, note = None, None
    if rho:
        note = "the committed ncu traffic capture ran rho = 1; none for this density"
    elif os.path.exists(TRAFFIC):
        t = json.load(open(TRAFFIC))
        traffic = t["bytes_per_shot_step"] * shot_steps / max(launches, 1)
        note = t["note"]
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_note": note,
            "peak_source": "measured" if peaks else "fallback",
            "unit_of_work": "one launch of the step kernel (one time step of every shot of the "
                            "batch) in the G G^T stages",
            "bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_ms,
            "bytes_per_shot_step": per_shot_step}


def reference_runs(pkg, local, shots, base_out):
    """The plain FP32 port and the FP32-history step kernels on `shots`, one
    staged batch at a time; shots/hour of each and the mixed path's error
    against the FP32-history outputs."""
    res = {}
    for name, preset, opt in (("plain_fp32", "plain", {}),
                              ("fused_fp32", "mixed", {"history": 0, "scalars": 0})):
        with pkg.Handle(local, preset=preset, **opt) as h:
            h.set_model(*base_out["model"], rho=base_out["rho"])
            h.set_datum(base_out["datum"])
            ms, outs, launches, i = 0.0, [], 0, 0
            try:
                while i < len(shots):
                    k = stage_batch(pkg, h, shots, i, len(shots))
                    h.reset_timing()
                    ms += h.run_staged()
                    launches += h.timing()["kernel_launches"]
                    outs += h.fetch_staged(outputs=("deltade", "redatumed"))
                    i += k
            except pkg.DawError as e:
                if e.code != -2:
                    raise
                # the plain port keeps whole FP32 histories (no windows)
                res[name] = {"unavailable": f"does not fit the GPU: {e}", "outs": None}
                continue
            res[name] = {"value": len(shots) * 3600.0 / (ms * 1e-3), "unit": "shots/hour",
                         "ms": ms, "shots": len(shots), "kernel_launches": int(launches),
                         "outs": outs}
    return res


def cfg5_checks(pkg, h, w, shots, args):
    """2001x8001: the history window HBM admission picks for one full
    10000-step shot, and, on the reduced shot, the whole-record outputs
    against windows of nt/4 steps (equal bit for bit by construction)."""
    ne = (w.n1 + 2 * w.npml) * (w.n2 + 2 * w.npml)
    n1h = ((w.npml - (w.npml & ~7)) + w.n1 + 7) // 8 * 8
    hist_step = 3 * n1h * w.n2 * 2
    full = dict(shots[0])
    full.update(nt=10000, s=w.wavelet(10000),
                dobs=np.zeros((10000, full["rec"].shape[0]), np.float32, order="F"))
    _, win_full = h.admit_shots([full])
    out = {"history_bytes_per_step_fp16": hist_step,
           "whole_history_bytes_nt10000": hist_step * 10000,
           "state_bytes": 5 * ne * 4,
           "auto_window_nt10000": win_full,
           "auto_windows_nt10000": -(-10000 // win_full) if win_full else 1}
    k = max(1, w.nt // 4)
    outs = {}
    for name, ck in (("whole", 0), ("windows", k)):
        h.set_options(checkpoint=ck)
        h.stage_shots(shots[:1])
        h.reset_timing()
        ms = h.run_staged()
        outs[name] = h.fetch_staged(outputs=("deltade", "redatumed"))[0]
        out[f"{name}_ms"] = ms
    h.set_options(checkpoint=args.checkpoint)
    out["window_checked"] = k
    out["windows_vs_whole_rel_l2"] = {
        key: rel(outs["windows"][key], outs["whole"][key]) for key in ("deltade", "redatumed")}
    return out


def run_ours(args):
    pkg = entry.load_package()
    from daw_b200 import ranks
    rank, world, local = ranks.rank_env()
    dist = ranks.init_group(world)
    w = make_workload(args.config, args.nt, args.maxiter)
    reduced = args.config == 2 and (w.nt != 7500 or w.maxiter != 20)
    # variants (reduced records, the 2001x8001 grid) skip the CPU arms
    variant = reduced or args.config == 5
    cfg1 = None
    if rank == 0 and world == 1 and not variant and not args.no_accuracy:
        cfg1 = Cfg1Oracle(pkg)  # CPU threads overlap the GPU timing
    # this rank's shots (para_range of the shot set), cycled when a run needs more
    nsh = len(w.src_pos)
    ista, iend = ranks.para_range(1, nsh, world, rank)
    mine = list(range(ista - 1, iend))
    cap = args.batch if args.config == 2 else 8
    h = pkg.Handle(local, preset="mixed", checkpoint=args.checkpoint,
                   step={"split": 0, "step": 1, "auto": 2}[args.kernel], tile_cols=args.tile_cols,
                   ctas_per_sm=args.ctas_per_sm, pdl=1 if args.pdl else 0)
    if args.config in (2, 5):
        per_step = args.batch
        need = per_step
    else:
        need = min(len(mine), 4 * (args.warmup + args.steps))
    ids = [mine[i % len(mine)] for i in range(need)]
    # reduced records end before a reflection separates the true and
    # background models: observed data zero (residual = -datar) there
    rho = densities(w, args)
    shots = shot_dicts(pkg, h, w, ids, model_dobs=not variant, rho=rho)
    cfg5 = cfg5_checks(pkg, h, w, shots, args) if args.config == 5 else None
    # config 4: batches of similar record lengths (the shots sorted by nt,
    # each batch as many as HBM admits, as daw_shots forms them), run in a
    # seeded shuffled order so the warm-up and timed steps draw a
    # representative mix of the set's record lengths; config 2: the same
    # batch each step
    batches = []
    if args.config == 4:
        srt = sorted(shots, key=lambda sh: -sh["nt"])
        i = 0
        while i < len(srt):
            k = min(h.admit_shots(srt[i:i + cap])[0], cap)
            batches.append(srt[i:i + k])
            i += k
        np.random.default_rng(4).shuffle(batches)
    pos = 0
    dev_ms, step_shots = [], []
    first_batch = None

    timed_batches = []

    def one_step(timed):
        nonlocal pos, first_batch
        if args.config in (2, 5):
            if pos == 0:
                stage_batch(pkg, h, shots, 0, cap)
                pos = 1
            k = len(shots)
        else:
            bt = batches[pos % len(batches)]
            k = stage_batch(pkg, h, bt, 0, len(bt))
            if timed and first_batch is None:
                first_batch = bt[:k]
            if timed:
                timed_batches.append(bt[:k])
            pos += 1
        ms = h.run_staged()
        if timed:
            dev_ms.append(ms)
            step_shots.append(k)
        return k

    for _ in range(args.warmup):
        one_step(False)
    if args.config in (2, 5):
        first_batch = shots
    h.reset_timing()
    ranks.barrier(dist)
    with Clocks(local) as clk:
        for _ in range(args.steps):
            one_step(True)
    ranks.barrier(dist)
    tim = h.timing()
    total_ms = ranks.max_over_ranks(dist, sum(dev_ms))
    shots_done = ranks.sum_over_ranks(dist, sum(step_shots))
    value = shots_done * 3600.0 / (total_ms * 1e-3)
    roof = roofline(tim, w, rho=rho[1] is not None)
    upd_per_s = tim["point_updates"] / (sum(dev_ms) * 1e-3) * world
    # mixed outputs of the first timed batch (accuracy against FP32 histories)
    mixed_first = None
    if rank == 0 and not args.no_plain:
        k = stage_batch(pkg, h, first_batch, 0, len(first_batch))
        h.run_staged()
        mixed_first = h.fetch_staged(outputs=("deltade", "redatumed"))[:k]
        first_batch = first_batch[:k]
    # e2e through the public API with host buffers (daw_shots forms its batches)
    e2e = None
    if not args.no_e2e:
        # the shots of the first two timed steps (config 2: the batch), with
        # the device-timed throughput of the same shots beside
        nb = min(2, len(dev_ms))
        e2e_shots = ([sh for bt in timed_batches[:nb] for sh in bt] if timed_batches
                     else first_batch)
        same = (sum(len(bt) for bt in timed_batches[:nb]) * 3600.0 / (sum(dev_ms[:nb]) * 1e-3)
                if timed_batches else value / world)
        t0 = time.perf_counter()
        outs = h.shots(e2e_shots, outputs=("deltade", "redatumed"))
        e2e_s = time.perf_counter() - t0
        h_bytes = sum(sh["s"].nbytes + sh["dobs"].nbytes + sh["rec"].nbytes for sh in e2e_shots)
        d_bytes = sum(o["deltade"].nbytes + o["redatumed"].nbytes for o in outs)
        e2e = {"value": len(e2e_shots) * 3600.0 / e2e_s * world, "unit": "shots/hour",
               "h2d_bytes_per_step": int(h_bytes / max(nb, 1)),
               "d2h_bytes_per_step": int(d_bytes / max(nb, 1)),
               "shots": len(e2e_shots), "device_value_same_shots": same * world,
               "note": "daw_shots with host buffers on the shots of the first two timed steps "
                       "(wall clock: H2D of wavelets, tables and observed data, the batches, "
                       "D2H of deltade and the redatumed gathers)"}
    model = (w.c0, w.npml, w.h, w.dt, w.ofs)
    datum = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
    h.close()
    del h
    plain = fused = acc = None
    if rank == 0 and not args.no_plain:
        refs = reference_runs(pkg, local, first_batch,
                              {"model": model, "datum": datum, "rho": rho[1]})
        out32 = refs["fused_fp32"].pop("outs")
        outp = refs["plain_fp32"].pop("outs")
        per_shot_value = value / world
        plain, fused = refs["plain_fp32"], refs["fused_fp32"]
        # the denominators ran the first timed batch's shots; the mixed path's
        # shots/hour on the same shots comes from its device time per shot-step
        mixed_same = None
        if args.config == 4:
            mixed_same = len(first_batch) * 3600.0 / (dev_ms[0] * 1e-3)
        if "value" in plain:
            plain["ratio_mixed_over_plain"] = (mixed_same or per_shot_value) / plain["value"]
            plain["mixed_vs_plain_rel_l2"] = {
                "redatumed": max(rel(a["redatumed"], b["redatumed"])
                                 for a, b in zip(mixed_first, outp)),
                "deltade": max(rel(a["deltade"], b["deltade"]) for a, b in zip(mixed_first, outp))}
        fused["ratio_mixed_over_fused_fp32"] = (mixed_same or per_shot_value) / fused["value"]
        acc = {"batch_mixed_vs_fp32_history": {
            "shots": [sh["shot"] for sh in first_batch],
            "redatumed": max(rel(a["redatumed"], b["redatumed"]) for a, b in zip(mixed_first, out32)),
            "deltade": max(rel(a["deltade"], b["deltade"]) for a, b in zip(mixed_first, out32)),
            "note": "max over the batch's shots of rel. L2 against the same kernels with FP32 "
                    "histories and FP32 MINRES scalars, full nt and 20 iterations"}}
    cpu = None
    if cfg1 is not None:
        g1 = cfg1.gpu_shot(pkg, local)
        cfg1.join()
        r64, t64 = cfg1.res["f64"]
        r32, t32 = cfg1.res["f32"]
        acc = acc or {}
        acc["cfg1_mixed_vs_f64"] = {
            k: rel(g1[k], r64[k]) for k in ("datar", "deltade", "dataesc", "datae",
                                            "redatumed_raw", "redatumed")}
        acc["cfg1_mixed_vs_f64"]["workload"] = ("151x461 h=20 m, npml 20, nt 2000, 230 receivers, "
                                                "10 MINRES iterations, whole shot")
        cw = cfg1.w
        cfg1_upd = (7 + 2 * cw.maxiter) * cw.nt * (cw.n1 + 2 * cw.npml) * (cw.n2 + 2 * cw.npml)
        cfg1_full = {"seconds": t32, "ns_per_update": t32 / cfg1_upd * 1e9,
                     "note": "one whole 151x461 shot (nt 2000, 10 iterations) of the FP32 CPU "
                             "restatement, one thread, timed while the GPU bench ran"}
    if rank == 0 and world == 1 and not args.no_cpu and not variant:
        print(json.dumps({"partial": True, "value": value, "e2e": e2e, "plain_fp32": plain}),
              file=sys.stderr, flush=True)
        try:
            cpu = cpu_baseline(w, args.cpu_procs)
            if cfg1 is not None:
                cpu["full_shot_check"] = cfg1_full
        except Exception as ex:  # the GPU line is still reported
            cpu = {"error": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        tc = {m: {"family": ["p+v kernels", "one kernel per step"][tim["kernel_family"][i]],
                  "tile": f"64x{tim['tile_cols'][i]}",
                  "ctas_per_sm": ([tim["ctas_per_sm"][i], tim["ctas_per_sm_v"][i]]
                                  if tim["kernel_family"][i] == 0 else tim["ctas_per_sm"][i]),
                  "shots_per_launch": tim["shots_per_launch"][i]}
              for i, m in enumerate(("forward", "stage_a", "stage_b", "esource"))}
        result = {
            "metric": METRIC, "value": value, "unit": "shots/hour", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 stencil / f16 history / f64 scalars",
            "data": "synthetic (seeded; observed data modelled in the true model)",
            "config": bench_config(w, args, world),
            "run": {"shots_per_step": [int(x) for x in step_shots],
                    "shots_timed": int(shots_done),
                    "kernel": {"auto": "TMA time-step kernels, family and launch shape "
                                       "autotuned per mode",
                               "split": "TMA pressure and velocity kernels, shots per launch "
                                        "and CTAs per SM autotuned per mode",
                               "step": "one TMA kernel per time step (p recomputed on the "
                                       "v halo)"}[args.kernel]
                              + (", programmatic dependent launch" if args.pdl else ""),
                    "autotuned": tc},
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(tim["kernel_launches"]),
            "grid_point_updates_per_s": upd_per_s,
            "roofline": roof,
            "plain_fp32": plain,
            "fused_fp32": fused,
            "accuracy": acc,
            "cpu_baseline": cpu,
            "cfg5": cfg5,
            "timing_ms": {k: tim[k] for k in ("forward_ms", "operator_ms", "minres_vec_ms",
                                              "esource_ms", "filter_ms")},
        }
        print(json.dumps(result), flush=True)
    if dist:
        ranks.barrier(dist)
        dist.destroy_process_group()


def run_reference(args):
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    if rank != 0:
        return
    w = make_workload(args.config, args.nt, args.maxiter)
    K, W = args.steps, args.warmup
    vals = []
    for i in range(W + K):
        r = cpu_baseline(w, args.cpu_procs, sample_nt=args.ref_sample_nt)
        if i >= W:
            vals.append(r)
    value = statistics.median(v["value"] for v in vals)
    r = vals[-1]
    step_ms = 1e3 * statistics.mean(v["wall_s"] for v in vals)  # one bounded sample per step
    out = {"metric": METRIC, "value": value, "unit": "shots/hour", "n_gpus": world,
           "steps": K, "warmup": W, "higher_is_better": True, "impl": "reference",
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": bench_config(w, args, world),
           "cpu_baseline": {"value": value, "unit": "shots/hour", "cores": r["cores"],
                            "kind": "port", "sample": r["sample"]},
           "e2e": {"value": value, "unit": "shots/hour", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "ms_per_step": step_ms,
           "extrapolated_ms_per_shot_per_core": 3600e3 * r["cores"] / value}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=4, choices=[2, 4, 5])
    ap.add_argument("--batch", type=int, default=None,
                    help="--config 2 / 5: shots per batch (default 2 / 1)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=None)
    # reference arm: truncated record of each CPU sample (one per step)
    ap.add_argument("--ref-sample-nt", type=int, default=40)
    # profiling variants of the uniform workload (shorter records / fewer
    # iterations, same grid and kernels); a line printed with them is marked
    ap.add_argument("--nt", type=int, default=7500)
    ap.add_argument("--maxiter", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    # A/B: the one-kernel-per-step path (default) or the split p / v kernels
    # the TMA kernel family: autotuned (default), split p / v kernels, or one per step
    ap.add_argument("--kernel", default="split", choices=["split", "step", "auto"])
    ap.add_argument("--pdl", action="store_true",
                    help="programmatic dependent launch between steps (default: stream order)")
    # pin the step kernel's tile width / CTAs per SM (0 = autotuned)
    ap.add_argument("--tile-cols", type=int, default=0, choices=[0, 16, 32])
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    # stage-A history in windows of K steps (checkpointed; one shot per launch)
    ap.add_argument("--checkpoint", type=int, default=0)
    ap.add_argument("--density", default="1", choices=["1", "gardner"],
                    help="rho = 1 (the reference's) or Gardner's rho = 0.31 vp^0.25")
    args = ap.parse_args()
    if args.batch is None:
        args.batch = 1 if args.config == 5 else 2
    if args.config == 5 and args.nt == 7500:
        args.nt = 1000
    if args.checkpoint > 0 and (args.batch != 1 or args.config == 4):
        ap.error("--checkpoint runs one shot per launch: give --config 2 --batch 1")
    if (args.nt != 7500 or args.maxiter is not None) and args.config == 4:
        ap.error("--nt / --maxiter are profiling variants of --config 2 and 5")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
