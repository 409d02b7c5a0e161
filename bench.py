"""Benchmark: shots/hour of DAW redatuming on the 751x2301 (h = 4 m) model.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one batch of shots through the whole hot path): the
751x2301 model, npml 40, nt = 7500 at dt = 0.4 ms, 576 receivers every 16 m,
15 Hz Ricker, 20 MINRES iterations, datum receivers at 1200 m; every shot is
forward modelling, the MINRES solve of the data-assimilation normal equation
(2 + 1 + 20 G G^T applications), the final extended-source simulation, the
on-the-fly datum extraction and the band-pass filter.  Inputs are seeded
synthetic data of those shapes (the reference publishes no data set).

`value`: mixed path (FP32 stencils, FP16 histories with per-step power-of-two
scales, FP64 MINRES scalars), shots batched per launch, inputs resident in
HBM.  `e2e`: the same through daw_shots with host buffers.  `plain_fp32`: the
plain FP32 GPU port (kernel per reference loop, FP32 histories) on one shot of
the same workload.  The reference arm (--impl reference) times the CPU
restatement of the reference (FP32, one single-threaded process per core as
the reference's MPI ranks run) on a truncated sample scaled by point updates.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as entry  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes of one G G^T time step (p + v kernels), measured by ncu on the
# same grid and batch
TRAFFIC = os.path.join(ROOT, "profiles", "k_tma_751x2301_traffic.json")
METRIC = "shots/hour redatumed at <=1e-3 rel err vs FP64: batched mixed vs plain FP32"


def env_int(k, d):
    return int(os.environ.get(k, d))


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_workload(nt=None):
    entry.load_package()
    from daw_b200 import synthetic
    w = synthetic.config2(2, nshot=50, nt=nt or 7500)
    return w


def shot_dicts(pkg, h, w, shot_ids, model_dobs=True):
    """Observed data are modelled in the true model (mode 0) on the GPU.  The
    reduced profiling variants use dobs = 0 instead: their records are too
    short for a reflection to separate the true and background models, and a
    zero residual would stop MINRES before its first iteration."""
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    s = w.wavelet(w.nt)
    h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs)
    shots = []
    for i in shot_ids:
        src = pkg.subacqui(w.src_pos[i:i + 1], w.h, w.npml, w.ofs)[0]
        if model_dobs:
            dobs, _ = h.submodeling(s, src, rec)
        else:
            dobs = np.zeros((w.nt, rec.shape[0]), np.float32, order="F")
        shots.append(dict(s=s, nt=w.nt, src=src, rec=rec, dobs=dobs, mu=w.mu,
                          maxiter=w.maxiter, rtol=0.0, band=w.band, shot=i + 1))
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
    h.set_datum(pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs))
    return shots


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
    w = make_workload()
    from daw_b200 import synthetic  # noqa
    rec = O.acqui_table(w.rec_pos[0], w.h, w.npml, w.ofs)
    src = O.acqui_table(w.src_pos[args:args + 1], w.h, w.npml, w.ofs)[0]
    nt = SAMPLE_NT
    s = w.wavelet(w.nt)[:nt]
    dobs = np.zeros((nt, rec.shape[0]), np.float32, order="F")
    t0 = time.perf_counter()
    upd = O.baseline_sample(w.c0, w.npml, w.h, w.ofs, nt, w.dt, s, src, rec, dobs, w.mu, 1)
    return time.perf_counter() - t0, upd


def cpu_baseline(max_procs=None):
    w = make_workload()
    ne = (w.n1 + 2 * w.npml) * (w.n2 + 2 * w.npml)
    full = (7 + 2 * w.maxiter) * w.nt * ne  # point updates of one full shot
    ncpu = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 16 << 30
    per_proc = 3 * w.n1 * w.n2 * SAMPLE_NT * 4 + 12 * ne * 4 + (256 << 20)
    procs = max(1, min(ncpu, int(avail * 0.6 // per_proc), max_procs or ncpu))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [i % 50 for i in range(procs)])
    wall = time.perf_counter() - t0
    t_sample = max(r[0] for r in res)
    upd = res[0][1]
    t_shot = t_sample * full / upd
    value = procs * 3600.0 / t_shot
    return dict(value=value, unit="shots/hour", cores=procs, kind="port",
                sample=(f"{procs} single-threaded processes (one per core), each one 751x2301 "
                        f"shot truncated to nt={SAMPLE_NT} with 1 MINRES iteration "
                        f"({upd:.3g} point updates, {t_sample:.1f} s), scaled by point updates "
                        f"to the full shot ({full:.3g}); FP32 CPU restatement of the reference"),
                wall_s=wall)


# ---------------------------------------------------------------------------
def op_steps_per_application(nt, window):
    """Time steps of one G G^T application: stage A (nt steps + the history
    flush step) and stage B (nt steps); with history windows of `window`
    steps, stage A also re-runs every window but the last, each with its own
    flush step."""
    if window <= 0 or window >= nt:
        return 2 * nt + 1
    nwin = -(-nt // window)
    last = nt - (nwin - 1) * window
    return nt + (nt - last) + (2 * nwin - 1) + nt


def roofline(pkg, tim, nshots, w, steps_per_op):
    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    ne = (w.n1 + 2 * w.npml) * (w.n2 + 2 * w.npml)
    ni = w.n1 * w.n2
    # dominant work: one fused time step (pressure + velocity kernel) of the
    # G G^T stages; algorithmic bytes per shot-step: 36 B per extended point
    # (px,pz,vx,vz read+write, kappa read) + 6 B per interior point (three FP16
    # history fields written in stage A / read in stage B)
    per_step = (36.0 * ne + 6.0 * ni) * nshots
    ms = tim["operator_ms"]
    launches = steps_per_op
    avg_ms = ms / max(launches, 1)
    achieved = per_step / (avg_ms * 1e-3) / 1e9
    traffic, traffic_note = None, None
    if os.path.exists(TRAFFIC):
        t = json.load(open(TRAFFIC))
        traffic = t["step_bytes"] * nshots / t["shots_per_launch"]
        traffic_note = t["note"]
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_note": traffic_note,
            "peak_source": "measured" if peaks else "fallback",
            "unit_of_work": "one fused time step (p+v kernels) of the G G^T stages",
            "bytes_per_step": per_step, "avg_step_ms": avg_ms}


def run_ours(args):
    pkg = entry.load_package()
    from daw_b200 import ranks
    rank, world, local = ranks.rank_env()
    dist = ranks.init_group(world)
    w = make_workload(args.nt)
    if args.maxiter is not None:
        w.maxiter = args.maxiter
    B = args.batch
    # this rank's shots: the first B of its para_range block of the 50 shots
    ids = ranks.rank_shots(len(w.src_pos), B, rank, world)
    reduced = w.nt != 7500 or w.maxiter != 20  # profiling-sized variant
    h = pkg.Handle(local, preset="mixed", checkpoint=args.checkpoint)
    shots = shot_dicts(pkg, h, w, ids, model_dobs=not reduced)
    h.stage_shots(shots)
    for _ in range(args.warmup):
        h.run_staged()

    h.reset_timing()
    ranks.barrier(dist)
    dev_ms = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            dev_ms.append(h.run_staged())
    ranks.barrier(dist)
    tim = h.timing()
    total_ms = ranks.max_over_ranks(dist, sum(dev_ms))
    shots_done = B * args.steps * world
    value = shots_done * 3600.0 / (total_ms * 1e-3)
    # G G^T applications per shot: the shift's (1), the reference's unused one
    # (1) and one per MINRES iteration (rtol 0: all run); each is stage A (nt
    # steps + the history flush step) followed by stage B (nt steps)
    op_steps = op_steps_per_application(w.nt, args.checkpoint) * (2 + w.maxiter) * args.steps
    roof = roofline(pkg, tim, B, w, op_steps)
    # accuracy of the mixed path against the FP32-history fused path on the same shots
    out_mixed = h.fetch_staged(outputs=("deltade", "redatumed"))
    # e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        h.reset_timing()
        t0 = time.perf_counter()
        outs = h.shots(shots, outputs=("deltade", "redatumed"))
        e2e_s = time.perf_counter() - t0
        h_bytes = sum(sh["s"].nbytes + sh["dobs"].nbytes + sh["rec"].nbytes for sh in shots)
        d_bytes = sum(o["deltade"].nbytes + o["redatumed"].nbytes for o in outs)
        e2e = {"value": B * 3600.0 / e2e_s, "unit": "shots/hour",
               "h2d_bytes_per_step": int(h_bytes), "d2h_bytes_per_step": int(d_bytes)}
    h.close()
    del h
    result = None
    plain = None
    if rank == 0 and not args.no_plain:
        hp = pkg.Handle(local, preset="plain")
        hp.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        hp.set_datum(pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs))
        hp.stage_shots(shots[:1])
        hp.reset_timing()
        pms = hp.run_staged()
        ptim = hp.timing()
        out_plain = hp.fetch_staged(outputs=("deltade", "redatumed"))
        hp.close()
        err_red = float(np.linalg.norm(out_mixed[0]["redatumed"] - out_plain[0]["redatumed"]) /
                        np.linalg.norm(out_plain[0]["redatumed"]))
        err_de = float(np.linalg.norm(out_mixed[0]["deltade"] - out_plain[0]["deltade"]) /
                       np.linalg.norm(out_plain[0]["deltade"]))
        plain = {"value": 3600.0 / (pms * 1e-3), "unit": "shots/hour", "ms_per_shot": pms,
                 "kernel_launches": int(ptim["kernel_launches"]),
                 "mixed_vs_plain_rel_l2": {"redatumed": err_red, "deltade": err_de},
                 "ratio_mixed_over_plain": value / world / (3600.0 / (pms * 1e-3))}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not reduced:
        print(json.dumps({"partial": True, "value": value, "e2e": e2e, "plain_fp32": plain}),
              file=sys.stderr, flush=True)
        try:
            cpu = cpu_baseline(args.cpu_procs)
        except Exception as ex:  # the GPU line is still reported
            cpu = {"error": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        result = {
            "metric": METRIC, "value": value, "unit": "shots/hour", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 stencil / f16 history / f64 scalars",
            "data": "synthetic (seeded; observed data modelled in the true model)",
            "config": {"workload": f"751x2301 h=4 m, npml 40, nt {w.nt} @ 0.4 ms, 576 receivers, "
                                   f"15 Hz, {w.maxiter} MINRES iterations, datum at 1200 m"
                                   + (" (reduced profiling variant with dobs = 0, not the "
                                      "benchmark)" if reduced else ""),
                       "shots_per_step_per_gpu": B, "parallelism": f"shots x{world} (no collective)",
                       "stage_a_history": (f"windows of {args.checkpoint} steps (checkpointed)"
                                           if 0 < args.checkpoint < w.nt else "whole record"),
                       "l2": "working set (78 GB FP16 history per shot) far exceeds L2"},
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(tim["kernel_launches"]),
            "roofline": roof,
            "plain_fp32": plain,
            "cpu_baseline": cpu,
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
    K, W = args.steps, args.warmup
    vals = []
    for i in range(W + K):
        r = cpu_baseline(args.cpu_procs)
        if i >= W:
            vals.append(r)
    value = statistics.median(v["value"] for v in vals)
    r = vals[-1]
    out = {"metric": METRIC, "value": value, "unit": "shots/hour", "n_gpus": world,
           "steps": K, "warmup": W, "higher_is_better": True, "impl": "reference",
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "751x2301 h=4 m, npml 40, nt 7500 @ 0.4 ms, 576 receivers, "
                                  "15 Hz, 20 MINRES iterations, datum at 1200 m"},
           "cpu_baseline": {"value": value, "unit": "shots/hour", "cores": r["cores"],
                            "kind": "port", "sample": r["sample"]},
           "e2e": {"value": value, "unit": "shots/hour", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "ms_per_step": 3600e3 / value}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=2)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=None)
    # profiling variants of the same workload (shorter records / fewer
    # iterations, same grid and kernels); a line printed with them is marked
    ap.add_argument("--nt", type=int, default=7500)
    ap.add_argument("--maxiter", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    # stage-A history in windows of K steps (checkpointed; one shot per launch)
    ap.add_argument("--checkpoint", type=int, default=0)
    args = ap.parse_args()
    if args.checkpoint > 0 and args.batch != 1:
        ap.error("--checkpoint runs one shot per launch: give --batch 1")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
