"""Seeded synthetic workloads with the shapes of the five benchmark
configurations (the reference publishes no data set; its Marmousi demo inputs
come from external generators that are not in its repository).

Each config builds a true model (for the observed data), a background model
c0 (the smooth trend of the true model, as the demo's gradient vinit), a
Ricker wavelet already divided by h^2 (main_redatum_DAW.f90:111), the source
and receiver tables in the subacqui layout, datum receivers and the filter
band.  Observed data are modelled in the true model by the caller (mode 0).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Workload:
    name: str
    n1: int
    n2: int
    h: float
    npml: int
    dt: float
    nt: int
    f0: float
    ofs: int
    mu: float
    maxiter: int
    rtol: float
    vtrue: np.ndarray
    c0: np.ndarray
    src_pos: np.ndarray       # (nshot, 2) z, x
    rec_pos: list             # per shot (nrec_i, 2)
    datum_pos: np.ndarray     # (nd, 2)
    nts: list                 # per-shot record lengths
    band: tuple

    def wavelet(self, nt: int | None = None) -> np.ndarray:
        nt = nt or self.nt
        t = np.arange(nt) * self.dt - 1.2 / self.f0
        a = (np.pi * self.f0 * t) ** 2
        return (((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32) / np.float32(self.h * self.h))


def gardner(vp) -> np.ndarray:
    """Gardner's density rho = 0.31 vp^0.25 (g/cm^3, vp in m/s) of a velocity
    model, the density the benchmark configurations name (the reference
    itself runs rho = 1)."""
    return np.asfortranarray((0.31 * np.asarray(vp, np.float64) ** 0.25).astype(np.float32))


def ricker_band(f0):
    # flow = 0.5 f0, fhig = 2.5 f0, llow = lhig = 0.5 f0
    return (0.5 * f0, 2.5 * f0, 0.5 * f0, 0.5 * f0)


def _layers(rng, n1, h, v0, v1, nlayer, jump):
    z = np.arange(n1) * h
    v = v0 + (v1 - v0) * z / z[-1]
    bounds = np.sort(rng.uniform(0.1, 0.95, nlayer)) * z[-1]
    for b in bounds:
        v = v + np.where(z >= b, rng.uniform(-jump, jump), 0.0)
    return v, v0 + (v1 - v0) * z / z[-1]


def config1(seed: int = 1, nt: int = 2000) -> Workload:
    """Plain DAW, 1 shot: 151x461, h=20, gradient 1500->4000 + 8 layers."""
    rng = np.random.default_rng(seed)
    n1, n2, h = 151, 461, 20.0
    v, trend = _layers(rng, n1, h, 1500.0, 4000.0, 8, 200.0)
    vtrue = np.repeat(v[:, None], n2, axis=1).astype(np.float32)
    c0 = np.repeat(trend[:, None], n2, axis=1).astype(np.float32)
    rec = np.array([[20.0, x] for x in np.arange(0.0, 9160.0 + 1, 40.0)], np.float32)
    datum = np.array([[1000.0, x] for x in np.arange(0.0, 9160.0 + 1, 40.0)], np.float32)
    return Workload("cfg1", n1, n2, h, 20, 0.0015, nt, 10.0, 1, 1e-2, 10, 0.0,
                    np.asfortranarray(vtrue), np.asfortranarray(c0),
                    np.array([[10.0, 4600.0]], np.float32), [rec], datum, [nt],
                    ricker_band(10.0))


def _faulted_model(rng, n1, n2, h, vmin, vmax):
    z = (np.arange(n1) * h)[:, None]
    x = (np.arange(n2) * h)[None, :]
    zmax, xmax = z.max(), x.max()
    trend = vmin + (vmax - vmin) * (z / zmax) ** 0.8 + 0 * x
    v = trend.copy()
    dip = np.tan(np.deg2rad(rng.uniform(-8, 8)))
    nl = 14
    bounds = np.sort(rng.uniform(0.05, 0.95, nl)) * zmax
    jumps = rng.uniform(-250, 350, nl)
    faults = np.sort(rng.uniform(0.2, 0.8, 3)) * xmax
    throws = rng.uniform(40, 160, 3)
    for b, j in zip(bounds, jumps):
        depth = b + dip * (x - xmax / 2)
        for f, t in zip(faults, throws):
            depth = depth + np.where(x > f + 0.3 * (z - b), t, 0.0)
        v = v + np.where(z >= depth, j, 0.0)
    # high-velocity wedge
    wz0, wx0 = 0.45 * zmax, 0.3 * xmax
    wedge = (z > wz0) & (z < wz0 + 0.25 * (x - wx0)) & (x > wx0)
    v = np.where(wedge, vmax * 0.95, v)
    v = np.clip(v, vmin, vmax)
    return v.astype(np.float32), np.clip(trend, vmin, vmax).astype(np.float32)


def config2(seed: int = 2, nshot: int = 50, nt: int = 7500) -> Workload:
    """751x2301 at h=4, faulted dipping layers 1500-5500, 50 shots, 576 receivers."""
    rng = np.random.default_rng(seed)
    n1, n2, h = 751, 2301, 4.0
    vtrue, c0 = _faulted_model(rng, n1, n2, h, 1500.0, 5500.0)
    xs = 190.0 + 180.0 * np.arange(nshot)
    src = np.stack([np.full(nshot, 8.0), xs], 1).astype(np.float32)
    rec = np.array([[12.0, 16.0 * i] for i in range(576)], np.float32)
    datum = np.array([[1200.0, 16.0 * i] for i in range(576)], np.float32)
    return Workload("cfg2", n1, n2, h, 40, 0.0004, nt, 15.0, 1, 1e-2, 20, 0.0,
                    np.asfortranarray(vtrue), np.asfortranarray(c0), src,
                    [rec] * nshot, datum, [nt] * nshot, ricker_band(15.0))


def config3(seed: int = 3, nshot: int = 256) -> Workload:
    """cfg2 model, 256 shots, nt ~ U[3000,7500], spreads of 100-576 channels.
    The sources are spread evenly over the model (100 m .. 9100 m at z = 8 m):
    the 180 m spacing of the 50-shot set would run off the 9.2 km model."""
    base = config2(2, nshot=nshot)
    base.src_pos = np.stack([np.full(nshot, 8.0), np.linspace(100.0, 9100.0, nshot)],
                            1).astype(np.float32)
    rng = np.random.default_rng(seed)
    nts = rng.integers(3000, 7501, nshot).tolist()
    recs = []
    allrec = np.array([[12.0, 16.0 * i] for i in range(576)], np.float32)
    for i in range(nshot):
        k = int(rng.integers(100, 577))
        lo = int(rng.integers(0, 576 - k + 1))
        recs.append(allrec[lo:lo + k].copy())
    base.name = "cfg3"
    base.rec_pos = recs
    base.nts = nts
    base.nt = max(nts)
    return base


def config5(seed: int = 5) -> Workload:
    """2001x8001 at h=5 with a rugose salt body, 1024 shots, nt=10000."""
    rng = np.random.default_rng(seed)
    n1, n2, h = 2001, 8001, 5.0
    v, trend = _faulted_model(rng, n1, n2, h, 1480.0, 6000.0)
    x = np.arange(n2) * h
    curve = 0.45 * n1 * h + sum(rng.uniform(-1, 1) * 300.0 / (k + 1) *
                                np.sin(2 * np.pi * (k + 1) * x / x[-1] + rng.uniform(0, 6.3))
                                for k in range(12))
    z = (np.arange(n1) * h)[:, None]
    salt = (z > curve[None, :]) & (z < curve[None, :] + 2500.0)
    v = np.where(salt, 4500.0, v).astype(np.float32)
    src = np.stack([np.full(1024, 10.0), 39.0 * np.arange(1024)], 1).astype(np.float32)
    rec = np.array([[10.0, 12.5 * i] for i in range(1200)], np.float32)
    datum = np.array([[2500.0, 12.5 * i] for i in range(1200)], np.float32)
    return Workload("cfg5", n1, n2, h, 50, 0.0004, 10000, 20.0, 1, 1e-2, 30, 0.0,
                    np.asfortranarray(v), np.asfortranarray(trend.astype(np.float32)), src,
                    [rec] * 1024, datum, [10000] * 1024, ricker_band(20.0))


def small(seed: int = 7, n1: int = 60, n2: int = 90, nt: int = 400, nrec: int = 24,
          nshot: int = 1, npml: int = 12, h: float = 10.0, dt: float = 0.002,
          f0: float = 10.0, maxiter: int = 4) -> Workload:
    """A seconds-sized case with the structure of cfg1, for parity tests
    (nto*dt >= 1 so the filter's integer bin spacing is not degenerate)."""
    rng = np.random.default_rng(seed)
    v, trend = _layers(rng, n1, h, 1500.0, 2600.0, 5, 150.0)
    vtrue = np.repeat(v[:, None], n2, axis=1).astype(np.float32)
    vtrue += rng.uniform(-30, 30, vtrue.shape).astype(np.float32)
    c0 = np.repeat(trend[:, None], n2, axis=1).astype(np.float32)
    xmax = (n2 - 1) * h
    xs = np.linspace(0.3, 0.7, nshot) * xmax if nshot > 1 else np.array([0.47 * xmax])
    src = np.stack([np.full(nshot, 1.5 * h), xs], 1).astype(np.float32)
    rec = np.stack([np.full(nrec, 2.0 * h), np.linspace(0, xmax, nrec)], 1).astype(np.float32)
    datum = np.stack([np.full(nrec // 2, 0.6 * (n1 - 1) * h),
                      np.linspace(0.1 * xmax, 0.9 * xmax, nrec // 2)], 1).astype(np.float32)
    return Workload("small", n1, n2, h, npml, dt, nt, f0, 1, 1e-2, maxiter, 0.0,
                    np.asfortranarray(vtrue), np.asfortranarray(c0), src,
                    [rec] * nshot, datum, [nt] * nshot, ricker_band(f0))


CONFIGS = {"cfg1": config1, "cfg2": config2, "cfg3": config3, "cfg5": config5, "small": small}
