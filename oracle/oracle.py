"""ctypes front end of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference arms import this module, as the checker.  The product never
does.  Parity status: unpinned against the reference build (the reference is
Fortran + MPI and no Fortran compiler exists here; the reference ships no
golden vectors).  See ``daw_oracle.cpp`` for the restatement itself.

Every array follows the reference's Fortran layout: column-major ("F" order),
first index fastest; acquisition tables are (n, 5) int32 column-major.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libdaw_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="F_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="F_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="F_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _opt(ptype):
    """Pointer argument that also accepts None (NULL)."""

    class _Opt(ptype):  # type: ignore[misc, valid-type]
        @classmethod
        def from_param(cls, obj):
            if obj is None:
                return C.c_void_p(None)
            return ptype.from_param(obj)

    return _Opt


def _declare(L):
    i, f, d = C.c_int, C.c_float, C.c_double
    L.oracle_kws_tile.argtypes = [i, i, i, _f32p]
    L.oracle_kws_table1d.argtypes = [_f32p]
    L.oracle_bessi0.argtypes = [f]
    L.oracle_bessi0.restype = f
    L.oracle_subsourcekws.argtypes = [f, f, f, i, _i32p]
    L.oracle_sponges.argtypes = [i, i, _f32p, _f32p, _f32p, _f32p]
    for suf, rp in (("f32", _f32p), ("f64", _f64p)):
        getattr(L, f"oracle_submodeling_{suf}").argtypes = [
            _f32p, i, i, i, f, i, i, f, _f32p, i, i, _i32p, _i32p, i, rp, _opt(rp)]
        getattr(L, f"oracle_esource_data_{suf}").argtypes = [
            _f32p, i, i, i, f, i, i, f, rp, i, i, _i32p, rp]
        fn = getattr(L, f"oracle_esource_{suf}")
        fn.argtypes = [_f32p, i, i, i, f, i, i, f, rp, i, i, _i32p, rp, _opt(rp)]
        fn.restype = d
        getattr(L, f"oracle_resample_{suf}").argtypes = [i, i, i, i, _i32p, i, rp, rp]
        getattr(L, f"oracle_minres_{suf}").argtypes = [
            _f32p, i, i, i, f, i, i, f, i, i, _i32p, rp, f, i, f, rp, _i32p, _f64p,
            _opt(_f64p), i]
        fn = getattr(L, f"oracle_daw_shot_{suf}")
        fn.argtypes = [_f32p, i, i, i, f, i, i, f, _f32p, i, i, _i32p, _i32p, i, _f32p, f,
                       i, f, _i32p, i, f, f, f, f, rp, rp, rp, rp, rp, rp, _f32p, _i32p,
                       _f64p]
        fn.restype = i
    L.oracle_filmartin2d.argtypes = [_f32p, i, i, f, C.POINTER(f), C.POINTER(f),
                                     C.POINTER(f), C.POINTER(f), _f32p]
    L.oracle_filmartin2d.restype = i
    L.oracle_filmartin_weights.argtypes = [i, f, f, f, f, f, _opt(_f64p), C.POINTER(i)]
    L.oracle_filmartin_weights.restype = i
    L.oracle_baseline_sample.argtypes = [_f32p, i, i, i, f, i, i, f, _f32p, _i32p, _i32p, i,
                                         _f32p, f, i]
    L.oracle_baseline_sample.restype = d
    L.oracle_set_rho.argtypes = [_opt(_f32p), i, i]
    L.oracle_set_rho.restype = None


def _dt(prec):
    return np.float32 if prec == "f32" else np.float64


def _f(a, dtype):
    return np.asfortranarray(a, dtype=dtype)


# -- Hicks / acquisition -----------------------------------------------------

def kws_tile(ia1: int, ia2: int, nfs: int) -> np.ndarray:
    """21x21 monopole tile, index [i1+10, i2+10] (kwsinc.f90:262-368)."""
    t = np.zeros((21, 21), np.float32, order="F")
    lib().oracle_kws_tile(ia1, ia2, nfs, t)
    return t


def kws_table1d() -> np.ndarray:
    t = np.zeros((21, 100), np.float32, order="F")
    lib().oracle_kws_table1d(t)
    return t


def bessi0(x: float) -> float:
    return float(lib().oracle_bessi0(x))


def subsourcekws(z: float, x: float, dz: float, ifs: int) -> np.ndarray:
    out = np.zeros(5, np.int32)
    lib().oracle_subsourcekws(z, x, dz, ifs, out)
    return out


def acqui_table(pos, h: float, npml: int, ofs: int) -> np.ndarray:
    """(n,5) table as subacqui builds it (subacqui.f90:30-58)."""
    pos = np.asarray(pos, np.float32).reshape(-1, 2)
    tab = np.zeros((len(pos), 5), np.int32, order="F")
    for k, (z, x) in enumerate(pos):
        t = subsourcekws(float(z), float(x), h, ofs)
        tab[k] = [t[0] + npml, t[1] + npml, t[2], t[3], t[4] if ofs != 0 else 0]
    return tab


def sponges(npml: int, n: int):
    a, a1, b, b1 = (np.zeros(n + 2 * npml, np.float32) for _ in range(4))
    lib().oracle_sponges(npml, n, a, a1, b, b1)
    return a, a1, b, b1


@contextlib.contextmanager
def density(rho):
    """Runs the enclosed oracle calls of this thread with density rho (then
    back to 1)."""
    set_rho(rho)
    try:
        yield
    finally:
        set_rho(None)


def set_rho(rho=None):
    """Density (n1, n2) of the media that later calls of this thread build
    (None = 1, the reference's)."""
    if rho is None:
        lib().oracle_set_rho(None, 0, 0)
    else:
        r = _f(rho, np.float32)
        lib().oracle_set_rho(r, r.shape[0], r.shape[1])


# -- simulations -------------------------------------------------------------

def submodeling(vp, npml, h, ofs, nt, dt, s, is5, ir, type_src=0, type_rec=0,
                prec="f32", want_wavefield=False):
    """Forward modelling (submodeling2.f90:11-288). Returns (sis, wavefield|None)."""
    T = _dt(prec)
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    nr = ir.shape[0]
    sis = np.zeros((nt, nr), T, order="F")
    wf = np.zeros((n1, n2, nt), T, order="F") if want_wavefield else None
    getattr(lib(), f"oracle_submodeling_{prec}")(
        vp, n1, n2, npml, h, ofs, nt, dt, _f(s, np.float32), type_src, type_rec,
        _f(is5, np.int32), ir, nr, sis, wf)
    return sis, wf


def esource_data(vp, npml, h, ofs, nt, dt, res, ir, type_rec=0, prec="f32"):
    """G G^T operator (submodeling2.f90:880-1217)."""
    T = _dt(prec)
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    nr = ir.shape[0]
    sis = np.zeros((nt, nr), T, order="F")
    getattr(lib(), f"oracle_esource_data_{prec}")(
        vp, n1, n2, npml, h, ofs, nt, dt, _f(res, T), type_rec, nr, ir, sis)
    return sis


def esource(vp, npml, h, ofs, nt, dt, res, ir, type_rec=0, prec="f32", want_wavefield=True):
    """Final extended-source simulation (submodeling2.f90:523-878).

    Returns (sis, wavefieldp|None, cost)."""
    T = _dt(prec)
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    nr = ir.shape[0]
    sis = np.zeros((nt, nr), T, order="F")
    wf = np.zeros((n1, n2, nt), T, order="F") if want_wavefield else None
    cost = getattr(lib(), f"oracle_esource_{prec}")(
        vp, n1, n2, npml, h, ofs, nt, dt, _f(res, T), type_rec, nr, ir, sis, wf)
    return sis, wf, cost


def resample(npml, wavefield, ir, prec="f32"):
    """subwavefieldresample (subwavefieldresample.f90:1-41)."""
    T = _dt(prec)
    wf = _f(wavefield, T)
    n1, n2, nt = wf.shape
    ir = _f(ir, np.int32)
    nr = ir.shape[0]
    sis = np.zeros((nt, nr), T, order="F")
    getattr(lib(), f"oracle_resample_{prec}")(n1, n2, npml, nt, ir, nr, wf, sis)
    return sis


def linear_minres(vp, npml, h, ofs, nt, dt, ir, deltadr, mu, itnlim, rtol, type_rec=0,
                  prec="f32", log_capacity=1000):
    """sublinearminres + MINRES (sublinearminres.f90:7-86). Returns (deltade, info)."""
    T = _dt(prec)
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    nr = ir.shape[0]
    out = np.zeros((nt, nr), T, order="F")
    istat = np.zeros(3, np.int32)
    scal = np.zeros(6, np.float64)
    rows = np.zeros((5, log_capacity), np.float64, order="F")
    getattr(lib(), f"oracle_minres_{prec}")(
        vp, n1, n2, npml, h, ofs, nt, dt, type_rec, nr, ir, _f(deltadr, T), mu, itnlim, rtol,
        out, istat, scal, rows, log_capacity)
    info = dict(istop=int(istat[0]), itn=int(istat[1]), anorm=scal[0], acond=scal[1],
                rnorm=scal[2], arnorm=scal[3], ynorm=scal[4], shift=scal[5],
                log=rows[:, : istat[2]].T.copy())
    return out, info


def filmartin2d(data, dt, flow, fhig, llow, lhig):
    """Band-pass filter (minresModule.f90:486-614). Returns (out, (flow,fhig,llow,lhig))."""
    d = _f(data, np.float32)
    nt, nr = d.shape
    out = np.zeros_like(d, order="F")
    a, b, c, e = C.c_float(flow), C.c_float(fhig), C.c_float(llow), C.c_float(lhig)
    rc = lib().oracle_filmartin2d(d, nr, nt, dt, C.byref(a), C.byref(b), C.byref(c),
                                  C.byref(e), out)
    if rc != 0:
        raise ValueError("filmartin2d: nt exceeds 65536")
    return out, (a.value, b.value, c.value, e.value)


def filmartin_weights(nt, dt, flow, fhig, llow, lhig):
    nto = C.c_int(0)
    lib().oracle_filmartin_weights(nt, dt, flow, fhig, llow, lhig, None, C.byref(nto))
    w = np.zeros(nto.value + 1, np.float64)
    lib().oracle_filmartin_weights(nt, dt, flow, fhig, llow, lhig, w, C.byref(nto))
    return w


def daw_shot(vp, npml, h, ofs, nt, dt, s, is5, ir, dobs, mu, itnlim, rtol, ird,
             band, type_src=0, type_rec=0, prec="f64"):
    """Mode 1 + mode 2 for one shot (sub_redatum_DAW.f90:82-145, :238-240)."""
    T = _dt(prec)
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    ird = _f(ird, np.int32)
    nr, nd = ir.shape[0], ird.shape[0]
    outs = {k: np.zeros((nt, nr), T, order="F")
            for k in ("datar", "deltadr", "deltade", "dataesc", "datae")}
    raw = np.zeros((nt, nd), T, order="F")
    red = np.zeros((nt, nd), np.float32, order="F")
    istat = np.zeros(3, np.int32)
    scal = np.zeros(6, np.float64)
    flow, fhig, llow, lhig = band
    rc = getattr(lib(), f"oracle_daw_shot_{prec}")(
        vp, n1, n2, npml, h, ofs, nt, dt, _f(s, np.float32), type_src, type_rec,
        _f(is5, np.int32), ir, nr, _f(dobs, np.float32), mu, itnlim, rtol, ird, nd,
        flow, fhig, llow, lhig, outs["datar"], outs["deltadr"], outs["deltade"],
        outs["dataesc"], outs["datae"], raw, red, istat, scal)
    if rc != 0:
        raise ValueError("oracle daw_shot failed")
    outs["redatumed_raw"] = raw
    outs["redatumed"] = red
    outs["minres"] = dict(istop=int(istat[0]), itn=int(istat[1]), shift=scal[5])
    return outs


def baseline_sample(vp, npml, h, ofs, nt, dt, s, is5, ir, dobs, mu, iters):
    """Timed CPU-baseline unit: one truncated FP32 mode-1 shot; returns point updates."""
    vp = _f(vp, np.float32)
    n1, n2 = vp.shape
    ir = _f(ir, np.int32)
    return float(lib().oracle_baseline_sample(
        vp, n1, n2, npml, h, ofs, nt, dt, _f(s, np.float32), _f(is5, np.int32), ir,
        ir.shape[0], _f(dobs, np.float32), mu, iters))
