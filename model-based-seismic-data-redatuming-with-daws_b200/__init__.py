"""daw_b200 -- Python host mirror of the B200 DAW redatuming library.

The compute path is libdaw_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/daw_b200.h); this module only binds it with ctypes and keeps the
reference's routine names and argument meanings
(guogs93/Model-based-seismic-data-redatuming-with-DAWs):

    submodeling                        src/submodeling2.f90:11
    submodeling_adjoint_esource_data   src/submodeling2.f90:880
    submodeling_adjoint_esource        src/submodeling2.f90:523
    sublinearminres                    src/sublinearminres.f90:7
    subwavefieldresample               src/subwavefieldresample.f90:1
    filmartin2d                        src/minresModule.f90:486
    kwsinc2d / subsourcekws / subacqui src/kwsinc.f90, src/subacqui.f90

Arrays use the reference's Fortran layout (numpy order="F"): data (nt, nr),
wavefields (n1, n2, nt), models (n1, n2), acquisition tables (n, 5) int32
with 1-based extended-grid indices.

There is no CPU fallback: loading fails if the library is missing and
``Handle()`` raises if no sm_100 GPU is usable.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdaw_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "daw_b200.h")

DAW_OK = 0
STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_OOM", -3: "ERR_CUDA", -4: "ERR_TIMEOUT",
          -5: "ERR_NAN", -6: "ERR_IO", -7: "ERR_STATE", -8: "ERR_NODEV"}
OPT = {"preset": 0, "history": 1, "scalars": 2, "fused": 3, "graph": 4, "skip_dead_op": 5,
       "max_batch": 6, "chunk": 7, "checkpoint": 8, "step": 9, "tile_cols": 10,
       "ctas_per_sm": 11, "pdl": 12}


class DawError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class MinresInfo(C.Structure):
    _fields_ = [("istop", C.c_int32), ("itn", C.c_int32), ("nlog", C.c_int32),
                ("log_capacity", C.c_int32), ("anorm", C.c_double), ("acond", C.c_double),
                ("rnorm", C.c_double), ("arnorm", C.c_double), ("ynorm", C.c_double),
                ("shift", C.c_double), ("beta1", C.c_double), ("log", C.POINTER(C.c_double))]


class ShotDesc(C.Structure):
    _fields_ = [("shot", C.c_int32), ("nt", C.c_int32), ("s", C.POINTER(C.c_float)),
                ("src_tab", C.c_int32 * 5), ("rec_tab", C.POINTER(C.c_int32)),
                ("nrec", C.c_int32), ("dobs", C.POINTER(C.c_float)), ("type_src", C.c_int32),
                ("type_rec", C.c_int32), ("mu", C.c_float), ("maxiter", C.c_int32),
                ("rtol", C.c_float), ("band", C.c_float * 4)]


class ShotOut(C.Structure):
    _fields_ = [("datar", C.POINTER(C.c_float)), ("deltadr", C.POINTER(C.c_float)),
                ("deltade", C.POINTER(C.c_float)), ("dataesc", C.POINTER(C.c_float)),
                ("datae", C.POINTER(C.c_float)), ("redatumed_raw", C.POINTER(C.c_float)),
                ("redatumed", C.POINTER(C.c_float)), ("wavefield_exd", C.POINTER(C.c_float)),
                ("cost", C.c_double), ("minres", MinresInfo)]


class Timing(C.Structure):
    _fields_ = [("forward_ms", C.c_double), ("operator_ms", C.c_double),
                ("minres_vec_ms", C.c_double), ("esource_ms", C.c_double),
                ("filter_ms", C.c_double), ("total_ms", C.c_double),
                ("sim_fwd_ms", C.c_double), ("sim_a_ms", C.c_double), ("sim_b_ms", C.c_double),
                ("steps_fwd", C.c_double), ("steps_a", C.c_double), ("steps_b", C.c_double),
                ("shot_steps", C.c_double), ("point_updates", C.c_double), ("hist_bytes", C.c_double),
                ("kernel_launches", C.c_int64), ("shot_steps_fwd", C.c_double),
                ("shot_steps_a", C.c_double), ("shot_steps_b", C.c_double),
                ("kernel_family", C.c_int32 * 4), ("tile_cols", C.c_int32 * 4),
                ("ctas_per_sm", C.c_int32 * 4), ("ctas_per_sm_v", C.c_int32 * 4),
                ("shots_per_launch", C.c_int32 * 4)]


_lib = None


def lib():
    """Load libdaw_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run build.py (no CPU fallback exists)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    vp, i32, f32, f64 = C.c_void_p, C.c_int32, C.c_float, C.c_double
    fp, ip, dp = C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_double)
    L.daw_create.argtypes = [C.POINTER(vp), i32]
    L.daw_destroy.argtypes = [vp]
    L.daw_destroy.restype = None
    L.daw_last_error.argtypes = [vp]
    L.daw_last_error.restype = C.c_char_p
    L.daw_set_option.argtypes = [vp, i32, f64]
    L.daw_get_option.argtypes = [vp, i32, dp]
    L.daw_set_model.argtypes = [vp, fp, i32, i32, i32, f32, f32, i32]
    L.daw_set_model_rho.argtypes = [vp, fp, fp, i32, i32, i32, f32, f32, i32]
    L.daw_set_datum.argtypes = [vp, ip, i32]
    L.daw_submodeling.argtypes = [vp, fp, i32, ip, i32, i32, ip, i32, fp, fp]
    L.daw_esource_data.argtypes = [vp, fp, i32, i32, ip, i32, fp]
    L.daw_esource.argtypes = [vp, fp, i32, i32, ip, i32, fp, fp, dp]
    L.daw_linear_minres.argtypes = [vp, fp, i32, i32, ip, i32, f32, i32, f32, fp,
                                    C.POINTER(MinresInfo)]
    L.daw_wavefield_resample.argtypes = [vp, fp, i32, ip, i32, fp]
    L.daw_filmartin2d.argtypes = [vp, fp, i32, i32, f32, fp, fp, fp, fp, fp]
    L.daw_filmartin2d_noalloc.argtypes = [vp, i32, i32, f32, fp, fp, fp, fp, vp, vp,
                                          C.c_char_p, i32]
    L.daw_shot.argtypes = [vp, C.POINTER(ShotDesc), C.POINTER(ShotOut)]
    L.daw_shots.argtypes = [vp, i32, C.POINTER(ShotDesc), C.POINTER(ShotOut)]
    L.daw_submodeling_shots.argtypes = [vp, i32, C.POINTER(ShotDesc), C.POINTER(fp)]
    L.daw_stage_shots.argtypes = [vp, i32, C.POINTER(ShotDesc)]
    L.daw_admit_shots.argtypes = [vp, i32, C.POINTER(ShotDesc), ip, ip]
    L.daw_run_staged.argtypes = [vp, fp]
    L.daw_fetch_shots.argtypes = [vp, C.POINTER(ShotOut)]
    L.daw_run_parfile.argtypes = [vp, C.c_char_p, i32, i32]
    L.daw_get_timing.argtypes = [vp, C.POINTER(Timing)]
    L.daw_reset_timing.argtypes = [vp]
    L.daw_reset_timing.restype = None
    L.daw_version.restype = C.c_char_p
    L.daw_selftest_wait_timeout.argtypes = [vp]
    L.daw_hicks_tile.argtypes = [i32, i32, i32, fp]
    L.daw_hicks_tile.restype = None
    L.daw_hicks_locate.argtypes = [f32, f32, f32, i32, ip]
    L.daw_hicks_locate.restype = None


def header_symbols(path: str = HEADER) -> list[str]:
    """Function names declared in include/daw_b200.h."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(daw_[a-z0-9_]+)\s*\(", txt)))


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def _f32(a):
    return np.asfortranarray(a, dtype=np.float32)


def _i32(a):
    return np.asfortranarray(a, dtype=np.int32)


# -- Hicks / acquisition (host side, same values the library uses) -----------

def kws_tile(ialpha1: int, ialpha2: int, nalpha_frees: int) -> np.ndarray:
    """21x21 monopole tile [i1+10, i2+10] (kwsinc2d, src/kwsinc.f90:212-378)."""
    t = np.zeros((21, 21), np.float32, order="F")
    lib().daw_hicks_tile(ialpha1, ialpha2, nalpha_frees, _p(t, C.c_float))
    return t


def subsourcekws(z: float, x: float, h: float, ofs: int) -> np.ndarray:
    """(ix1, ix2, ialpha1, ialpha2, nalpha_frees) of a position (src/kwsinc.f90:582)."""
    out = np.zeros(5, np.int32)
    lib().daw_hicks_locate(z, x, h, ofs, _p(out, C.c_int32))
    return out


def subacqui(positions, h: float, npml: int, ofs: int) -> np.ndarray:
    """(n,5) table as subacqui builds it from (z, x) positions (src/subacqui.f90:30-58)."""
    pos = np.asarray(positions, np.float32).reshape(-1, 2)
    tab = np.zeros((len(pos), 5), np.int32, order="F")
    for k, (z, x) in enumerate(pos):
        t = subsourcekws(float(z), float(x), h, ofs)
        tab[k] = [t[0] + npml, t[1] + npml, t[2], t[3], t[4] if ofs else 0]
    return tab


# -- handle ------------------------------------------------------------------

class Handle:
    """One GPU, one model; mirrors the reference's per-rank state."""

    def __init__(self, device: int = 0, preset: str = "mixed", **options):
        self._h = C.c_void_p()
        rc = lib().daw_create(C.byref(self._h), device)
        if rc != DAW_OK:
            raise DawError(rc, "daw_create failed (no usable sm_100 GPU)")
        self.set_options(preset=0 if preset == "plain" else 1)
        if options:
            self.set_options(**options)
        self.grid = None

    def close(self):
        if self._h:
            lib().daw_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != DAW_OK:
            raise DawError(rc, lib().daw_last_error(self._h).decode())

    def set_options(self, **kw):
        for k, v in kw.items():
            self._ck(lib().daw_set_option(self._h, OPT[k], float(v)))

    def get_option(self, key):
        v = C.c_double()
        self._ck(lib().daw_get_option(self._h, OPT[key], C.byref(v)))
        return v.value

    def set_model(self, vp, npml: int, h: float, dt: float, ofs: int, rho=None):
        """Velocity vp (n1, n2) and, optionally, density rho of the same shape
        (None = rho 1, the reference's)."""
        vp = _f32(vp)
        n1, n2 = vp.shape
        if rho is None:
            self._ck(lib().daw_set_model(self._h, _p(vp, C.c_float), n1, n2, npml, h, dt, ofs))
        else:
            rho = _f32(rho)
            if rho.shape != vp.shape:
                raise ValueError("rho must have the shape of vp")
            self._ck(lib().daw_set_model_rho(self._h, _p(vp, C.c_float), _p(rho, C.c_float),
                                             n1, n2, npml, h, dt, ofs))
        self.grid = dict(n1=n1, n2=n2, npml=npml, h=h, dt=dt, ofs=ofs, rho=rho is not None)

    def set_datum(self, tab):
        tab = _i32(tab)
        self._ck(lib().daw_set_datum(self._h, _p(tab, C.c_int32), tab.shape[0]))
        self.grid["ndatum"] = tab.shape[0]

    # -- reference routines ---------------------------------------------------
    def submodeling(self, s, is5, ir, type_src=0, type_rec=0, wavefield=False):
        s = _f32(s)
        nt = s.shape[0]
        ir = _i32(ir)
        nr = ir.shape[0]
        sis = np.zeros((nt, nr), np.float32, order="F")
        g = self.grid
        wf = np.zeros((g["n1"], g["n2"], nt), np.float32, order="F") if wavefield else None
        self._ck(lib().daw_submodeling(self._h, _p(s, C.c_float), nt, _p(_i32(is5), C.c_int32),
                                       type_src, type_rec, _p(ir, C.c_int32), nr,
                                       _p(sis, C.c_float), _p(wf, C.c_float)))
        return sis, wf

    def submodeling_shots(self, shots):
        """Batched forward modelling (mode 0): `shots` are dicts with s, src,
        rec and optionally nt, type_src, type_rec; returns each shot's
        (nt, nrec) receiver data."""
        n = len(shots)
        descs = (ShotDesc * n)()
        outs = (C.POINTER(C.c_float) * n)()
        keep, results = [], []
        for i, sh in enumerate(shots):
            s = _f32(sh["s"])
            rec = _i32(sh["rec"])
            nt = int(sh.get("nt", s.shape[0]))
            sis = np.zeros((nt, rec.shape[0]), np.float32, order="F")
            keep += [s, rec]
            results.append(sis)
            d = descs[i]
            d.shot = int(sh.get("shot", i + 1))
            d.nt = nt
            d.s = _p(s, C.c_float)
            for k in range(5):
                d.src_tab[k] = int(sh["src"][k])
            d.rec_tab = _p(rec, C.c_int32)
            d.nrec = rec.shape[0]
            d.type_src = int(sh.get("type_src", 0))
            d.type_rec = int(sh.get("type_rec", 0))
            outs[i] = _p(sis, C.c_float)
        self._ck(lib().daw_submodeling_shots(self._h, n, descs, outs))
        return results

    def submodeling_adjoint_esource_data(self, res, ir, type_rec=0):
        res = _f32(res)
        nt, nr = res.shape
        ir = _i32(ir)
        sis = np.zeros((nt, nr), np.float32, order="F")
        self._ck(lib().daw_esource_data(self._h, _p(res, C.c_float), nt, type_rec,
                                        _p(ir, C.c_int32), nr, _p(sis, C.c_float)))
        return sis

    def submodeling_adjoint_esource(self, res, ir, type_rec=0, wavefield=True):
        res = _f32(res)
        nt, nr = res.shape
        ir = _i32(ir)
        sis = np.zeros((nt, nr), np.float32, order="F")
        g = self.grid
        wf = np.zeros((g["n1"], g["n2"], nt), np.float32, order="F") if wavefield else None
        cost = C.c_double()
        self._ck(lib().daw_esource(self._h, _p(res, C.c_float), nt, type_rec, _p(ir, C.c_int32),
                                   nr, _p(sis, C.c_float), _p(wf, C.c_float), C.byref(cost)))
        return sis, wf, cost.value

    def sublinearminres(self, deltadr, ir, mu, maxiter, rtol, type_rec=0):
        d = _f32(deltadr)
        nt, nr = d.shape
        ir = _i32(ir)
        out = np.zeros((nt, nr), np.float32, order="F")
        logbuf = np.zeros((max(1, maxiter), 5), np.float64)
        info = MinresInfo()
        info.log = _p(logbuf, C.c_double)
        info.log_capacity = logbuf.shape[0]
        self._ck(lib().daw_linear_minres(self._h, _p(d, C.c_float), nt, type_rec,
                                         _p(ir, C.c_int32), nr, mu, maxiter, rtol,
                                         _p(out, C.c_float), C.byref(info)))
        return out, _info(info, logbuf)

    def subwavefieldresample(self, wavefield, ir):
        wf = _f32(wavefield)
        nt = wf.shape[2]
        ir = _i32(ir)
        sis = np.zeros((nt, ir.shape[0]), np.float32, order="F")
        self._ck(lib().daw_wavefield_resample(self._h, _p(wf, C.c_float), nt, _p(ir, C.c_int32),
                                              ir.shape[0], _p(sis, C.c_float)))
        return sis

    def filmartin2d(self, data, dt, flow, fhig, llow, lhig):
        d = _f32(data)
        nt, nr = d.shape
        out = np.zeros_like(d, order="F")
        band = [C.c_float(flow), C.c_float(fhig), C.c_float(llow), C.c_float(lhig)]
        self._ck(lib().daw_filmartin2d(self._h, _p(d, C.c_float), nr, nt, dt,
                                       *[C.byref(b) for b in band], _p(out, C.c_float)))
        return out, tuple(b.value for b in band)

    # -- pipeline ---------------------------------------------------------------
    def shots(self, shots, outputs=("datar", "deltadr", "deltade", "dataesc", "datae",
                                    "redatumed_raw", "redatumed"), wavefield=False):
        """Run mode-1 DAW shots (batched).  Each item of ``shots`` is a dict with
        keys s, nt, src (5,), rec (n,5), dobs (nt,n), mu, maxiter, rtol, band and
        optionally shot, type_src, type_rec.  Returns one dict of arrays per shot."""
        descs, outs, keep, results = _pack(shots, outputs, wavefield, self.grid)
        n = len(shots)
        self._ck(lib().daw_shots(self._h, n, descs, outs))
        for i in range(n):
            results[i]["minres"] = _info(outs[i].minres, results[i].pop("_log"))
            results[i]["cost"] = outs[i].cost
        del keep
        return results

    def shot(self, **shot):
        return self.shots([shot])[0]

    def admit_shots(self, shots):
        """(count, window): how many of `shots`, in order, HBM admits as one
        batch, and the history window a lone shot would use."""
        descs, _, keep, _ = _pack(shots, (), False, self.grid)
        cnt, win = C.c_int32(), C.c_int32()
        self._ck(lib().daw_admit_shots(self._h, len(shots), descs, C.byref(cnt), C.byref(win)))
        del keep
        return cnt.value, win.value

    def stage_shots(self, shots):
        descs, _, keep, _ = _pack(shots, (), False, self.grid)
        self._staged_keep = keep
        self._staged_n = len(shots)
        self._staged_shapes = [(int(sh["nt"]), np.asarray(sh["rec"]).shape[0]) for sh in shots]
        self._ck(lib().daw_stage_shots(self._h, len(shots), descs))

    def run_staged(self) -> float:
        ms = C.c_float()
        self._ck(lib().daw_run_staged(self._h, C.byref(ms)))
        return ms.value

    def fetch_staged(self, outputs=("deltade", "redatumed")):
        shots = [dict(nt=nt, rec=np.zeros((nr, 5), np.int32)) for nt, nr in self._staged_shapes]
        _, outs, keep, results = _pack_outputs(shots, outputs, False, self.grid)
        self._ck(lib().daw_fetch_shots(self._h, outs))
        for i in range(len(shots)):
            results[i]["minres"] = _info(outs[i].minres, results[i].pop("_log"))
        del keep
        return results

    def run_parfile(self, workdir: str, first: int = 0, last: int = 0):
        self._ck(lib().daw_run_parfile(self._h, workdir.encode(), first, last))

    def timing(self) -> dict:
        t = Timing()
        self._ck(lib().daw_get_timing(self._h, C.byref(t)))
        out = {}
        for k, _ in Timing._fields_:
            v = getattr(t, k)
            out[k] = list(v) if isinstance(v, C.Array) else v
        return out

    def reset_timing(self):
        lib().daw_reset_timing(self._h)


def _info(info, logbuf):
    n = int(info.nlog)
    return dict(istop=int(info.istop), itn=int(info.itn), anorm=info.anorm, acond=info.acond,
                rnorm=info.rnorm, arnorm=info.arnorm, ynorm=info.ynorm, shift=info.shift,
                beta1=info.beta1, log=np.array(logbuf[:n]) if logbuf is not None else None)


def _pack_outputs(shots, outputs, wavefield, grid):
    n = len(shots)
    outs = (ShotOut * n)()
    keep, results = [], []
    for i, sh in enumerate(shots):
        nt = int(sh["nt"])
        nr = np.asarray(sh["rec"]).shape[0]
        res = {}
        for name in outputs:
            if name.startswith("redatumed"):
                nd = sh.get("ndatum", grid.get("ndatum", 0) if grid else 0)
                if not nd:
                    continue
                arr = np.zeros((nt, nd), np.float32, order="F")
            else:
                arr = np.zeros((nt, nr), np.float32, order="F")
            setattr(outs[i], name, _p(arr, C.c_float))
            res[name] = arr
            keep.append(arr)
        if wavefield:
            wf = np.zeros((grid["n1"], grid["n2"], nt), np.float32, order="F")
            outs[i].wavefield_exd = _p(wf, C.c_float)
            res["wavefield_exd"] = wf
            keep.append(wf)
        lg = np.zeros((max(1, int(sh.get("maxiter", 1))), 5), np.float64)
        outs[i].minres.log = _p(lg, C.c_double)
        outs[i].minres.log_capacity = lg.shape[0]
        res["_log"] = lg
        keep.append(lg)
        results.append(res)
    return None, outs, keep, results


def _pack(shots, outputs, wavefield, grid):
    n = len(shots)
    descs = (ShotDesc * n)()
    _, outs, keep, results = _pack_outputs(shots, outputs, wavefield, grid)
    for i, sh in enumerate(shots):
        s = _f32(sh["s"])
        rec = _i32(sh["rec"])
        dobs = _f32(sh["dobs"])
        keep += [s, rec, dobs]
        d = descs[i]
        d.shot = int(sh.get("shot", i + 1))
        d.nt = int(sh["nt"])
        d.s = _p(s, C.c_float)
        for k in range(5):
            d.src_tab[k] = int(sh["src"][k])
        d.rec_tab = _p(rec, C.c_int32)
        d.nrec = rec.shape[0]
        d.dobs = _p(dobs, C.c_float)
        d.type_src = int(sh.get("type_src", 0))
        d.type_rec = int(sh.get("type_rec", 0))
        d.mu = float(sh["mu"])
        d.maxiter = int(sh["maxiter"])
        d.rtol = float(sh.get("rtol", 0.0))
        for k in range(4):
            d.band[k] = float(sh["band"][k])
    return descs, outs, keep, results


def version() -> str:
    return lib().daw_version().decode()
