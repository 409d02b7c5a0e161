"""GPU parity on grids whose tiles include interior tiles.

The TMA kernels compile their stencil pass twice.  A tile that touches no grid
edge, PML frame row or column, free-surface row or physical-interior boundary
takes the second version, in which every boundary predicate is a constant and
the sponge multiplies are dropped (the factors there are exactly 1).  The small
parity grids of test_gpu_parity.py have no such tile; the two grids here do:

- the 151 x 461 single-shot configuration (h = 20 m, npml 20, nt 2000, 230
  receivers, datum at 1000 m, 10 MINRES iterations): one tile row of interior
  tiles, through which the waves of every stage pass;
- the 751 x 2301 grid of the benchmark (npml 40, 576 receivers, datum at
  1200 m) at a reduced record length: about 80 % of its tiles are interior.

Bars, as in test_gpu_parity.py: the FP32 paths equal the FP32 oracle bit for
bit in every simulation (forward, G G^T, final esource); whole shots of the
FP32 paths are within 1e-4 of the FP32 oracle; the FP16-history mixed path is
within 1e-3 (rel. L2) of the FP64 oracle, and its measured errors are printed.
The oracle's long runs start in background threads when the module starts
(ctypes releases the GIL), so they overlap the GPU runs.
"""
import concurrent.futures as cf

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4
MIXED_TOL = 1e-3
TR, TC = 64, 32  # tile of the TMA kernels (rows x columns)


def interior_tiles(n1, n2, npml, ofs, mode):
    """Tiles for which the TMA kernels take their interior stencil pass: the
    tile lies inside the rows and columns that every stencil loop updates,
    inside the physical region and below the free-surface rows (mode 0 =
    forward, 1 = stage A, 2 = stage B; the final esource narrows the source
    range by one point on each side)."""
    n1e, n2e = n1 + 2 * npml, n2 + 2 * npml
    off = 2 if mode == 0 else 3
    slo, shi1, shi2 = (1, n1 - 1, n2 - 1) if mode == 3 else (0, n1, n2)
    fsrows = npml + 1 if ofs == 1 else 0
    rlo, rhi = max(2, npml + slo, fsrows), min(n1e - off, npml + shi1, n1e)
    clo, chi = max(2, npml + slo), min(n2e - off, npml + shi2, n2e)
    return sum(1 for r0 in range(0, n1e, TR) for c0 in range(0, n2e, TC)
               if r0 >= rlo and r0 + TR <= rhi and c0 >= clo and c0 + TC <= chi)


def _acq(pkg, w):
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    ird = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
    return src, rec, ird


@pytest.fixture(scope="module")
def pool():
    ex = cf.ThreadPoolExecutor(max_workers=6)
    yield ex
    ex.shutdown(wait=True)


# -- the 151 x 461 configuration -------------------------------------------------

@pytest.fixture(scope="module")
def c1(pkg, O, pool):
    from daw_b200 import synthetic
    w = synthetic.config1()
    src, rec, ird = _acq(pkg, w)
    s = w.wavelet()
    dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, w.nt, w.dt, s, src, rec)
    res = np.asfortranarray(dobs[::-1])
    args = (w.c0, w.npml, w.h, w.ofs, w.nt, w.dt)
    fut = {
        "fwd": pool.submit(O.submodeling, *args, s, src, rec, want_wavefield=True),
        "ggt": pool.submit(O.esource_data, *args, res, rec),
        "es": pool.submit(O.esource, *args, res, rec),
        "shot32": pool.submit(O.daw_shot, *args, s, src, rec, dobs, w.mu, w.maxiter, 0.0, ird,
                              w.band, prec="f32"),
        "shot64": pool.submit(O.daw_shot, *args, s, src, rec, dobs, w.mu, w.maxiter, 0.0, ird,
                              w.band, prec="f64"),
    }
    return dict(w=w, src=src, rec=rec, ird=ird, s=s, dobs=dobs, res=res, fut=fut)


def _handle(pkg, w, preset, **opt):
    h = pkg.Handle(0, preset=preset, **opt)
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
    return h


PATHS = [("plain", {}), ("mixed", {"history": 0}), ("mixed", {"history": 0, "graph": 0}),
         ("mixed", {"history": 0, "step": 1, "tile_cols": 16}),
         ("mixed", {"history": 0, "step": 1, "tile_cols": 32}),
         ("mixed", {"history": 0, "step": 0}), ("mixed", {"history": 0, "pdl": 1}),
         ("mixed", {"history": 0, "chunk": 1}), ("mixed", {"history": 0, "chunk": 2}),
         ("mixed", {"history": 0, "chunk": 4})]


def test_config1_has_interior_tiles():
    for mode in range(4):
        assert interior_tiles(151, 461, 20, 1, mode) >= 10, mode
    # the small parity grids have none
    assert interior_tiles(60, 90, 12, 1, 0) == 0


@pytest.mark.parametrize("preset,opt", PATHS)
def test_config1_forward_bitexact(pkg, c1, preset, opt):
    w = c1["w"]
    ref, refwf = c1["fut"]["fwd"].result()
    with _handle(pkg, w, preset, **opt) as h:
        sis, wf = h.submodeling(c1["s"], c1["src"], c1["rec"], wavefield=True)
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)


@pytest.mark.parametrize("preset,opt", PATHS)
def test_config1_ggt_bitexact(pkg, c1, preset, opt):
    w = c1["w"]
    ref = c1["fut"]["ggt"].result()
    with _handle(pkg, w, preset, **opt) as h:
        g = h.submodeling_adjoint_esource_data(c1["res"], c1["rec"])
    assert np.array_equal(g, ref)


@pytest.mark.parametrize("preset,opt", PATHS[:3])
def test_config1_esource_bitexact(pkg, c1, preset, opt):
    w = c1["w"]
    ref, refwf, _ = c1["fut"]["es"].result()
    with _handle(pkg, w, preset, **opt) as h:
        sis, wf, _ = h.submodeling_adjoint_esource(c1["res"], c1["rec"])
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)


def _shot_kw(c, w):
    return dict(s=c["s"], nt=w.nt, src=c["src"], rec=c["rec"], dobs=c["dobs"], mu=w.mu,
                maxiter=w.maxiter, rtol=0.0, band=w.band)


KEYS = ("deltade", "dataesc", "datae", "redatumed_raw", "redatumed")


@pytest.mark.parametrize("preset,opt", [("plain", {}), ("mixed", {"history": 0})])
def test_config1_fp32_shot(pkg, c1, preset, opt):
    w = c1["w"]
    with _handle(pkg, w, preset, **opt) as h:
        h.set_datum(c1["ird"])
        out = h.shot(**_shot_kw(c1, w))
    ref = c1["fut"]["shot32"].result()
    assert np.array_equal(out["datar"], ref["datar"])
    assert np.array_equal(out["deltadr"], ref["deltadr"])
    for k in KEYS:
        err = rel_l2(out[k], ref[k])
        assert err <= FP32_TOL, (k, err)
    assert out["minres"]["itn"] == w.maxiter


def test_config1_mixed_shot_vs_fp64(pkg, c1):
    """The benchmark's precision (FP16 histories, FP32 stencils, FP64 MINRES
    scalars) over a whole 151 x 461 shot, 2000 steps and 10 iterations,
    against the FP64 oracle; the errors are printed."""
    w = c1["w"]
    with _handle(pkg, w, "mixed") as h:
        h.set_datum(c1["ird"])
        out = h.shot(**_shot_kw(c1, w))
    ref = c1["fut"]["shot64"].result()
    errs = {k: rel_l2(out[k], ref[k]) for k in ("datar",) + KEYS}
    print("\n151x461 mixed vs FP64 oracle, rel. L2:",
          " ".join(f"{k}={v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= MIXED_TOL, (k, v)


# -- the 751 x 2301 grid at a reduced record length ------------------------------

NT2 = 200


@pytest.fixture(scope="module")
def c2(pkg, O, pool):
    from daw_b200 import synthetic
    w = synthetic.config2(nshot=1, nt=NT2)
    src, rec, ird = _acq(pkg, w)
    # the Ricker peak moved to step 60 so the wave travels within 200 steps
    s = w.wavelet(NT2 + 140)[140:].copy()
    args = (w.c0, w.npml, w.h, w.ofs, NT2, w.dt)
    dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, NT2, w.dt, s, src, rec)
    res = np.asfortranarray(dobs[::-1])
    fut = {"fwd": pool.submit(O.submodeling, *args, s, src, rec),
           "ggt": pool.submit(O.esource_data, *args, res, rec),
           "es": pool.submit(O.esource, *args, res, rec, want_wavefield=False)}
    return dict(w=w, src=src, rec=rec, ird=ird, s=s, dobs=dobs, res=res, fut=fut)


def test_config2_grid_is_mostly_interior():
    total = ((831 + TR - 1) // TR) * ((2381 + TC - 1) // TC)
    for mode in range(4):
        assert interior_tiles(751, 2301, 40, 1, mode) >= 0.75 * total, mode


@pytest.mark.parametrize("preset,opt", [("plain", {}), ("mixed", {"history": 0}),
                                        ("mixed", {"history": 0, "graph": 0}),
                                        ("mixed", {"history": 0, "step": 1, "tile_cols": 16}),
                                        ("mixed", {"history": 0, "pdl": 0})])
def test_config2_grid_forward_and_ggt_bitexact(pkg, c2, preset, opt):
    w = c2["w"]
    with _handle(pkg, w, preset, **opt) as h:
        sis, _ = h.submodeling(c2["s"], c2["src"], c2["rec"])
        g = h.submodeling_adjoint_esource_data(c2["res"], c2["rec"])
        es, _, _ = h.submodeling_adjoint_esource(c2["res"], c2["rec"], wavefield=False)
    assert np.abs(sis).max() > 0
    assert np.array_equal(sis, c2["fut"]["fwd"].result()[0])
    assert np.array_equal(g, c2["fut"]["ggt"].result())
    assert np.array_equal(es, c2["fut"]["es"].result()[0])


def test_config2_grid_shot_tma_equals_plain(pkg, c2):
    """Two MINRES iterations of a whole shot: the TMA kernels with FP32
    histories and FP32 scalars equal the plain port; the FP16-history path
    is within 1e-3 of both."""
    w = c2["w"]
    kw = dict(s=c2["s"], nt=NT2, src=c2["src"], rec=c2["rec"], dobs=c2["dobs"], mu=w.mu,
              maxiter=2, rtol=0.0, band=w.band)
    outs = {}
    for name, preset, opt in [("plain", "plain", {}),
                              ("tma32", "mixed", {"history": 0, "scalars": 0}),
                              ("mixed", "mixed", {})]:
        with _handle(pkg, w, preset, **opt) as h:
            h.set_datum(c2["ird"])
            outs[name] = h.shot(**kw)
    for k in ("datar", "deltadr") + KEYS:
        assert np.array_equal(outs["tma32"][k], outs["plain"][k]), k
    for k in KEYS:
        err = rel_l2(outs["mixed"][k], outs["plain"][k])
        assert err <= MIXED_TOL, (k, err)
