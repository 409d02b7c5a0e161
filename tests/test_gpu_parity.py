"""GPU parity: the CUDA library through its C ABI against the CPU oracle.

Bars (rel. L2 unless stated): the plain FP32 port and the fused path with
FP32 histories reproduce the FP32 oracle's simulations bit for bit (same
operations, same rounding); MINRES and the full shot (parallel reductions)
are within 1e-4 of the FP64 oracle; the mixed path (FP16 histories, FP64
MINRES scalars) within 1e-3 of the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4
MIXED_TOL = 1e-3


@pytest.fixture(scope="module")
def case(pkg, O):
    from daw_b200 import synthetic
    w = synthetic.small()
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    ird = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
    s = w.wavelet()
    dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, w.nt, w.dt, s, src, rec)
    return dict(w=w, src=src, rec=rec, ird=ird, s=s, dobs=dobs)


def handle(pkg, case, preset="plain", **opt):
    w = case["w"]
    h = pkg.Handle(0, preset=preset, **opt)
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
    return h


# "mixed" with FP32 histories: the TMA kernels with the family and launch
# shape autotuned (the default), the split pressure/velocity kernels pinned
# (also with programmatic dependent launch), direct launches instead of
# graphs, the one-kernel-per-step path (both tile widths pinned), and the
# register kernels.
PATHS = [("plain", {}), ("mixed", {"history": 0}), ("mixed", {"history": 0, "graph": 0}),
         ("mixed", {"history": 0, "step": 1, "tile_cols": 16, "ctas_per_sm": 1}),
         ("mixed", {"history": 0, "step": 1, "tile_cols": 32, "ctas_per_sm": 2}),
         ("mixed", {"history": 0, "step": 0}), ("mixed", {"history": 0, "pdl": 1}),
         ("mixed", {"history": 0, "chunk": 1}), ("mixed", {"history": 0, "chunk": 4})]


@pytest.mark.parametrize("preset,opt", PATHS)
def test_forward_bitexact(pkg, O, case, preset, opt):
    w = case["w"]
    ref, refwf = O.submodeling(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["s"], case["src"],
                               case["rec"], want_wavefield=True)
    with handle(pkg, case, preset, **opt) as h:
        sis, wf = h.submodeling(case["s"], case["src"], case["rec"], wavefield=True)
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)


@pytest.mark.parametrize("preset,opt", PATHS)
def test_ggt_bitexact(pkg, O, case, preset, opt):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    ref = O.esource_data(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res, case["rec"])
    with handle(pkg, case, preset, **opt) as h:
        g = h.submodeling_adjoint_esource_data(res, case["rec"])
    assert np.array_equal(g, ref)


@pytest.mark.parametrize("preset,opt", PATHS[:2])
def test_esource_bitexact(pkg, O, case, preset, opt):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    ref, refwf, _ = O.esource(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res, case["rec"])
    with handle(pkg, case, preset, **opt) as h:
        sis, wf, cost = h.submodeling_adjoint_esource(res, case["rec"])
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)
    # `cost` is accumulated in FP64 on the device; the reference's sequential
    # FP32 sum of ~2e6 terms is itself off by ~1e-3, so compare with FP64
    _, _, cost64 = O.esource(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res.astype(np.float64),
                             case["rec"], prec="f64", want_wavefield=False)
    assert abs(cost - cost64) <= 1e-5 * abs(cost64)


def test_ggt_fp16_history(pkg, O, case):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    ref = O.esource_data(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res.astype(np.float64),
                         case["rec"], prec="f64")
    with handle(pkg, case, "mixed") as h:
        g = h.submodeling_adjoint_esource_data(res, case["rec"])
    err = rel_l2(g, ref)
    assert err <= MIXED_TOL, err


def test_ggt_power_of_two_linearity(pkg, case):
    """Size-independent identity: A(2x) == 2 A(x), also with FP16 histories
    (their per-step scales are powers of two).  Exact except for values in
    the FP32 subnormal range (the stencil's exponentially small precursors
    ahead of the wavefront), where doubling is not exact."""
    res = np.asfortranarray(case["dobs"][::-1])
    for preset, opt in (("plain", {}), ("mixed", {})):
        with handle(pkg, case, preset, **opt) as h:
            g1 = h.submodeling_adjoint_esource_data(res, case["rec"])
            g2 = h.submodeling_adjoint_esource_data(2 * res, case["rec"])
        # 1-ulp differences born in the subnormal precursor grow with the
        # wave, so the identity holds to FP32 accuracy, not bit for bit (the
        # FP32 oracle shows the same on this case)
        assert rel_l2(g2, 2 * g1) <= 1e-5, preset


@pytest.mark.parametrize("preset,opt,prec,tol", [
    ("plain", {}, "f32", FP32_TOL), ("mixed", {}, "f64", MIXED_TOL),
    ("mixed", {"history": 0}, "f64", FP32_TOL)])
def test_minres(pkg, O, case, preset, opt, prec, tol):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    T = np.float32 if prec == "f32" else np.float64
    ref, rinfo = O.linear_minres(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["rec"],
                                 res.astype(T), w.mu, w.maxiter, 0.0, prec=prec)
    with handle(pkg, case, preset, **opt) as h:
        x, info = h.sublinearminres(res, case["rec"], w.mu, w.maxiter, 0.0)
    assert info["itn"] == rinfo["itn"] == w.maxiter
    assert info["istop"] == rinfo["istop"] == 5
    assert abs(info["shift"] - rinfo["shift"]) <= 1e-5 * abs(rinfo["shift"])
    err = rel_l2(x, ref)
    assert err <= tol, err
    assert np.allclose(info["log"][:, 2], rinfo["log"][:, 2], rtol=1e-3)


def _shot(case, w):
    return dict(s=case["s"], nt=w.nt, src=case["src"], rec=case["rec"], dobs=case["dobs"],
                mu=w.mu, maxiter=w.maxiter, rtol=0.0, band=w.band)


@pytest.fixture(scope="module")
def oracle_shots(O, case):
    w = case["w"]
    return {p: O.daw_shot(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["s"], case["src"],
                          case["rec"], case["dobs"], w.mu, w.maxiter, 0.0, case["ird"], w.band,
                          prec=p) for p in ("f32", "f64")}


# The FP32 paths are held to the FP32 oracle (the reference computes in REAL):
# forward data and residuals bit for bit, MINRES and after within 1e-4 (its
# inner products are parallel reductions).  The FP16-history path is held to
# the FP64 oracle within 1e-3.  (FP32 against FP64 is limited by cancellation
# in dobs - datar, a property of the reference's own precision.)
@pytest.mark.parametrize("preset,opt,prec,tol", [("plain", {}, "f32", FP32_TOL),
                                                 ("mixed", {}, "f64", MIXED_TOL),
                                                 ("mixed", {"history": 0}, "f32", FP32_TOL)])
def test_shot_pipeline(pkg, case, oracle_shots, preset, opt, prec, tol):
    w = case["w"]
    with handle(pkg, case, preset, **opt) as h:
        h.set_datum(case["ird"])
        out = h.shot(**_shot(case, w))
    ref = oracle_shots[prec]
    if prec == "f32":
        assert np.array_equal(out["datar"], ref["datar"])
        assert np.array_equal(out["deltadr"], ref["deltadr"])
    else:
        assert rel_l2(out["datar"], ref["datar"]) <= 1e-6
    for k in ("deltade", "dataesc", "datae", "redatumed_raw", "redatumed"):
        err = rel_l2(out[k], ref[k])
        assert err <= tol, (k, err)
    assert out["minres"]["itn"] == w.maxiter


def test_batched_uneven_shots(pkg, O, case):
    """Three shots with different record lengths, receiver spreads and source
    positions in one batched launch equal the same shots run one at a time."""
    w = case["w"]
    from daw_b200 import synthetic
    shots = []
    for k, (nt, lo, hi, x) in enumerate([(400, 0, 24, 300.0), (330, 4, 17, 520.0),
                                         (371, 10, 24, 700.0)]):
        src = pkg.subacqui([[15.0, x]], w.h, w.npml, w.ofs)[0]
        rec = case["rec"][lo:hi]
        s = w.wavelet(nt)
        dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, nt, w.dt, s, src, rec)
        shots.append(dict(s=s, nt=nt, src=src, rec=rec, dobs=dobs, mu=w.mu, maxiter=3,
                          rtol=0.0, band=w.band, shot=k + 1))
    with handle(pkg, case, "mixed") as h:
        h.set_datum(case["ird"])
        batched = h.shots(shots)
        single = [h.shots([sh])[0] for sh in shots]
        h.set_options(max_batch=1)
        serial = h.shots(shots)
    for b, s1, s2 in zip(batched, single, serial):
        for key in ("deltade", "dataesc", "redatumed"):
            assert np.array_equal(b[key], s1[key]), key
            assert np.array_equal(b[key], s2[key]), key


def test_filter(pkg, O, case):
    w = case["w"]
    rng = np.random.default_rng(4)
    for nt, dt, band in [(400, 0.002, w.band), (2000, 0.0015, (5.0, 25.0, 5.0, 5.0)),
                         (7500, 0.0004, (7.5, 37.5, 7.5, 7.5)),
                         (20000, 0.0004, (10.0, 50.0, 10.0, 10.0)),
                         (300, 0.004, (5.0, 300.0, 2.0, 30.0))]:  # fhig above Nyquist
        x = np.asfortranarray(rng.standard_normal((nt, 7)).astype(np.float32))
        ref, rband = O.filmartin2d(x, dt, *band)
        with handle(pkg, case) as h:
            y, hband = h.filmartin2d(x, dt, *band)
        assert rel_l2(y, ref) <= 1e-6, (nt, rel_l2(y, ref))
        assert np.allclose(hband, rband)


def test_resample_bitexact(pkg, O, case):
    w = case["w"]
    _, wf = O.submodeling(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["s"], case["src"],
                          case["rec"], want_wavefield=True)
    ref = O.resample(w.npml, wf, case["ird"])
    with handle(pkg, case) as h:
        got = h.subwavefieldresample(wf, case["ird"])
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("preset", ["plain", "mixed"])
def test_edge_stations_and_options(pkg, O, preset):
    """Receivers within 10 points of every edge (support clipped), a source
    above the free surface, ofs=0 and type_src=1 (vz injection)."""
    n1, n2, npml, h, dt, nt = 36, 50, 8, 10.0, 0.001, 120
    rng = np.random.default_rng(9)
    vp = np.asfortranarray((1700 + rng.uniform(-40, 40, (n1, n2))).astype(np.float32))
    s = (np.sin(np.arange(nt) * 0.3) * np.exp(-0.03 * np.arange(nt))).astype(np.float32)
    # z = -4 m lies above the free surface (all ten upper taps mirrored);
    # x = -50 m and x = 540 m put stations in the side sponges
    pos = [[0.0, 0.0], [5.0, 490.0], [350.0, 0.0], [350.0, 490.0], [-4.0, 250.0],
           [170.0, -50.0], [100.0, 540.0], [400.0, 250.0]]
    for ofs in (0, 1):
        rec = O.acqui_table(pos, h, npml, ofs)
        src = O.acqui_table([[2.0, 240.0]], h, npml, ofs)[0]
        for type_src in (0, 1):
            ref, _ = O.submodeling(vp, npml, h, ofs, nt, dt, s, src, rec, type_src=type_src)
            with pkg.Handle(0, preset=preset, history=0) if preset == "mixed" else \
                    pkg.Handle(0, preset="plain") as hd:
                hd.set_model(vp, npml, h, dt, ofs)
                got, _ = hd.submodeling(s, src, rec, type_src=type_src)
            assert np.array_equal(got, ref), (ofs, type_src)
        res = np.asfortranarray(ref[::-1])
        gref = O.esource_data(vp, npml, h, ofs, nt, dt, res, rec)
        with pkg.Handle(0, preset=preset, history=0) if preset == "mixed" else \
                pkg.Handle(0, preset="plain") as hd:
            hd.set_model(vp, npml, h, dt, ofs)
            g = hd.submodeling_adjoint_esource_data(res, rec)
        assert np.array_equal(g, gref), ofs


def test_type_rec_nonzero_gives_zero_data(pkg, case):
    w = case["w"]
    with handle(pkg, case, "mixed") as h:
        sis, _ = h.submodeling(case["s"], case["src"], case["rec"], type_rec=1)
    assert not sis.any()


def test_zero_residual_minres(pkg, case):
    """beta1 = 0: MINRES stops at once with x = 0 (minresModule.f90:94-97)."""
    w = case["w"]
    z = np.zeros((w.nt, case["rec"].shape[0]), np.float32, order="F")
    for preset in ("plain", "mixed"):
        with handle(pkg, case, preset) as h:
            x, info = h.sublinearminres(z, case["rec"], w.mu, 3, 0.0)
        assert not x.any() and info["itn"] == 0 and info["istop"] == 0


def test_errors_are_reported(pkg, case):
    w = case["w"]
    with pkg.Handle(0) as h:
        with pytest.raises(pkg.DawError) as e:
            h.submodeling(case["s"], case["src"], case["rec"])
        assert e.value.code == -7  # no model
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        bad = case["rec"].copy()
        bad[0, 2] = 101  # ialpha out of range
        with pytest.raises(pkg.DawError) as e:
            h.submodeling(case["s"], case["src"], bad)
        assert e.value.code == -1
        with pytest.raises(pkg.DawError):
            h.set_options(preset=3)


@pytest.mark.parametrize("opt", [{}, {"chunk": 2}, {"history": 0}])
def test_non_finite_history_is_reported(pkg, case, opt):
    """A NaN in the residual reaches the stage-A histories; the fused paths
    report DAW_ERR_NAN from their max-|x| reduction, and the handle stays
    usable afterwards."""
    w = case["w"]
    res = np.zeros((w.nt, case["rec"].shape[0]), np.float32, order="F")
    res[7, 3] = np.nan
    with handle(pkg, case, preset="mixed", **opt) as h:
        with pytest.raises(pkg.DawError) as e:
            h.submodeling_adjoint_esource_data(res, case["rec"])
        assert e.value.code == -5, str(e.value)
        res[7, 3] = 1.0
        g = h.submodeling_adjoint_esource_data(res, case["rec"])
        assert np.isfinite(g).all() and np.abs(g).max() > 0


def test_bounded_wait_reports_timeout(pkg, case):
    """The failure path of the device-side bounded waits: a wait that nothing
    completes gives up after its budget and is reported as DAW_ERR_TIMEOUT;
    no GPU fault is involved and the handle keeps working afterwards."""
    w = case["w"]
    with handle(pkg, case, preset="mixed") as h:
        assert pkg.lib().daw_selftest_wait_timeout(h._h) == -4
        assert "bounded device wait" in pkg.lib().daw_last_error(h._h).decode()
        sis, _ = h.submodeling(case["s"], case["src"], case["rec"])
        assert np.isfinite(sis).all() and np.abs(sis).max() > 0


@pytest.mark.parametrize("preset", ["plain", "mixed"])
def test_batched_forward_matches_single(pkg, O, case, preset):
    """daw_submodeling_shots (mode 0, many shots per launch) equals
    daw_submodeling shot by shot, bit for bit, with uneven record lengths
    and receiver spreads; the FP32 paths also equal the FP32 oracle."""
    w = case["w"]
    rng = np.random.default_rng(7)
    shots = []
    for i, (nt, nr) in enumerate([(w.nt, case["rec"].shape[0]), (w.nt - 37, 9), (w.nt - 5, 17)]):
        rec = case["rec"][:nr].copy()
        s = case["s"][:nt].copy()
        src = case["src"].copy()
        src[1] += 3 * i  # move the source a few columns per shot
        shots.append(dict(s=s, src=src, rec=rec, nt=nt))
    with handle(pkg, case, preset=preset) as h:
        got = h.submodeling_shots(shots)
        for sh, g1 in zip(shots, got):
            ref, _ = h.submodeling(sh["s"], sh["src"], sh["rec"])
            assert np.array_equal(g1, ref)
            ora, _ = O.submodeling(w.c0, w.npml, w.h, w.ofs, sh["nt"], w.dt, sh["s"], sh["src"],
                                   sh["rec"])
            assert np.array_equal(g1, ora)


@pytest.mark.parametrize("opt", [{}, {"step": 0}, {"step": 1}])
def test_batched_eleven_uneven_shots(pkg, O, case, opt):
    """Eleven shots in one batch -- more than the 8 whose per-shot pointers
    travel as kernel parameters, so the rest take the descriptor-load path --
    with record lengths 250..400 and receiver spreads of 7..24 channels; the
    short records end early, so later steps run on a subset of the batch.
    Every output equals the same shots run one per batch, bit for bit."""
    w = case["w"]
    rng = np.random.default_rng(11)
    shots = []
    for k in range(11):
        nt = int(rng.integers(250, 401))
        lo = int(rng.integers(0, 12))
        hi = int(rng.integers(lo + 7, 25))
        x = float(rng.uniform(200.0, 700.0))
        src = pkg.subacqui([[15.0, x]], w.h, w.npml, w.ofs)[0]
        rec = case["rec"][lo:hi]
        s = w.wavelet(nt)
        dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, nt, w.dt, s, src, rec)
        shots.append(dict(s=s, nt=nt, src=src, rec=rec, dobs=dobs, mu=w.mu, maxiter=2,
                          rtol=0.0, band=w.band, shot=k + 1))
    with handle(pkg, case, "mixed", **opt) as h:
        h.set_datum(case["ird"])
        batched = h.shots(shots)
        h.set_options(max_batch=1)
        serial = h.shots(shots)
    for b, s1 in zip(batched, serial):
        for key in ("datar", "deltadr", "deltade", "dataesc", "redatumed"):
            assert np.array_equal(b[key], s1[key]), key
