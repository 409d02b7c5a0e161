"""GPU parity with a density model (Gardner's rho = 0.31 vp^0.25) against the
CPU oracle.

The reference fixes rho = 1 (submodeling2.f90:88-93) but carries density
through substagger (:1227-1270): kappa = rho vp^2, buoyancy 1/rho averaged
onto the staggered grids, and the buoyancy weight of the velocity sources
(:252, :838, :845).  The bars are those of the rho = 1 parity tests: the
plain port and the split TMA kernels with FP32 histories reproduce the FP32
oracle bit for bit; full shots are within 1e-4 of the FP32 oracle (FP32
paths) or 1e-3 of the FP64 oracle (FP16 histories).
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
    w = synthetic.small(seed=11)
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    ird = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
    s = w.wavelet()
    rho_true, rho0 = synthetic.gardner(w.vtrue), synthetic.gardner(w.c0)
    with O.density(rho_true):
        dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, w.nt, w.dt, s, src, rec)
    return dict(w=w, src=src, rec=rec, ird=ird, s=s, dobs=dobs, rho=rho0)


def handle(pkg, case, preset="plain", rho=True, **opt):
    w = case["w"]
    h = pkg.Handle(0, preset=preset, **opt)
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs, rho=case["rho"] if rho is True else rho)
    return h


# the plain port, the split TMA kernels (autotuned launch shape, direct
# launches, PDL) and the autotuner allowed to consider the step family
PATHS = [("plain", {}), ("mixed", {"history": 0}), ("mixed", {"history": 0, "graph": 0}),
         ("mixed", {"history": 0, "pdl": 1}), ("mixed", {"history": 0, "step": 2})]


@pytest.mark.parametrize("type_src", [0, 1])
@pytest.mark.parametrize("preset,opt", PATHS)
def test_forward_bitexact(pkg, O, case, preset, opt, type_src):
    w = case["w"]
    with O.density(case["rho"]):
        ref, refwf = O.submodeling(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["s"], case["src"],
                                   case["rec"], type_src=type_src, want_wavefield=True)
    with handle(pkg, case, preset, **opt) as h:
        sis, wf = h.submodeling(case["s"], case["src"], case["rec"], type_src=type_src,
                                wavefield=True)
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)


@pytest.mark.parametrize("preset,opt", PATHS)
def test_ggt_bitexact(pkg, O, case, preset, opt):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    with O.density(case["rho"]):
        ref = O.esource_data(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res, case["rec"])
    with handle(pkg, case, preset, **opt) as h:
        g = h.submodeling_adjoint_esource_data(res, case["rec"])
    assert np.array_equal(g, ref)


@pytest.mark.parametrize("preset,opt", PATHS[:2])
def test_esource_bitexact(pkg, O, case, preset, opt):
    w = case["w"]
    res = np.asfortranarray(case["dobs"][::-1])
    with O.density(case["rho"]):
        ref, refwf, _ = O.esource(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, res, case["rec"])
    with handle(pkg, case, preset, **opt) as h:
        sis, wf, _ = h.submodeling_adjoint_esource(res, case["rec"])
    assert np.array_equal(sis, ref)
    assert np.array_equal(wf, refwf)


@pytest.fixture(scope="module")
def oracle_shots(O, case):
    w = case["w"]
    with O.density(case["rho"]):
        return {p: O.daw_shot(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["s"], case["src"],
                              case["rec"], case["dobs"], w.mu, w.maxiter, 0.0, case["ird"],
                              w.band, prec=p) for p in ("f32", "f64")}


def _shot(case):
    w = case["w"]
    return dict(s=case["s"], nt=w.nt, src=case["src"], rec=case["rec"], dobs=case["dobs"],
                mu=w.mu, maxiter=w.maxiter, rtol=0.0, band=w.band)


@pytest.mark.parametrize("preset,opt,prec,tol", [("plain", {}, "f32", FP32_TOL),
                                                 ("mixed", {}, "f64", MIXED_TOL),
                                                 ("mixed", {"history": 0}, "f32", FP32_TOL)])
def test_shot_pipeline(pkg, case, oracle_shots, preset, opt, prec, tol):
    with handle(pkg, case, preset, **opt) as h:
        h.set_datum(case["ird"])
        out = h.shot(**_shot(case))
    ref = oracle_shots[prec]
    if prec == "f32":
        assert np.array_equal(out["datar"], ref["datar"])
        assert np.array_equal(out["deltadr"], ref["deltadr"])
    for k in ("deltade", "dataesc", "datae", "redatumed_raw", "redatumed"):
        err = rel_l2(out[k], ref[k])
        assert err <= tol, (k, err)


def test_density_changes_the_result(pkg, case):
    """The density reaches the kernels: the same shot with rho = 1 differs."""
    with handle(pkg, case, "mixed", rho=None) as h:
        h.set_datum(case["ird"])
        one = h.shot(**_shot(case))
    with handle(pkg, case, "mixed") as h:
        h.set_datum(case["ird"])
        gard = h.shot(**_shot(case))
    assert rel_l2(gard["datar"], one["datar"]) > 1e-2


def test_density_one_equals_default(pkg, case):
    """rho = 1 given explicitly takes the 2-D buoyancy path and reproduces the
    default (1-D profile) path bit for bit, through a whole mixed shot."""
    w = case["w"]
    outs = []
    for rho in (None, np.ones_like(w.c0)):
        with handle(pkg, case, "mixed", rho=rho) as h:
            h.set_datum(case["ird"])
            outs.append(h.shot(**_shot(case)))
    for k in ("datar", "deltade", "dataesc", "redatumed"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.parametrize("opt", [{"step": 1}, {"chunk": 1}])
def test_kernels_without_density_refuse_it(pkg, case, opt):
    from daw_b200 import DawError
    with handle(pkg, case, "mixed", **opt) as h:
        with pytest.raises(DawError, match="density"):
            h.submodeling(case["s"], case["src"], case["rec"])


def _with_density(O, rho, fn, *args, **kw):
    with O.density(rho):
        return fn(*args, **kw)


NT2 = 200


def test_751x2301_forward_and_ggt_bitexact(pkg, O):
    """The benchmark grid (751x2301, h = 4 m, npml 40, 576 receivers) with
    Gardner density, nt 200: forward modelling (pressure and velocity
    sources) and G G^T of the plain port and the split TMA kernels (FP32
    histories) against the FP32 oracle, bit for bit.  The oracle runs in
    worker threads while the GPU runs."""
    from concurrent.futures import ThreadPoolExecutor
    from daw_b200 import synthetic
    w = synthetic.config2(nshot=1, nt=NT2)
    rho = synthetic.gardner(w.c0)
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    s = w.wavelet(NT2 + 140)[140:].copy()  # Ricker peak at step 60
    args = (w.c0, w.npml, w.h, w.ofs, NT2, w.dt)
    with ThreadPoolExecutor(3) as pool:
        fut = {t: pool.submit(_with_density, O, rho, O.submodeling, *args, s, src, rec,
                              type_src=t) for t in (0, 1)}
        dobs = fut[0].result()[0]
        res = np.asfortranarray(dobs[::-1])
        fut["ggt"] = pool.submit(_with_density, O, rho, O.esource_data, *args, res, rec)
        got = {}
        for preset, opt in (("plain", {}), ("mixed", {"history": 0})):
            with pkg.Handle(0, preset=preset, **opt) as h:
                h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs, rho=rho)
                got[preset] = ([h.submodeling(s, src, rec, type_src=t)[0] for t in (0, 1)],
                               h.submodeling_adjoint_esource_data(res, rec))
        ref = ([fut[0].result()[0], fut[1].result()[0]], fut["ggt"].result())
    assert np.abs(ref[0][0]).max() > 0
    for preset, (fw, g) in got.items():
        for t in (0, 1):
            assert np.array_equal(fw[t], ref[0][t]), (preset, t)
        assert np.array_equal(g, ref[1]), preset


def _equal_above_precursor(a, b):
    """a == b bit for bit wherever |b| > 1e-6 max|b|; below, |a - b| <=
    1e-9 max|b|.  A power-of-two scaling commutes with rounding except in the
    FP32 subnormal range, reached by the stencil's exponentially small
    precursor ahead of the wavefront; its 1-ulp differences grow with the
    precursor but stay many decades below the signal."""
    peak = np.abs(b).max()
    big = np.abs(b) > 1e-6 * peak
    assert np.array_equal(a[big], b[big])
    assert np.abs(a - b).max() <= 1e-9 * peak


def test_power_of_two_density_on_751x2301(pkg):
    """Size-independent identity on the benchmark grid (751x2301, h = 4 m,
    576 receivers, FP16-history mixed preset, nt 300): rho = 2 doubles kappa
    and halves the buoyancy, so a pressure source's data double and a
    velocity source's are unchanged (exactly, above the precursor)."""
    from daw_b200 import synthetic
    w = synthetic.config2(nshot=1, nt=300)
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    s = w.wavelet(300)
    out = {}
    for r in (None, 2.0):
        with pkg.Handle(0, preset="mixed") as h:
            h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs,
                        rho=None if r is None else np.full_like(w.c0, r))
            out[r] = [h.submodeling(s, src, rec, type_src=t)[0] for t in (0, 1)]
    assert np.abs(out[None][0]).max() > 0
    _equal_above_precursor(out[2.0][0], 2 * out[None][0])
    _equal_above_precursor(out[2.0][1], out[None][1])


def test_batched_windowed_shots_with_density(pkg, O, case):
    """Three uneven shots with density in one batch equal the same shots run
    one at a time, and stage-A history windows change no bit."""
    w = case["w"]
    shots = []
    for k, (nt, lo, hi, x) in enumerate([(400, 0, 24, 300.0), (330, 4, 17, 520.0),
                                         (371, 10, 24, 700.0)]):
        src = pkg.subacqui([[15.0, x]], w.h, w.npml, w.ofs)[0]
        rec = case["rec"][lo:hi]
        s = w.wavelet(nt)
        with O.density(synthetic_rho_true(case)):
            dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, nt, w.dt, s, src, rec)
        shots.append(dict(s=s, nt=nt, src=src, rec=rec, dobs=dobs, mu=w.mu, maxiter=3,
                          rtol=0.0, band=w.band, shot=k + 1))
    with handle(pkg, case, "mixed") as h:
        h.set_datum(case["ird"])
        batched = h.shots(shots)
        single = [h.shots([sh])[0] for sh in shots]
        h.set_options(checkpoint=37)
        windowed = h.shots(shots)
    for b, s1, s2 in zip(batched, single, windowed):
        for key in ("deltade", "dataesc", "redatumed"):
            assert np.array_equal(b[key], s1[key]), key
            assert np.array_equal(b[key], s2[key]), key


def synthetic_rho_true(case):
    from daw_b200 import synthetic
    return synthetic.gardner(case["w"].vtrue)
