"""Checkpointed stage A (DAW_OPT_CHECKPOINT = K): the stage-A history is kept
in windows of K steps.  Stage A runs once over the record, saving its state
before each window, and is re-run over each window from the saved state while
stage B consumes the windows in reverse order.  The recomputed histories come
from the same operations as the whole-record run, so every output must equal
the whole-record path's bit for bit: the G G^T operator, the final esource
(sis, wavefield), MINRES and the full shot pipeline.  Only the FP64 `cost`
sum, whose order is unspecified in both paths, is compared with a tolerance.
Windows that divide the record and windows that leave a short last window,
FP16 and FP32 histories, and the TMA and register kernels are covered."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(pkg):
    from daw_b200 import synthetic
    w = synthetic.small()
    src = pkg.subacqui(w.src_pos, w.h, w.npml, w.ofs)[0]
    rec = pkg.subacqui(w.rec_pos[0], w.h, w.npml, w.ofs)
    ird = pkg.subacqui(w.datum_pos, w.h, w.npml, w.ofs)
    s = w.wavelet()
    with pkg.Handle(0, preset="plain") as h:
        h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs)
        dobs, _ = h.submodeling(s, src, rec)
    return dict(w=w, src=src, rec=rec, ird=ird, s=s, dobs=dobs,
                res=np.asfortranarray(dobs[::-1]))


def handle(pkg, case, **opt):
    w = case["w"]
    h = pkg.Handle(0, preset="mixed", **opt)
    h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
    return h


def test_option_roundtrip(pkg, case):
    with handle(pkg, case) as h:
        assert h.get_option("checkpoint") == 0
        h.set_options(checkpoint=25)
        assert h.get_option("checkpoint") == 25
        with pytest.raises(pkg.DawError):
            h.set_options(checkpoint=-1)
        assert h.get_option("checkpoint") == 25


# (options, window lengths): nt = 400, so 1 and 399 are the extremes, 7 leaves
# a last window of 1 step and 100 divides the record.
GGT_CASES = [({}, (1, 7, 100, 399)), ({"history": 0}, (7, 64)), ({"graph": 0}, (50,)),
             ({"step": 1}, (7, 100)), ({"step": 1, "history": 0}, (33,)),
             ({"chunk": 2}, (7,)), ({"chunk": 1, "history": 0}, (33,))]


@pytest.mark.parametrize("opt,windows", GGT_CASES)
def test_windowed_ggt_bitexact(pkg, case, opt, windows):
    with handle(pkg, case, **opt) as h:
        ref = h.submodeling_adjoint_esource_data(case["res"], case["rec"])
        assert np.abs(ref).max() > 0
        for k in windows:
            h.set_options(checkpoint=k)
            got = h.submodeling_adjoint_esource_data(case["res"], case["rec"])
            assert np.array_equal(got, ref), k
        h.set_options(checkpoint=0)
        assert np.array_equal(h.submodeling_adjoint_esource_data(case["res"], case["rec"]), ref)


def test_windowed_ggt_matches_oracle(pkg, O, case):
    """FP32 histories: the windowed operator equals the FP32 CPU oracle."""
    w = case["w"]
    ref = O.esource_data(w.c0, w.npml, w.h, w.ofs, w.nt, w.dt, case["res"], case["rec"])
    with handle(pkg, case, history=0, checkpoint=9) as h:
        got = h.submodeling_adjoint_esource_data(case["res"], case["rec"])
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("opt", [{}, {"history": 0}, {"step": 1}])
def test_windowed_esource_bitexact(pkg, case, opt):
    with handle(pkg, case, **opt) as h:
        sis0, wf0, cost0 = h.submodeling_adjoint_esource(case["res"], case["rec"])
        h.set_options(checkpoint=13)
        sis, wf, cost = h.submodeling_adjoint_esource(case["res"], case["rec"])
    assert np.array_equal(sis, sis0)
    assert np.array_equal(wf, wf0)
    assert abs(cost - cost0) <= 1e-12 * abs(cost0)


def test_windowed_minres_bitexact(pkg, case):
    w = case["w"]
    with handle(pkg, case) as h:
        x0, i0 = h.sublinearminres(case["res"], case["rec"], w.mu, 4, 0.0)
        h.set_options(checkpoint=41)
        x, i = h.sublinearminres(case["res"], case["rec"], w.mu, 4, 0.0)
    assert np.array_equal(x, x0)
    assert i["itn"] == i0["itn"] and i["istop"] == i0["istop"]
    assert np.array_equal(i["log"], i0["log"])


def _shots(pkg, case):
    w = case["w"]
    out = []
    for k, (nt, lo, hi, x) in enumerate([(400, 0, 24, 300.0), (330, 4, 17, 520.0)]):
        src = pkg.subacqui([[15.0, x]], w.h, w.npml, w.ofs)[0]
        rec = case["rec"][lo:hi]
        s = w.wavelet(nt)
        with pkg.Handle(0, preset="plain") as h:
            h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs)
            dobs, _ = h.submodeling(s, src, rec)
        out.append(dict(s=s, nt=nt, src=src, rec=rec, dobs=dobs, mu=w.mu, maxiter=3,
                        rtol=0.0, band=w.band, shot=k + 1))
    return out


def test_windowed_shots_bitexact(pkg, case):
    """The full pipeline (forward, MINRES, final esource with the datum gather
    and the filter) of two shots of different lengths: windowed shots run one
    at a time and equal the whole-record batch."""
    shots = _shots(pkg, case)
    keys = ("datar", "deltadr", "deltade", "dataesc", "datae", "redatumed_raw", "redatumed")
    with handle(pkg, case) as h:
        h.set_datum(case["ird"])
        ref = h.shots(shots)
        h.set_options(checkpoint=64)
        got = h.shots(shots)
    for r, g in zip(ref, got):
        for k in keys:
            assert np.array_equal(g[k], r[k]), k
        assert g["minres"]["itn"] == r["minres"]["itn"]
        assert abs(g["cost"] - r["cost"]) <= 1e-12 * abs(r["cost"])
        assert np.abs(r["redatumed"]).max() > 0


def test_requested_window_too_small_is_refused(pkg, case):
    """DAW_OPT_CHECKPOINT = K keeps ceil(nt/K) saved states of the extended
    grid.  On the 751 x 2301 grid (npml 40, 40 MB per state) windows of one
    step over 7500 steps would need ~300 GB of states: the request is refused
    at admission with DAW_ERR_OOM, before any history is allocated, and the
    handle keeps working."""
    from daw_b200 import synthetic
    w2 = synthetic.config2(nshot=1, nt=7500)
    rec = pkg.subacqui(w2.rec_pos[0][:4], w2.h, w2.npml, w2.ofs)
    res = np.zeros((7500, 4), np.float32, order="F")
    with pkg.Handle(0, preset="mixed", checkpoint=1) as h:
        h.set_model(w2.c0, w2.npml, w2.h, w2.dt, w2.ofs)
        with pytest.raises(pkg.DawError) as e:
            h.submodeling_adjoint_esource_data(res, rec)
        assert e.value.code == -2, str(e.value)
        assert "history windows of 1 steps" in str(e.value)
        h.set_options(checkpoint=3000)
        g = h.submodeling_adjoint_esource_data(np.zeros((300, 4), np.float32, order="F"), rec)
        assert not g.any()


def test_windowed_equals_whole_record_on_2001x8001(pkg):
    """The 2001 x 8001 grid (h = 5 m, npml 50, 1200 receivers, datum at
    2500 m) with a short record: a shot with stage-A history windows of 30
    steps equals the whole-record shot bit for bit (two MINRES iterations).
    Within 90 steps the wave stays where the true and background models
    coincide, so the observed data are zero (residual = -datar)."""
    from daw_b200 import synthetic
    w = synthetic.config5()
    nt = 90
    src = pkg.subacqui(w.src_pos[100:101], w.h, w.npml, w.ofs)[0]  # x = 3900 m, a receiver below
    rec = pkg.subacqui(w.rec_pos[0][::8], w.h, w.npml, w.ofs)
    ird = pkg.subacqui(w.datum_pos[::8], w.h, w.npml, w.ofs)
    s = w.wavelet(nt + 60)[60:].copy()
    with pkg.Handle(0, preset="mixed") as h:
        dobs = np.zeros((nt, rec.shape[0]), np.float32, order="F")
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        h.set_datum(ird)
        kw = dict(s=s, nt=nt, src=src, rec=rec, dobs=dobs, mu=w.mu, maxiter=2, rtol=0.0,
                  band=w.band)
        whole = h.shot(**kw)
        h.set_options(checkpoint=30)
        win = h.shot(**kw)
    assert np.abs(whole["deltade"]).max() > 0
    for key in ("datar", "deltade", "dataesc", "redatumed"):
        assert np.array_equal(win[key], whole[key]), key
