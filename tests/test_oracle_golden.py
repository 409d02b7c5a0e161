"""The CPU oracle against the golden fixtures of the independent numpy
restatement (tests/golden/make_golden.py).  CPU only."""
import numpy as np

from conftest import rel_l2

TOL = 2e-6  # 1-ulp differences of float transcendental functions in the 1-D KWS table


def test_kws_table(O, golden):
    c = O.kws_table1d()
    assert np.abs(c - golden["kws1d"]).max() <= 1.2e-7
    assert np.count_nonzero(c != golden["kws1d"]) <= 40


def test_tiles(O, golden):
    for t, a in zip(golden["tiles"], golden["tile_args"]):
        assert np.abs(O.kws_tile(*a) - t).max() <= 1.2e-7


def test_subsourcekws(O, golden):
    for p, t in zip(golden["kws_positions"], golden["kws_tables"]):
        assert np.array_equal(O.subsourcekws(*p[:3], int(p[3])), t)


def test_sponges(O, golden):
    npml, n1 = int(golden["npml"]), golden["vp"].shape[0]
    for a, b in zip(O.sponges(npml, n1), golden["sponge"]):
        assert np.array_equal(a, b)


def _args(g):
    return g["vp"], int(g["npml"]), float(g["h"]), int(g["ofs"]), int(g["nt"]), float(g["dt"])


def test_forward(O, golden):
    vp, npml, h, ofs, nt, dt = _args(golden)
    sis, wf = O.submodeling(vp, npml, h, ofs, nt, dt, golden["s"], golden["is5"], golden["ir"],
                            want_wavefield=True)
    assert rel_l2(sis, golden["fwd_sis"]) <= TOL
    assert rel_l2(wf[:, :, ::16], golden["fwd_wf_slices"]) <= TOL


def test_esource_data(O, golden):
    vp, npml, h, ofs, nt, dt = _args(golden)
    g = O.esource_data(vp, npml, h, ofs, nt, dt, golden["res"], golden["ir"])
    assert rel_l2(g, golden["ggt"]) <= TOL


def test_esource(O, golden):
    vp, npml, h, ofs, nt, dt = _args(golden)
    sis, wf, cost = O.esource(vp, npml, h, ofs, nt, dt, golden["res"], golden["ir"])
    assert rel_l2(sis, golden["es_sis"]) <= TOL
    assert rel_l2(wf[:, :, ::16], golden["es_wf_slices"]) <= TOL
    assert abs(cost - float(golden["es_cost"])) <= 1e-5 * abs(float(golden["es_cost"]))


def test_resample(O, golden):
    vp, npml, h, ofs, nt, dt = _args(golden)
    _, wf = O.submodeling(vp, npml, h, ofs, nt, dt, golden["s"], golden["is5"], golden["ir"],
                          want_wavefield=True)
    _, ewf, _ = O.esource(vp, npml, h, ofs, nt, dt, golden["res"], golden["ir"])
    rs = O.resample(npml, wf + ewf, golden["ird"])
    assert rel_l2(rs, golden["resampled"]) <= TOL


def test_filter(O, golden):
    vp, npml, h, ofs, nt, dt = _args(golden)
    sis, _ = O.submodeling(vp, npml, h, ofs, nt, dt, golden["s"], golden["is5"], golden["ir"])
    f, band = O.filmartin2d(sis, dt, *golden["band"])
    # the reference's REALFT2S keeps single-precision temporaries; the numpy
    # restatement is a pure FP64 FFT
    assert rel_l2(f, golden["filtered"]) <= 1e-6
