"""The reference workflow through daw_run_parfile: redatum.par, raw float32
models and wavelet, the acquisition text file, and the output files of modes
0-3 (sub_redatum_DAW.f90).  The driver batches shots in modes 0 and 1 without
wavefield files and runs the reference's per-shot steps otherwise; its files
must equal the C-ABI calls on the same inputs bit for bit."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(pkg):
    from daw_b200 import synthetic
    w = synthetic.small()
    return dict(w=w, s=w.wavelet())


def _raw(path, a):
    np.asarray(a, np.float32).ravel(order="F").tofile(path)


def _acqui(path, src_pos, rec_pos):
    with open(path, "w") as f:
        f.write(f"{len(src_pos)} {len(rec_pos)}\n")
        for z, x in list(src_pos) + list(rec_pos):
            f.write(f"{float(z):.9g} {float(x):.9g}\n")


def _par(path, w, mode, nsrc_maxiter, datum_file=None, oio=0):
    band = w.band
    lines = [
        f"{mode}                    !modeling",
        "vtrue.bin vinit.bin      !velocity model",
        "acqui.txt                !acquisition",
        "wavelet.bin              !wavelet file",
        f"{band[0]} {band[1]} {band[2]} {band[3]}   !filter",
        f"{w.n1} {w.n2} {w.npml} {w.h} {w.nt} {w.dt} {w.dt}   !n1 n2 npml h nt dt dto",
        "0 0                      !source/receiver type",
        f"{w.ofs}                  !ofs",
        f"{w.mu}                  !penalty",
        f"{oio}                        !oio",
        f"0.0 {nsrc_maxiter}      !error maxiter",
    ]
    if datum_file:
        lines.append(datum_file)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def test_parfile_modes_0_and_1(pkg, case, tmp_path):
    w = case["w"]
    d = str(tmp_path)
    src_pos = np.array([w.src_pos[0], w.src_pos[0] + np.array([0.0, 3 * w.h]),
                        w.src_pos[0] + np.array([0.0, 7 * w.h])], np.float32)
    rec_pos = np.asarray(w.rec_pos[0], np.float32)
    hh = np.float32(w.h) * np.float32(w.h)
    s_file = (case["s"] * hh).astype(np.float32)
    s_api = (s_file / hh).astype(np.float32)  # the driver's division (main_redatum_DAW.f90:111)
    _raw(os.path.join(d, "vtrue.bin"), w.vtrue)
    _raw(os.path.join(d, "vinit.bin"), w.c0)
    _raw(os.path.join(d, "wavelet.bin"), s_file)
    _acqui(os.path.join(d, "acqui.txt"), src_pos, rec_pos)
    _acqui(os.path.join(d, "datum.txt"), [], np.asarray(w.datum_pos, np.float32))
    rec = pkg.subacqui(rec_pos, w.h, w.npml, w.ofs)
    srcs = [pkg.subacqui(src_pos[i:i + 1], w.h, w.npml, w.ofs)[0] for i in range(3)]
    with pkg.Handle(0, preset="mixed") as h:
        # mode 0: observed data of every shot in the true model
        _par(os.path.join(d, "redatum.par"), w, 0, w.maxiter)
        h.run_parfile(d)
        h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs)
        dobs = []
        for i in range(3):
            got = np.fromfile(os.path.join(d, f"dataobs_{i + 1:05d}.bin"), np.float32)
            ref, _ = h.submodeling(s_api, srcs[i], rec)
            assert np.array_equal(got.reshape(ref.shape, order="F"), ref)
            dobs.append(ref)
            os.replace(os.path.join(d, f"dataobs_{i + 1:05d}.bin"),
                       os.path.join(d, f"dataobs_org_{i + 1:05d}.bin"))
        # mode 1 with the datum record: redatumed data of every shot
        _par(os.path.join(d, "redatum.par"), w, 1, w.maxiter, "datum.txt")
        h.run_parfile(d)
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        ird = pkg.subacqui(np.asarray(w.datum_pos, np.float32), w.h, w.npml, w.ofs)
        h.set_datum(ird)
        outs = h.shots([dict(s=s_api, nt=w.nt, src=srcs[i], rec=rec, dobs=dobs[i], mu=w.mu,
                             maxiter=w.maxiter, rtol=0.0, band=w.band) for i in range(3)],
                       outputs=("redatumed",))
        for i in range(3):
            got = np.fromfile(os.path.join(d, f"dataobs_redatum_{i + 1:05d}.bin"), np.float32)
            ref = outs[i]["redatumed"]
            assert np.abs(ref).max() > 0
            assert np.array_equal(got.reshape(ref.shape, order="F"), ref)


def _read(path, shape):
    return np.fromfile(path, np.float32).reshape(shape, order="F")


def test_parfile_wavefield_files_and_modes_2_3(pkg, case, tmp_path):
    """oio = 1: mode 1 writes every intermediate of the reference
    (sub_redatum_DAW.f90:82-156), mode 3 (the Symes variant, :157-228)
    inverts the time-reversed observed data itself, and mode 2 (:229-257)
    resamples the stored DAW wavefields at the acquisition's receivers."""
    w = case["w"]
    d = str(tmp_path)
    src_pos = np.array([w.src_pos[0], w.src_pos[0] + np.array([0.0, 5 * w.h])], np.float32)
    rec_pos = np.asarray(w.rec_pos[0], np.float32)
    hh = np.float32(w.h) * np.float32(w.h)
    s_file = (case["s"] * hh).astype(np.float32)
    s_api = (s_file / hh).astype(np.float32)
    _raw(os.path.join(d, "vtrue.bin"), w.vtrue)
    _raw(os.path.join(d, "vinit.bin"), w.c0)
    _raw(os.path.join(d, "wavelet.bin"), s_file)
    _acqui(os.path.join(d, "acqui.txt"), src_pos, rec_pos)
    _acqui(os.path.join(d, "datum.txt"), [], np.asarray(w.datum_pos, np.float32))
    rec = pkg.subacqui(rec_pos, w.h, w.npml, w.ofs)
    ird = pkg.subacqui(np.asarray(w.datum_pos, np.float32), w.h, w.npml, w.ofs)
    srcs = [pkg.subacqui(src_pos[i:i + 1], w.h, w.npml, w.ofs)[0] for i in range(2)]
    nt, nr = w.nt, rec.shape[0]
    wshape = (w.n1, w.n2, nt)
    f = lambda name, i: os.path.join(d, f"{name}{i + 1:05d}.bin")
    rev = lambda a: np.asfortranarray(a[::-1])
    with pkg.Handle(0, preset="mixed") as h:
        h.set_model(w.vtrue, w.npml, w.h, w.dt, w.ofs)
        dobs = [h.submodeling(s_api, srcs[i], rec)[0] for i in range(2)]
        for i in range(2):
            _raw(f("dataobs_org_", i), dobs[i])
        # mode 1 with every intermediate file
        _par(os.path.join(d, "redatum.par"), w, 1, 3, "datum.txt", oio=1)
        h.run_parfile(d)
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        for i in range(2):
            datar, wr = h.submodeling(s_api, srcs[i], rec, wavefield=True)
            assert np.array_equal(_read(f("datar_", i), (nt, nr)), datar)
            assert np.array_equal(_read(f("wavefield_ini", i), wshape), wr)
            deltadr = rev(dobs[i] - datar)  # subresiduals.f90:12-16
            assert np.array_equal(_read(f("deltadr_", i), (nt, nr)), rev(deltadr))
            deltade, info = h.sublinearminres(deltadr, rec, w.mu, 3, 0.0)
            assert info["itn"] == 3
            assert np.array_equal(_read(f("deltade_", i), (nt, nr)), rev(deltade))
            dataesc, we, _ = h.submodeling_adjoint_esource(deltade, rec)
            assert np.array_equal(_read(f("dataesc_", i), (nt, nr)), dataesc)
            assert np.array_equal(_read(f("datae_", i), (nt, nr)), datar + dataesc)
            wexd = wr + we
            assert np.array_equal(_read(f("wavefield_exd", i), wshape), wexd)
            red, _ = h.filmartin2d(h.subwavefieldresample(wexd, ird), w.dt, *w.band)
            assert np.abs(red).max() > 0
            assert np.array_equal(_read(f("dataobs_redatum_", i), (nt, ird.shape[0])), red)
            with open(os.path.join(d, f"MINRES_{i + 1:05d}.txt")) as fh:
                assert "Enter MINRES" in fh.read()
        # mode 3: the time-reversed observed data is the residual
        _par(os.path.join(d, "redatum.par"), w, 3, 3, oio=1)
        h.run_parfile(d)
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        wexd3 = []
        for i in range(2):
            assert np.array_equal(_read(f("deltadr_", i), (nt, nr)), dobs[i])
            deltade, _ = h.sublinearminres(rev(dobs[i]), rec, w.mu, 3, 0.0)
            assert np.array_equal(_read(f("deltade_", i), (nt, nr)), rev(deltade))
            dataesc, we, _ = h.submodeling_adjoint_esource(deltade, rec)
            assert np.array_equal(_read(f("dataesc_", i), (nt, nr)), dataesc)
            assert np.array_equal(_read(f("wavefield_exd", i), wshape), we)
            wexd3.append(we)
        # mode 2: the stored wavefields resampled at the acquisition's receivers
        _par(os.path.join(d, "redatum.par"), w, 2, 3)
        h.run_parfile(d)
        h.set_model(w.c0, w.npml, w.h, w.dt, w.ofs)
        for i in range(2):
            red, _ = h.filmartin2d(h.subwavefieldresample(wexd3[i], rec), w.dt, *w.band)
            assert np.array_equal(_read(f("dataobs_redatum_", i), (nt, nr)), red)


@pytest.mark.parametrize("preset,prec,tol", [("plain", "f32", 1e-4), ("mixed", "f64", 1e-3)])
def test_parfile_mode3_against_oracle(pkg, O, case, tmp_path, preset, prec, tol):
    """Mode 3 (the Symes variant, sub_redatum_DAW.f90:157-228) against the
    CPU oracle: the time-reversed observed data are the residual
    (:174-178), MINRES solves for deltade (:192), and the final extended
    source gives dataesc and the wavefield (:208-219).  The plain FP32 port is
    held to the FP32 oracle (1e-4), the mixed path to the FP64 oracle (1e-3);
    deltadr is a reversal, bit for bit."""
    w = case["w"]
    d = str(tmp_path)
    src_pos = np.array([w.src_pos[0]], np.float32)
    rec_pos = np.asarray(w.rec_pos[0], np.float32)
    hh = np.float32(w.h) * np.float32(w.h)
    s_file = (case["s"] * hh).astype(np.float32)
    s_api = (s_file / hh).astype(np.float32)
    _raw(os.path.join(d, "vtrue.bin"), w.vtrue)
    _raw(os.path.join(d, "vinit.bin"), w.c0)
    _raw(os.path.join(d, "wavelet.bin"), s_file)
    _acqui(os.path.join(d, "acqui.txt"), src_pos, rec_pos)
    rec = O.acqui_table(rec_pos, w.h, w.npml, w.ofs)
    src = O.acqui_table(src_pos, w.h, w.npml, w.ofs)[0]
    nt, nr = w.nt, rec.shape[0]
    dobs, _ = O.submodeling(w.vtrue, w.npml, w.h, w.ofs, nt, w.dt, s_api, src, rec)
    _raw(os.path.join(d, "dataobs_org_00001.bin"), dobs)
    _par(os.path.join(d, "redatum.par"), w, 3, 3, oio=1)
    with pkg.Handle(0, preset=preset) as h:
        h.run_parfile(d)
    f = lambda name: os.path.join(d, f"{name}00001.bin")
    T = np.float32 if prec == "f32" else np.float64
    deltadr = np.asfortranarray(dobs[::-1]).astype(T)
    ref_de, info = O.linear_minres(w.c0, w.npml, w.h, w.ofs, nt, w.dt, rec, deltadr, w.mu, 3,
                                   0.0, prec=prec)
    assert info["itn"] == 3
    ref_esc, ref_wf, _ = O.esource(w.c0, w.npml, w.h, w.ofs, nt, w.dt, ref_de, rec, prec=prec)
    from conftest import rel_l2
    assert np.array_equal(_read(f("deltadr_"), (nt, nr)), dobs)
    got_de = _read(f("deltade_"), (nt, nr))[::-1]
    assert rel_l2(got_de, ref_de) <= tol, rel_l2(got_de, ref_de)
    got_esc = _read(f("dataesc_"), (nt, nr))
    assert rel_l2(got_esc, ref_esc) <= tol, rel_l2(got_esc, ref_esc)
    got_wf = _read(f("wavefield_exd"), (w.n1, w.n2, nt))
    assert rel_l2(got_wf, ref_wf) <= tol, rel_l2(got_wf, ref_wf)
