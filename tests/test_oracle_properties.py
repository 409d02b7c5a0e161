"""Algebraic and physical identities of the reference's algorithm, checked on
the CPU oracle (they pin the restatement beyond the golden fixtures)."""
import numpy as np
import pytest

from conftest import rel_l2


def _case():
    n1, n2, npml, h, dt, nt = 30, 46, 10, 10.0, 0.001, 150
    rng = np.random.default_rng(3)
    vp = np.asfortranarray((1800 + rng.uniform(-50, 50, (n1, n2))).astype(np.float32))
    return vp, npml, h, dt, nt


def test_monopole_tiles_sum_to_one(O):
    for a1 in (1, 17, 51, 88, 100):
        for a2 in (1, 40, 51, 99):
            assert abs(O.kws_tile(a1, a2, 0).sum() - 1.0) < 1e-5


def test_free_surface_mirror(O):
    # nfs nodes above the surface row keep their weights; the surface row is 0;
    # the nfs rows below get w(k) - w(mirror)
    base = O.kws_tile(37, 12, 0)
    for nfs in (1, 4, 9, 10):
        t = O.kws_tile(37, 12, nfs)
        assert np.all(t[nfs, :] == 0)
        for k in range(1, nfs + 1):
            assert np.allclose(t[nfs + k], base[nfs + k] - base[nfs - k], atol=0, rtol=0)
        assert np.array_equal(t[:nfs], base[:nfs])
        assert np.array_equal(t[2 * nfs + 1:], base[2 * nfs + 1:])


def test_locate_grid_node(O):
    # on a node: alpha = 0 -> ialpha 51, support symmetric
    assert list(O.subsourcekws(40.0, 100.0, 20.0, 1)) == [3, 6, 51, 51, 8]
    assert list(O.subsourcekws(40.0, 100.0, 20.0, 0))[4] == 0


def test_operator_power_of_two_linearity(O):
    """G G^T(2 x) == 2 G G^T(x) bit for bit (power-of-two scaling commutes
    with rounding)."""
    vp, npml, h, dt, nt = _case()
    ir = O.acqui_table([[15.0, x] for x in np.linspace(0, 450, 7)], h, npml, 1)
    x = np.asfortranarray(np.random.default_rng(1).standard_normal((nt, 7)).astype(np.float32))
    g1 = O.esource_data(vp, npml, h, 1, nt, dt, x, ir)
    g2 = O.esource_data(vp, npml, h, 1, nt, dt, 2 * x, ir)
    assert np.array_equal(g2, 2 * g1)


def test_operator_symmetry(O):
    """A = R G G^T is the symmetric operator MINRES assumes: <A a, b> = <a, A b>
    to the discretisation's adjoint accuracy (the disabled checkA probe of
    minresModule.f90:119-134)."""
    vp, npml, h, dt, nt = _case()
    ir = O.acqui_table([[15.0, x] for x in np.linspace(0, 450, 7)], h, npml, 1)
    rng = np.random.default_rng(2)
    a = np.asfortranarray(rng.standard_normal((nt, 7)))
    b = np.asfortranarray(rng.standard_normal((nt, 7)))
    A = lambda v: O.esource_data(vp, npml, h, 1, nt, dt, v, ir, prec="f64")[::-1]
    lhs, rhs = np.sum(A(a) * b), np.sum(a * A(b))
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs)


def test_fp32_vs_fp64(O):
    vp, npml, h, dt, nt = _case()
    ir = O.acqui_table([[15.0, x] for x in np.linspace(0, 450, 7)], h, npml, 1)
    is5 = O.acqui_table([[25.0, 230.0]], h, npml, 1)[0]
    s = np.sin(np.arange(nt) * 0.2).astype(np.float32) * np.exp(-np.arange(nt) * 0.02).astype(np.float32)
    a, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)
    b, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, prec="f64")
    assert rel_l2(a, b) <= 1e-5


def test_homogeneous_green_function(O):
    """Forward modelling in a homogeneous medium without free surface against
    the 2-D acoustic Green's function convolved with the source: the
    reference's scheme (staggered O(2,4), Hicks injection, s/h^2 scaling)
    models the point source p_tt = c^2 lap p + c^2 s delta."""
    n1 = n2 = 121
    npml, h, dt, nt, c = 30, 10.0, 0.001, 300, 2000.0
    vp = np.full((n1, n2), c, np.float32, order="F")
    f0 = 15.0
    t = np.arange(nt) * dt - 1.0 / f0
    w = ((1 - 2 * (np.pi * f0 * t) ** 2) * np.exp(-(np.pi * f0 * t) ** 2))
    s = (w / h ** 2).astype(np.float32)
    src = O.acqui_table([[600.0, 600.0]], h, npml, 0)[0]
    offs = np.array([150.0, 250.0, 350.0])
    ir = O.acqui_table([[600.0, 600.0 + o] for o in offs], h, npml, 0)
    sis, _ = O.submodeling(vp, npml, h, 0, nt, dt, s, src, ir, prec="f64")
    # The scheme injects dt*kappa*w/h^2 per step: p_t = kappa div v + kappa w(t) delta,
    # so p_tt = c^2 lap p + c^2 w'(t) delta and p = c^2 G * w' with the 2-D
    # Green's function G = H(t - r/c) / (2 pi c sqrt(c^2 t^2 - r^2)).  Written
    # with the integrated kernel K(t) = acosh(ct/r)/(2 pi) (K' = c^2 G):
    # p = K * w''.
    tt = np.arange(nt) * dt
    w2 = np.gradient(np.gradient(w, dt), dt)
    for k, r in enumerate(offs):
        K = np.arccosh(np.maximum(c * tt / r, 1.0)) / (2 * np.pi)
        ana = np.convolve(w2, K)[:nt] * dt
        num = sis[:, k]
        scale = np.dot(num, ana) / np.dot(ana, ana)
        assert rel_l2(num, scale * ana) < 0.1
        assert 0.9 < scale < 1.1, scale


def _sources(O, vp, npml, h, nt):
    ir = O.acqui_table([[15.0, x] for x in np.linspace(0, 450, 7)], h, npml, 1)
    is5 = O.acqui_table([[25.0, 230.0]], h, npml, 1)[0]
    s = np.sin(np.arange(nt) * 0.2).astype(np.float32) * np.exp(-np.arange(nt) * 0.02).astype(np.float32)
    return ir, is5, s


def test_density_one_is_the_reference(O):
    """A density of 1 given explicitly runs the reference's rho = 1 arithmetic
    bit for bit (substagger, submodeling2.f90:1227-1270)."""
    vp, npml, h, dt, nt = _case()
    ir, is5, s = _sources(O, vp, npml, h, nt)
    res = np.asfortranarray(np.random.default_rng(4).standard_normal((nt, 7)).astype(np.float32))
    a, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)
    v, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, type_src=1)
    g = O.esource_data(vp, npml, h, 1, nt, dt, res, ir)
    e, _, _ = O.esource(vp, npml, h, 1, nt, dt, res, ir, want_wavefield=False)
    with O.density(np.ones_like(vp)):
        assert np.array_equal(O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)[0], a)
        assert np.array_equal(O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, type_src=1)[0], v)
        assert np.array_equal(O.esource_data(vp, npml, h, 1, nt, dt, res, ir), g)
        assert np.array_equal(O.esource(vp, npml, h, 1, nt, dt, res, ir, want_wavefield=False)[0], e)


def test_density_power_of_two_scaling(O):
    """rho = 2 doubles kappa and halves the buoyancy: the pressure of a
    pressure source doubles exactly, and that of a velocity source (weighted
    by the buoyancy, :252) is unchanged bit for bit (power-of-two scalings
    commute with rounding)."""
    vp, npml, h, dt, nt = _case()
    ir, is5, s = _sources(O, vp, npml, h, nt)
    a, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)
    v, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, type_src=1)
    with O.density(np.full_like(vp, 2.0)):
        a2, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)
        v2, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, type_src=1)
    assert np.array_equal(a2, 2 * a)
    assert np.array_equal(v2, v)


@pytest.mark.parametrize("rho2", [2.0, 0.5])
def test_density_contrast_reflection(O, rho2):
    """A density step at constant velocity reflects with R = (rho2 - rho1) /
    (rho2 + rho1) at every angle (equal velocities: no refraction).  The
    reflected wave (the difference from the rho = 1 run) is compared with
    R times the direct wave of the rho = 1 run at the image distance."""
    n1 = n2 = 121
    npml, h, dt, nt, c = 30, 10.0, 0.001, 500, 2000.0
    vp = np.full((n1, n2), c, np.float32, order="F")
    rho = np.ones((n1, n2), np.float32, order="F")
    rho[61:, :] = rho2  # interface between rows 60 and 61 (z = 600-610 m)
    f0 = 12.0
    t = np.arange(nt) * dt - 1.0 / f0
    s = (((1 - 2 * (np.pi * f0 * t) ** 2) * np.exp(-(np.pi * f0 * t) ** 2)) / h ** 2).astype(np.float32)
    src = O.acqui_table([[300.0, 600.0]], h, npml, 0)[0]
    ir = O.acqui_table([[300.0, 650.0], [905.0, 650.0]], h, npml, 0)
    hom, _ = O.submodeling(vp, npml, h, 0, nt, dt, s, src, ir, prec="f64")
    with O.density(rho):
        het, _ = O.submodeling(vp, npml, h, 0, nt, dt, s, src, ir, prec="f64")
    refl = het[:, 0] - hom[:, 0]
    image = hom[:, 1]  # 605 m below the source: the image source's distance
    R = np.sign(np.dot(refl, image)) * np.max(np.abs(refl)) / np.max(np.abs(image))
    expect = (rho2 - 1.0) / (rho2 + 1.0)
    assert abs(R - expect) < 0.03, (R, expect)
    # arrival time within a few samples of the image wave's
    assert abs(int(np.argmax(np.abs(refl))) - int(np.argmax(np.abs(image)))) <= 8


def test_density_fp32_vs_fp64(O):
    """With a varying (Gardner) density the FP32 restatement stays within
    1e-5 of the FP64 one, as with density 1."""
    vp, npml, h, dt, nt = _case()
    ir, is5, s = _sources(O, vp, npml, h, nt)
    rho = np.asfortranarray((0.31 * vp.astype(np.float64) ** 0.25).astype(np.float32))
    with O.density(rho):
        a, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir)
        b, _ = O.submodeling(vp, npml, h, 1, nt, dt, s, is5, ir, prec="f64")
    assert rel_l2(a, b) <= 1e-5
