"""Generate the golden fixtures in this folder from an independent numpy
restatement of the reference's DAW hot path.

The reference (guogs93/Model-based-seismic-data-redatuming-with-DAWs) is
Fortran 90 + MPI and cannot be compiled in this image (no Fortran compiler),
and it ships no golden vectors.  This script is a second, vectorised
restatement written directly from the Fortran sources, independent of the
C++ oracle in ``oracle/``; the fixtures it writes pin the oracle (and through
it the CUDA library) to the reference's algorithm as read from its sources.

Run:  python tests/golden/make_golden.py   (writes golden_small.npz)

Arithmetic is float32 per operation (numpy float32 ops are separately
rounded, like the reference's REAL arithmetic); transcendental functions are
evaluated in float64 and rounded to float32.
"""
from __future__ import annotations

import os

import numpy as np

F = np.float32
IRAD, NALPHA = 10, 100
A0, A1 = F(1.125), F(-1.0) / F(24.0)


# -- kwsinc.f90 --------------------------------------------------------------

def bessi0(x):
    """kwsinc.f90:612-635 (A&S 9.8.1/9.8.2 with single-precision argument)."""
    x = F(x)
    if abs(x) < F(3.75):
        q = F(x / F(3.75))
        y = float(F(q * q))
        r = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (
            0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))))
        return F(r)
    ax = F(abs(x))
    y = float(F(F(3.75) / ax))
    pre = F(F(np.exp(float(ax))) / F(np.sqrt(float(ax))))
    r = float(pre) * (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 + y * (
        -0.157565e-2 + y * (0.916281e-2 + y * (-0.2057706e-1 + y * (
            0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))))
    return F(r)


def kws_table1d():
    """c[n+10, ia-1] (kwsinc.f90:94-179, monopole, b = bhicks0(10) = 14.18)."""
    pi = F(3.14159265359)
    b = F(14.18)
    den = bessi0(b)
    c = np.zeros((21, 100), F)
    for ia in range(1, 101):
        alpha = F(F(0.5) - F(F(ia - 1) / F(100)))
        for n in range(-10, 11):
            xn = F(F(n) + alpha)
            if abs(xn) <= F(10):
                if abs(xn) > F(1e-15):
                    arg = F(b * F(np.sqrt(float(F(F(1) - F(F(xn * xn) / F(100)))))))
                    kai = F(bessi0(arg) / den)
                    v = F(F(kai * F(np.sin(float(F(pi * xn))))) / F(pi * xn))
                    if abs(v) < F(1e-15):
                        v = F(0)
                else:
                    v = F(1)
                c[n + 10, ia - 1] = v
    return c


def kws_tile(c1, ia1, ia2, nfs):
    t = (c1[None, :, ia2 - 1] * c1[:, None, ia1 - 1]).astype(F)
    out = t.copy()
    if nfs > 0:
        sym = -IRAD + nfs + IRAD
        out[sym, :] = 0
        for k in range(1, nfs + 1):
            out[sym + k, :] = t[sym + k, :] - t[sym - k, :]
    return out


def subsourcekws(z, x, dz, ifs):
    xs = [F(z), F(x)]
    ix, ia = [], []
    for v in xs:
        q = F(v / F(dz))
        i = int(np.floor(abs(float(q)) + 0.5)) * (1 if q >= 0 else -1) + 1
        x0 = F(F(i - 1) * F(dz))
        alpha = F(F(x0 - v) / F(dz))
        w = F(F(F(0.5) - alpha) * F(100))
        a = int(np.floor(abs(float(w)) + 0.5)) * (1 if w >= 0 else -1) + 1
        ix.append(i)
        ia.append(min(a, 100))
    q = F(xs[0] / F(dz))
    nf = IRAD - int(np.floor(abs(float(q)) + 0.5)) * (1 if q >= 0 else -1)
    nf = max(nf, 0)
    if ifs == 0:
        nf = 0
    return np.array([ix[0], ix[1], ia[0], ia[1], nf], np.int32)


def table(pos, h, npml, ofs):
    tab = np.zeros((len(pos), 5), np.int32)
    for k, (z, x) in enumerate(pos):
        t = subsourcekws(z, x, h, ofs)
        tab[k] = [t[0] + npml, t[1] + npml, t[2], t[3], t[4] if ofs else 0]
    return tab


# -- submodeling2.f90 set-up ---------------------------------------------------

def sponge_a(npml, n):
    d = np.ones(n + 2 * npml, F)
    d1 = np.ones(n + 2 * npml, F)
    for i in range(1, npml + 1):
        q = F(F(0.12) * F(npml - i))
        s, s1 = F(np.exp(-float(F(q * q)))), F(np.exp(-float(F(F(0.5) * F(q * q)))))
        d[i - 1], d1[i - 1] = s, s1
        j = npml - i + 1  # damp(npml+n+i) = spg(npml-i+1)
        qj = F(F(0.12) * F(npml - j))
        d[npml + n + i - 1] = F(np.exp(-float(F(qj * qj))))
        d1[npml + n + i - 1] = F(np.exp(-float(F(F(0.5) * F(qj * qj)))))
    return d, d1


def sponge_b(npml, n):
    d = np.ones(n + 2 * npml, F)
    d1 = np.ones(n + 2 * npml, F)
    for i in range(1, npml):
        q = F(F(0.12) * F(F(npml - 1 - i) + F(0.5)))
        d[i - 1] = F(np.exp(-float(F(q * q))))
        d1[i - 1] = F(np.exp(-float(F(F(0.5) * F(q * q)))))
    for i in range(1, npml + 1):
        q = F(F(0.12) * F(F(i - 1) + F(0.5)))
        d[npml + n + i - 1] = F(np.exp(-float(F(q * q))))
        d1[npml + n + i - 1] = F(np.exp(-float(F(F(0.5) * F(q * q)))))
    return d, d1


class Model:
    def __init__(self, vp, npml, h, dt, ofs):
        n1, n2 = vp.shape
        self.n1, self.n2, self.npml, self.ofs = n1, n2, npml, ofs
        self.n1e, self.n2e = n1 + 2 * npml, n2 + 2 * npml
        self.dt = F(dt)
        dtdx = F(F(dt) / F(h))
        ve = np.pad(vp.astype(F), npml, mode="edge")
        self.kap = (ve.astype(np.float64) ** 2).astype(F)
        d2a, d2a1 = sponge_a(npml, n2)
        d2b, d2b1 = sponge_b(npml, n2)
        d1a, d1a1 = sponge_a(npml, n1)
        d1b, d1b1 = sponge_b(npml, n1)
        self.d1a, self.d1b, self.d2a, self.d2b = d1a, d1b, d2a, d2b
        self.kw2 = (dtdx * self.kap) * d2a1[None, :]
        self.kw1 = (dtdx * self.kap) * d1a1[:, None]
        self.bw2 = np.broadcast_to((dtdx * F(1)) * d2b1[None, :], self.kap.shape).astype(F)
        self.bw1 = np.broadcast_to((dtdx * F(1)) * d1b1[:, None], self.kap.shape).astype(F)


def p_step(m, px, pz, vx, vz, off, sign):
    a, b = 2, m.n1e - off  # 0-based slice [2, n-off) for 1-based 3..n-off
    c, d = 2, m.n2e - off
    der2 = A0 * (vx[a:b, c:d] - vx[a:b, c - 1:d - 1]) + A1 * (vx[a:b, c + 1:d + 1] - vx[a:b, c - 2:d - 2])
    der1 = A0 * (vz[a:b, c:d] - vz[a - 1:b - 1, c:d]) + A1 * (vz[a + 1:b + 1, c:d] - vz[a - 2:b - 2, c:d])
    t2 = m.d2a[None, c:d] * px[a:b, c:d]
    t1 = m.d1a[a:b, None] * pz[a:b, c:d]
    if sign > 0:
        px[a:b, c:d] = t2 + m.kw2[a:b, c:d] * der2
        pz[a:b, c:d] = t1 + m.kw1[a:b, c:d] * der1
    else:
        px[a:b, c:d] = t2 - m.kw2[a:b, c:d] * der2
        pz[a:b, c:d] = t1 - m.kw1[a:b, c:d] * der1


def v_step(m, p, vx, vz, off, sign):
    a, b = 2, m.n1e - off
    c, d = 2, m.n2e - off
    der2 = A0 * (p[a:b, c + 1:d + 1] - p[a:b, c:d]) + A1 * (p[a:b, c + 2:d + 2] - p[a:b, c - 1:d - 1])
    der1 = A0 * (p[a + 1:b + 1, c:d] - p[a:b, c:d]) + A1 * (p[a + 2:b + 2, c:d] - p[a - 1:b - 1, c:d])
    t2 = m.d2b[None, c:d] * vx[a:b, c:d]
    t1 = m.d1b[a:b, None] * vz[a:b, c:d]
    if sign > 0:
        vx[a:b, c:d] = t2 + m.bw2[a:b, c:d] * der2
        vz[a:b, c:d] = t1 + m.bw1[a:b, c:d] * der1
    else:
        vx[a:b, c:d] = t2 - m.bw2[a:b, c:d] * der2
        vz[a:b, c:d] = t1 - m.bw1[a:b, c:d] * der1


def support(ix1, ix2, hi1, hi2):
    return (max(1 - ix1, -IRAD), min(hi1 - ix1, IRAD), max(1 - ix2, -IRAD), min(hi2 - ix2, IRAD))


def scatter(m, fld, w, tile, ix1, ix2, amp, sign):
    r1a, r1b, r2a, r2b = support(ix1, ix2, m.n1e, m.n2e)
    for i1 in range(r1a, r1b + 1):
        for i2 in range(r2a, r2b + 1):
            k1, k2 = ix1 + i1 - 1, ix2 + i2 - 1
            term = F(F(F(tile[i1 + 10, i2 + 10] * m.dt) * F(amp)) * w[k1, k2])
            fld[k1, k2] = F(fld[k1, k2] + term) if sign > 0 else F(fld[k1, k2] - term)


def gather(m, p, tile, ix1, ix2):
    r1a, r1b, r2a, r2b = support(ix1, ix2, m.n1e, m.n2e)
    acc = F(0)
    for i1 in range(r1a, r1b + 1):
        for i2 in range(r2a, r2b + 1):
            acc = F(acc + F(tile[i1 + 10, i2 + 10] * p[ix1 + i1 - 1, ix2 + i2 - 1]))
    return acc


def psum(m, px, pz):
    p = px + pz
    if m.ofs == 1:
        p[: m.npml + 1, :] = 0
    return p


def interior(m, f):
    return f[m.npml:m.npml + m.n1, m.npml:m.npml + m.n2].copy()


def forward(m, c1, nt, s, is5, ir):
    px, pz, vx, vz = (np.zeros((m.n1e, m.n2e), F) for _ in range(4))
    stile = kws_tile(c1, is5[2], is5[3], is5[4])
    rt = [kws_tile(c1, r[2], r[3], r[4]) for r in ir]
    sis = np.zeros((nt, len(ir)), F)
    wf = np.zeros((m.n1, m.n2, nt), F)
    for it in range(nt):
        p_step(m, px, pz, vx, vz, 2, +1)
        scatter(m, px, m.kap, stile, is5[0], is5[1], s[it], +1)
        p = psum(m, px, pz)
        wf[:, :, it] = interior(m, p)
        for r, rr in enumerate(ir):
            sis[it, r] = gather(m, p, rt[r], rr[0], rr[1])
        v_step(m, p, vx, vz, 2, +1)
        if m.ofs == 1:
            vz[m.npml - 1, :] = vz[m.npml, :]
    return sis, wf


def esource(m, c1, nt, res, ir, final):
    """final=False: esource_data (:880-1217); True: esource (:523-878)."""
    rt = [kws_tile(c1, r[2], r[3], r[4]) for r in ir]
    n1, n2, npml = m.n1, m.n2, m.npml
    sp = np.zeros((n1, n2, nt), F)
    svx = np.zeros((n1, n2, nt), F)
    svz = np.zeros((n1, n2, nt), F)
    px, pz, vx, vz = (np.zeros((m.n1e, m.n2e), F) for _ in range(4))
    for it in range(nt):
        p_step(m, px, pz, vx, vz, 3, -1)
        for r, rr in enumerate(ir):
            scatter(m, px, m.kap, rt[r], rr[0], rr[1], res[it, r], -1)
        p = psum(m, px, pz)
        sp[:, :, it] = interior(m, p)
        v_step(m, p, vx, vz, 3, -1)
        if m.ofs == 1:
            vz[npml - 1, :] = vz[npml, :]
        svx[:, :, it] = interior(m, vx)
        svz[:, :, it] = interior(m, vz)
    cost = F(0)
    if final:
        for v in sp.transpose(2, 1, 0).reshape(-1):
            cost = F(cost + F(F(0.5) * v) * v)
    px, pz, vx, vz = (np.zeros((m.n1e, m.n2e), F) for _ in range(4))
    sis = np.zeros((nt, len(ir)), F)
    wf = np.zeros((n1, n2, nt), F)
    lo, hi1, hi2 = (1, n1 - 1, n2 - 1) if final else (0, n1, n2)
    for it in range(nt):
        p_step(m, px, pz, vx, vz, 3, +1)
        ic = nt - 1 - it
        sl = (slice(npml + lo, npml + hi1), slice(npml + lo, npml + hi2))
        px[sl] = px[sl] + (F(-1) * m.dt * sp[lo:hi1, lo:hi2, ic]) * m.kap[sl]
        p = psum(m, px, pz)
        wf[:, :, it] = interior(m, p)
        for r, rr in enumerate(ir):
            sis[it, r] = gather(m, p, rt[r], rr[0], rr[1])
        v_step(m, p, vx, vz, 3, +1)
        si = (slice(npml, npml + n1), slice(npml, npml + n2))
        vx[si] = vx[si] + (F(-1) * m.dt * svx[:, :, ic]) * F(1)
        vz[si] = vz[si] + (F(-1) * m.dt * svz[:, :, ic]) * F(1)
        if m.ofs == 1:
            vz[npml - 1, :] = vz[npml, :]
    return sis, wf, cost


def resample(c1, n1, n2, npml, wf, ir):
    nt = wf.shape[2]
    sis = np.zeros((nt, len(ir)), F)
    for r, rr in enumerate(ir):
        t = kws_tile(c1, rr[2], rr[3], rr[4])
        ix1, ix2 = rr[0] - npml, rr[1] - npml
        r1a, r1b, r2a, r2b = support(ix1, ix2, n1, n2)
        for it in range(nt):
            acc = F(0)
            for i1 in range(r1a, r1b + 1):
                for i2 in range(r2a, r2b + 1):
                    acc = F(acc + F(t[i1 + 10, i2 + 10] * wf[ix1 + i1 - 1, ix2 + i2 - 1, it]))
            sis[it, r] = acc
    return sis


def filter_weights(nt, dt, flow, fhig, llow, lhig):
    """minresModule.f90:505-586: per-bin weights dmartin(1..nto+1)."""
    nto = next(s for s in (8 << k for k in range(14)) if nt <= s)
    fe = F(F(1) / F(dt))
    fmax = F(fe / F(2))
    flow, fhig, llow, lhig = F(flow), F(fhig), F(llow), F(lhig)
    if fhig > fmax:
        fhig, lhig = fmax, F(0)
    conv = int(F(F(nto) / fe))
    iflow = int(F(flow * F(conv))) + 1
    ifhig = int(F(fhig * F(conv))) + 1
    illow = int(F(llow * F(conv))) + 1
    ilhig = int(F(lhig * F(conv))) + 1
    if iflow - illow < 1 and iflow > 0:
        illow = iflow - 1
    if ifhig + ilhig > nto:
        ilhig = nto - ifhig

    def han(nf):
        pi = F(3.14159265)
        out = []
        for j in range(1, nf + 2):
            a = F(F(F(F(2) * pi) * F(j - 1)) / F(2 * nf))
            b = F(F(F(F(np.cos(float(a))) + F(1)) / F(2)) + F(0.000001))
            c = F(F(np.log(float(b))) * F(2))
            out.append(F(np.exp(float(c))))
        return out

    fm = np.zeros(nto + 1, F)
    if illow > 0:
        h1 = han(illow)
        for j in range(1, illow + 1):
            fm[iflow - j] = h1[j - 1]
    if ilhig > 0:
        h2 = han(ilhig)
        for j in range(1, ilhig + 1):
            fm[ifhig + j - 2] = h2[j - 1]
    fm[iflow - 1:ifhig] = 1
    return (fm + F(0.0001)).astype(np.float64), nto


def filmartin2d(data, dt, band):
    """Zero-padded real FFT, bin k scaled by w[k] (k < nto/2), the Nyquist bin by
    w[0] (the packed REALFT layout multiplies it with the DC weight), inverse."""
    nt, nr = data.shape
    w, nto = filter_weights(nt, dt, *band)
    half = nto // 2
    wk = np.concatenate([w[:half], w[:1]])
    spec = np.fft.rfft(data.astype(np.float64), n=nto, axis=0)
    out = np.fft.irfft(spec * wk[:, None], n=nto, axis=0)[:nt]
    return out.astype(F)


def main():
    rng = np.random.default_rng(20251203)
    c1 = kws_table1d()
    n1, n2, npml, h, dt, nt = 24, 36, 8, 10.0, 0.001, 96
    z = np.arange(n1)[:, None] * h
    vp = (1500.0 + 1.2 * z + 0 * np.arange(n2)[None, :]).astype(F)
    vp[14:, :] += F(300)
    vp = vp + rng.uniform(-20, 20, vp.shape).astype(F)
    f0 = 25.0
    tt = np.arange(nt) * dt - 1.2 / f0
    arg = (np.pi * f0 * tt) ** 2
    s = (((1 - 2 * arg) * np.exp(-arg)) / h ** 2).astype(F)
    src = [[15.0, 173.0]]
    recs = [[20.0, x] for x in (0.0, 44.0, 96.0, 131.0, 230.0, 349.0)]
    datum = [[150.0, x] for x in (5.0, 120.0, 260.0)]
    ofs = 1
    is5 = table(src, h, npml, ofs)[0]
    ir = table(recs, h, npml, ofs)
    ird = table(datum, h, npml, ofs)
    m = Model(vp, npml, h, dt, ofs)
    sis, wf = forward(m, c1, nt, s, is5, ir)
    res = rng.standard_normal((nt, len(ir))).astype(F)
    ggt, _, _ = esource(m, c1, nt, res, ir, final=False)
    esis, ewf, cost = esource(m, c1, nt, res, ir, final=True)
    rs = resample(c1, n1, n2, npml, wf + ewf, ird)
    band = (20.0, 120.0, 10.0, 40.0)
    filt = filmartin2d(sis, dt, band)
    tiles = np.stack([kws_tile(c1, a, b, f) for a, b, f in
                      ((51, 51, 0), (1, 100, 0), (37, 12, 9), (100, 3, 4), (63, 77, 10))])
    positions = np.array([[10.0, 4600.0, 20.0, 1], [20.0, 0.0, 20.0, 1], [8.0, 12.5, 4.0, 1],
                          [12.0, 9.99, 4.0, 0], [1000.0, 3333.3, 20.0, 1], [0.0, 0.0, 5.0, 1]])
    kws_pos = np.stack([subsourcekws(p[0], p[1], p[2], int(p[3])) for p in positions])
    sponge = np.stack([*sponge_a(npml, n1), *sponge_b(npml, n1)])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_small.npz")
    np.savez_compressed(
        out, vp=vp, npml=npml, h=h, dt=dt, nt=nt, ofs=ofs, s=s, is5=is5, ir=ir, ird=ird,
        res=res, kws1d=c1, tiles=tiles, tile_args=np.array([[51, 51, 0], [1, 100, 0],
                                                             [37, 12, 9], [100, 3, 4],
                                                             [63, 77, 10]]),
        kws_positions=positions, kws_tables=kws_pos, sponge=sponge,
        fwd_sis=sis, fwd_wf_slices=wf[:, :, ::16], ggt=ggt, es_sis=esis,
        es_wf_slices=ewf[:, :, ::16], es_cost=np.float32(cost), resampled=rs,
        band=np.array(band), filtered=filt)
    print("wrote", out)


if __name__ == "__main__":
    main()
