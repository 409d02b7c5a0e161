// ORACLE -- test infrastructure only.
//
// CPU restatement of the reference's DAW redatuming hot path
// (guogs93/Model-based-seismic-data-redatuming-with-DAWs, Fortran 90).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
// reference arms load this library, and only as the checker or the timed CPU
// baseline.  The product (the CUDA library in the package) never links it.
//
// Parity status: UNPINNED against the reference build.  The reference is
// Fortran 90 + MPI; no Fortran compiler exists in this image and the
// reference ships no golden vectors, known-answer tests or fixtures.  This
// restatement is cross-checked against an independent numpy restatement
// (tests/golden/make_golden.py, committed fixtures) and against physical and
// algebraic identities (tests/test_oracle_*.py).
//
// Arithmetic type T: float reproduces the reference's REAL arithmetic
// operation by operation (build with -ffp-contract=off so no FMA contraction
// changes a rounding); double is the FP64 accuracy oracle of the same method.
// Set-up constants (sponge profiles, Hicks coefficients, finite-difference
// weights) are always the reference's single-precision values, so the FP32 and
// FP64 runs differ only in propagation arithmetic.
//
// Array conventions follow the Fortran code: column-major, first index
// fastest; acquisition tables are (n,5) column-major int32 with the 1-based
// extended-grid indices built by subacqui (src/subacqui.f90:30-58).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>

namespace {

constexpr int kRad = 10;          // irad (src/kwsinc.f90:25)
constexpr int kNAlpha = 100;      // nalpha (src/kwsinc.f90:26)
constexpr int kTap = 2 * kRad + 1;
constexpr float kA0 = 1.125f;            // src/submodeling2.f90:48
constexpr float kA1 = -1.0f / 24.0f;     // src/submodeling2.f90:49
constexpr float kSpongeFac = 0.12f;      // xxfac, src/submodeling2.f90:35

// ---------------------------------------------------------------------------
// Hicks / Kaiser-windowed sinc (src/kwsinc.f90)
// ---------------------------------------------------------------------------

// Modified Bessel function I0, Abramowitz & Stegun 9.8.1 / 9.8.2 polynomial
// fits with the precisions of src/kwsinc.f90:612-635: argument and result
// single precision, polynomial evaluated in double.
float bessel_i0(float x) {
  if (std::fabs(x) < 3.75f) {
    float q = x / 3.75f;
    double y = (double)(q * q);
    double r = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 +
               y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))));
    return (float)r;
  }
  float ax = std::fabs(x);
  double y = (double)(3.75f / ax);
  float pre = std::exp(ax) / std::sqrt(ax);
  double r = (double)pre * (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 +
             y * (-0.157565e-2 + y * (0.916281e-2 + y * (-0.2057706e-1 +
             y * (0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))));
  return (float)r;
}

// 1-D monopole table c1[n + kRad][ia - 1], n in [-10,10], ia in [1,100]
// (src/kwsinc.f90:94-179, monopole branch; b = 14.18 for irad = 10).
struct Kws1D {
  float c[kTap][kNAlpha];
  Kws1D() {
    const float pi = 3.14159265359f;
    const float b = 14.18f;
    const float den = bessel_i0(b);
    for (int ia = 1; ia <= kNAlpha; ++ia) {
      float alpha = 0.5f - (float)(ia - 1) / (float)kNAlpha;
      for (int n = -kRad; n <= kRad; ++n) {
        float xn = (float)n + alpha;
        float v = 0.0f;
        if (std::fabs(xn) <= (float)kRad) {
          if (std::fabs(xn) > 1e-15f) {
            float arg = b * std::sqrt(1.0f - xn * xn / (float)(kRad * kRad));
            float kaiser = bessel_i0(arg) / den;
            v = kaiser * std::sin(pi * xn) / (pi * xn);
            if (std::fabs(v) < 1e-15f) v = 0.0f;
          } else {
            v = 1.0f;
          }
        }
        c[n + kRad][ia - 1] = v;
      }
    }
  }
};

const Kws1D& kws1d() {
  static const Kws1D t;
  return t;
}

// 2-D monopole tile for (ialpha1, ialpha2, nalpha_frees) with the free-surface
// anti-mirroring of src/kwsinc.f90:262-368.  tile[(i1+10) + 21*(i2+10)].
void kws_tile(int ia1, int ia2, int nfs, float* tile) {
  const Kws1D& t = kws1d();
  float tmp[kTap][kTap];  // tmp[i1][i2]
  for (int i2 = 0; i2 < kTap; ++i2)
    for (int i1 = 0; i1 < kTap; ++i1)
      tmp[i1][i2] = t.c[i2][ia2 - 1] * t.c[i1][ia1 - 1];
  for (int i2 = 0; i2 < kTap; ++i2)
    for (int i1 = 0; i1 < kTap; ++i1) tile[i1 + kTap * i2] = tmp[i1][i2];
  if (nfs > 0) {
    const int sym = -kRad + nfs;  // tile row on the free surface
    for (int i2 = 0; i2 < kTap; ++i2) {
      tile[(sym + kRad) + kTap * i2] = 0.0f;
      for (int k = 1; k <= nfs; ++k)
        tile[(sym + k + kRad) + kTap * i2] =
            tmp[sym + k + kRad][i2] - tmp[sym - k + kRad][i2];
    }
  }
}

// Nearest-integer of Fortran NINT (half away from zero).
inline int nint(float x) { return (int)std::lround(x); }

// src/kwsinc.f90:582-606 for ndim = 2.
void source_kws(const float xs[2], float dz, int ifs, int ix[2], int ia[2], int* nfs) {
  for (int d = 0; d < 2; ++d) {
    ix[d] = nint(xs[d] / dz) + 1;
    float x0 = (float)(ix[d] - 1) * dz;
    float alpha = (x0 - xs[d]) / dz;
    int a = nint((0.5f - alpha) * (float)kNAlpha) + 1;
    ia[d] = std::min(a, kNAlpha);
  }
  int f = kRad - nint(xs[0] / dz);
  f = std::max(f, 0);
  if (ifs == 0) f = 0;
  *nfs = f;
}

// ---------------------------------------------------------------------------
// Medium set-up (src/submodeling2.f90:1227-1393 and :54-113)
// ---------------------------------------------------------------------------

// Gaussian sponge profiles (cspongea, src/submodeling2.f90:1331-1353).
void sponge_a(int npml, int n, std::vector<float>& damp, std::vector<float>& damp1) {
  damp.assign(n + 2 * npml, 1.0f);
  damp1.assign(n + 2 * npml, 1.0f);
  std::vector<float> s(npml + 1), s1(npml + 1);
  for (int i = 1; i <= npml; ++i) {
    float x = (float)(npml - i);
    float q = kSpongeFac * x;
    s[i] = std::exp(-(q * q));
    s1[i] = std::exp(-(0.5f * (q * q)));
  }
  for (int i = 1; i <= npml; ++i) {
    damp[i - 1] = s[i];
    damp1[i - 1] = s1[i];
    damp[npml + n + i - 1] = s[npml - i + 1];
    damp1[npml + n + i - 1] = s1[npml - i + 1];
  }
}

// Half-cell-shifted sponge profiles (cspongeb, src/submodeling2.f90:1363-1393).
void sponge_b(int npml, int n, std::vector<float>& damp, std::vector<float>& damp1) {
  damp.assign(n + 2 * npml, 1.0f);
  damp1.assign(n + 2 * npml, 1.0f);
  for (int i = 1; i <= npml - 1; ++i) {
    float q = kSpongeFac * ((float)(npml - 1 - i) + 0.5f);
    damp[i - 1] = std::exp(-(q * q));
    damp1[i - 1] = std::exp(-(0.5f * (q * q)));
  }
  for (int i = 1; i <= npml; ++i) {
    float q = kSpongeFac * ((float)(i - 1) + 0.5f);
    damp[npml + n + i - 1] = std::exp(-(q * q));
    damp1[npml + n + i - 1] = std::exp(-(0.5f * (q * q)));
  }
}

template <typename T>
struct Medium {
  int n1, n2, npml, n1e, n2e, ofs;
  T dt, dtdx;
  std::vector<T> kap, kw1, kw2, bw1, bw2, bue;  // n1e*n2e
  std::vector<T> d1a, d1b, d2a, d2b;            // 1-D damping
};

// Edge-replicated extension of an n1 x n2 grid (submodext, :1281-1321).
std::vector<float> extend(const float* v, int n1, int n2, int npml) {
  const int n1e = n1 + 2 * npml, n2e = n2 + 2 * npml;
  std::vector<float> ve((size_t)n1e * n2e);
  for (int j = 0; j < n2e; ++j) {
    int sj = std::min(std::max(j - npml, 0), n2 - 1);
    for (int i = 0; i < n1e; ++i) {
      int si = std::min(std::max(i - npml, 0), n1 - 1);
      ve[i + (size_t)n1e * j] = v[si + (size_t)n1 * sj];
    }
  }
  return ve;
}

// Optional density of the media that later calls of the same thread build
// (n1 x n2, column-major), set by oracle_set_rho; empty = the reference's
// rho = 1.  Per thread, so concurrent oracle calls do not see each other's.
thread_local std::vector<float> g_rho;
thread_local int g_rho_n1 = 0, g_rho_n2 = 0;

template <typename T>
Medium<T> make_medium(const float* vp, int n1, int n2, int npml, float h, float dt, int ofs) {
  Medium<T> m;
  m.n1 = n1; m.n2 = n2; m.npml = npml; m.ofs = ofs;
  m.n1e = n1 + 2 * npml; m.n2e = n2 + 2 * npml;
  m.dt = (T)dt;
  m.dtdx = (T)dt / (T)h;
  std::vector<float> d1a, d1a1, d1b, d1b1, d2a, d2a1, d2b, d2b1;
  sponge_a(npml, n2, d2a, d2a1);
  sponge_b(npml, n2, d2b, d2b1);
  sponge_a(npml, n1, d1a, d1a1);
  sponge_b(npml, n1, d1b, d1b1);
  m.d1a.assign(d1a.begin(), d1a.end());
  m.d1b.assign(d1b.begin(), d1b.end());
  m.d2a.assign(d2a.begin(), d2a.end());
  m.d2b.assign(d2b.begin(), d2b.end());
  // Density is identically 1 in the reference (src/submodeling2.f90:93), so
  // kappa = vp^2 (product formed in double, :1235), buoyancy = 1 and its
  // staggered averages bu1 = bu2 = 1.  With a density set (oracle_set_rho),
  // substagger (:1227-1270) on the edge-replicated grids: kappa = rho vp^2 in
  // double, bu = 1/rho (1e10 where rho <= 0), bu1 = (bu(i1+1) + bu(i1))/2,
  // bu2 = (bu(i2+1) + bu(i2))/2.  The last row of bu1 and the last column of
  // bu2 (which the reference fills from a bu2 not yet computed, :1252) are
  // never read: v_step stops two points short of the edge.  They keep bu.
  std::vector<float> ve = extend(vp, n1, n2, npml);
  const size_t np = (size_t)m.n1e * m.n2e;
  const bool rho = !g_rho.empty() && g_rho_n1 == n1 && g_rho_n2 == n2;
  std::vector<float> re = rho ? extend(g_rho.data(), n1, n2, npml) : std::vector<float>();
  m.kap.resize(np); m.kw1.resize(np); m.kw2.resize(np);
  m.bw1.resize(np); m.bw2.resize(np); m.bue.assign(np, (T)1);
  std::vector<T> bu1(np, (T)1), bu2(np, (T)1);
  if (rho) {
    for (size_t k = 0; k < np; ++k) m.bue[k] = re[k] > 0.f ? (T)1 / (T)re[k] : (T)1e10;
    for (int j = 0; j < m.n2e; ++j)
      for (int i = 0; i < m.n1e; ++i) {
        const size_t k = i + (size_t)m.n1e * j;
        bu1[k] = i + 1 < m.n1e ? (T)0.5 * (m.bue[k + 1] + m.bue[k]) : m.bue[k];
        bu2[k] = j + 1 < m.n2e ? (T)0.5 * (m.bue[k + m.n1e] + m.bue[k]) : m.bue[k];
      }
  }
  for (int j = 0; j < m.n2e; ++j)
    for (int i = 0; i < m.n1e; ++i) {
      size_t k = i + (size_t)m.n1e * j;
      double v = (double)ve[k];
      T kap = rho ? (T)((double)re[k] * (v * v)) : (T)(v * v);
      m.kap[k] = kap;
      m.kw2[k] = m.dtdx * kap * (T)d2a1[j];
      m.kw1[k] = m.dtdx * kap * (T)d1a1[i];
      m.bw2[k] = m.dtdx * bu2[k] * (T)d2b1[j];
      m.bw1[k] = m.dtdx * bu1[k] * (T)d1b1[i];
    }
  return m;
}

// ---------------------------------------------------------------------------
// Time stepping (src/submodeling2.f90)
// ---------------------------------------------------------------------------

template <typename T>
struct Fields {
  std::vector<T> p, px, pz, vx, vz;
  explicit Fields(size_t np) : p(np, 0), px(np, 0), pz(np, 0), vx(np, 0), vz(np, 0) {}
  void zero() {
    std::fill(p.begin(), p.end(), (T)0); std::fill(px.begin(), px.end(), (T)0);
    std::fill(pz.begin(), pz.end(), (T)0); std::fill(vx.begin(), vx.end(), (T)0);
    std::fill(vz.begin(), vz.end(), (T)0);
  }
};

// Hicks tile support of one source/receiver clipped to index range [lo1,hi1] x
// [lo2,hi2] (1-based), offsets relative to (ix1, ix2).
struct Support { int r1min, r1max, r2min, r2max; };
inline Support clip(int ix1, int ix2, int hi1, int hi2) {
  Support s;
  s.r1min = std::max(1 - ix1, -kRad); s.r1max = std::min(hi1 - ix1, kRad);
  s.r2min = std::max(1 - ix2, -kRad); s.r2max = std::min(hi2 - ix2, kRad);
  return s;
}

struct Station {
  int ix1, ix2;  // 1-based indices (extended or physical, per caller)
  float tile[kTap * kTap];
};

std::vector<Station> stations(const int* tab, int n) {
  std::vector<Station> st(n);
  for (int r = 0; r < n; ++r) {
    st[r].ix1 = tab[r + 0 * n];
    st[r].ix2 = tab[r + 1 * n];
    kws_tile(tab[r + 2 * n], tab[r + 3 * n], tab[r + 4 * n], st[r].tile);
  }
  return st;
}

// Pressure half step over i1 in [3, n1e-off], i2 in [3, n2e-off]; sign +1 for
// forward/stage B (:148-155, :1108-1115), -1 for stage A (:1014-1021).
template <typename T>
void p_step(const Medium<T>& m, Fields<T>& f, int off, int sign) {
  const int n1e = m.n1e;
  const T a0 = (T)kA0, a1 = (T)kA1;
  for (int i2 = 3; i2 <= m.n2e - off; ++i2) {
    for (int i1 = 3; i1 <= n1e - off; ++i1) {
      size_t k = (i1 - 1) + (size_t)n1e * (i2 - 1);
      T der2 = a0 * (f.vx[k] - f.vx[k - n1e]) + a1 * (f.vx[k + n1e] - f.vx[k - 2 * n1e]);
      T der1 = a0 * (f.vz[k] - f.vz[k - 1]) + a1 * (f.vz[k + 1] - f.vz[k - 2]);
      if (sign > 0) {
        f.px[k] = m.d2a[i2 - 1] * f.px[k] + m.kw2[k] * der2;
        f.pz[k] = m.d1a[i1 - 1] * f.pz[k] + m.kw1[k] * der1;
      } else {
        f.px[k] = m.d2a[i2 - 1] * f.px[k] - m.kw2[k] * der2;
        f.pz[k] = m.d1a[i1 - 1] * f.pz[k] - m.kw1[k] * der1;
      }
    }
  }
}

// Particle-velocity half step (:229-236, :1067-1074, :1165-1172).
template <typename T>
void v_step(const Medium<T>& m, Fields<T>& f, int off, int sign) {
  const int n1e = m.n1e;
  const T a0 = (T)kA0, a1 = (T)kA1;
  for (int i2 = 3; i2 <= m.n2e - off; ++i2) {
    for (int i1 = 3; i1 <= n1e - off; ++i1) {
      size_t k = (i1 - 1) + (size_t)n1e * (i2 - 1);
      T der2 = a0 * (f.p[k + n1e] - f.p[k]) + a1 * (f.p[k + 2 * n1e] - f.p[k - n1e]);
      T der1 = a0 * (f.p[k + 1] - f.p[k]) + a1 * (f.p[k + 2] - f.p[k - 1]);
      if (sign > 0) {
        f.vx[k] = m.d2b[i2 - 1] * f.vx[k] + m.bw2[k] * der2;
        f.vz[k] = m.d1b[i1 - 1] * f.vz[k] + m.bw1[k] * der1;
      } else {
        f.vx[k] = m.d2b[i2 - 1] * f.vx[k] - m.bw2[k] * der2;
        f.vz[k] = m.d1b[i1 - 1] * f.vz[k] - m.bw1[k] * der1;
      }
    }
  }
}

// p = px + pz over the whole extended grid, then the free surface zeroes
// rows 1..npml+1 of p only (:183-189).
template <typename T>
void p_sum(const Medium<T>& m, Fields<T>& f) {
  const size_t np = f.p.size();
  for (size_t k = 0; k < np; ++k) f.p[k] = f.px[k] + f.pz[k];
  if (m.ofs == 1)
    for (int i2 = 0; i2 < m.n2e; ++i2)
      for (int i1 = 0; i1 <= m.npml; ++i1) f.p[i1 + (size_t)m.n1e * i2] = 0;
}

// vz(npml,:) = vz(npml+1,:) (:260-264).
template <typename T>
void vz_free_surface(const Medium<T>& m, Fields<T>& f) {
  if (m.ofs != 1) return;
  for (int i2 = 0; i2 < m.n2e; ++i2) {
    size_t k = (m.npml - 1) + (size_t)m.n1e * i2;
    f.vz[k] = f.vz[k + 1];
  }
}

// Hicks scatter of amp into field: f += ((c*dt)*amp)*w at the tile points
// clipped to the extended grid (:172-177, :1039-1044).  sign -1 subtracts.
template <typename T>
void hicks_scatter(const Medium<T>& m, const Station& s, T amp, int sign,
                   std::vector<T>& fld, const std::vector<T>& w) {
  Support sp = clip(s.ix1, s.ix2, m.n1e, m.n2e);
  for (int i1 = sp.r1min; i1 <= sp.r1max; ++i1)
    for (int i2 = sp.r2min; i2 <= sp.r2max; ++i2) {
      T c = (T)s.tile[(i1 + kRad) + kTap * (i2 + kRad)];
      size_t k = (s.ix1 + i1 - 1) + (size_t)m.n1e * (s.ix2 + i2 - 1);
      T term = c * m.dt * amp * w[k];
      if (sign > 0) fld[k] = fld[k] + term; else fld[k] = fld[k] - term;
    }
}

// Hicks gather of p at a station (:214-219): sequential sum, i1 outer.
template <typename T>
T hicks_gather(const Medium<T>& m, const Station& s, const std::vector<T>& p) {
  Support sp = clip(s.ix1, s.ix2, m.n1e, m.n2e);
  T acc = 0;
  for (int i1 = sp.r1min; i1 <= sp.r1max; ++i1)
    for (int i2 = sp.r2min; i2 <= sp.r2max; ++i2) {
      T c = (T)s.tile[(i1 + kRad) + kTap * (i2 + kRad)];
      acc = acc + c * p[(s.ix1 + i1 - 1) + (size_t)m.n1e * (s.ix2 + i2 - 1)];
    }
  return acc;
}

template <typename T>
void store_interior(const Medium<T>& m, const std::vector<T>& fld, T* dst) {
  for (int i2 = 0; i2 < m.n2; ++i2)
    for (int i1 = 0; i1 < m.n1; ++i1)
      dst[i1 + (size_t)m.n1 * i2] = fld[(i1 + m.npml) + (size_t)m.n1e * (i2 + m.npml)];
}

// submodeling (src/submodeling2.f90:11-288).  wavefield may be null.
template <typename T>
void forward(const Medium<T>& m, int nt, const float* s, int type_src, int type_rec,
             const int* is, const int* ir, int nr, T* sis, T* wavefield) {
  const size_t ni = (size_t)m.n1 * m.n2;
  Fields<T> f((size_t)m.n1e * m.n2e);
  std::vector<Station> rec = stations(ir, nr);
  int is1[5] = {is[0], is[1], is[2], is[3], is[4]};
  std::vector<Station> src = stations(is1, 1);
  std::fill(sis, sis + (size_t)nt * nr, (T)0);
  if (wavefield) std::fill(wavefield, wavefield + ni * nt, (T)0);
  for (int it = 1; it <= nt; ++it) {
    p_step(m, f, 2, +1);
    if (type_src == 0) hicks_scatter(m, src[0], (T)s[it - 1], +1, f.px, m.kap);
    p_sum(m, f);
    if (type_rec == 0) {
      if (wavefield) store_interior(m, f.p, wavefield + ni * (it - 1));
      for (int r = 0; r < nr; ++r) sis[(it - 1) + (size_t)nt * r] = hicks_gather(m, rec[r], f.p);
    }
    v_step(m, f, 2, +1);
    if (type_src == 1) hicks_scatter(m, src[0], (T)s[it - 1], +1, f.vz, m.bue);
    vz_free_surface(m, f);
  }
}

// Shared stage A of submodeling_adjoint_esource(_data): adjoint-signed
// stepping driven by res at the receivers, recording sp, svx, svz
// (:1010-1089 and :653-732).
template <typename T>
void stage_a(const Medium<T>& m, int nt, const T* res, const std::vector<Station>& rec,
             int nr, T* sp, T* svx, T* svz) {
  const size_t ni = (size_t)m.n1 * m.n2;
  Fields<T> f((size_t)m.n1e * m.n2e);
  for (int it = 1; it <= nt; ++it) {
    p_step(m, f, 3, -1);
    for (int r = 0; r < nr; ++r)
      hicks_scatter(m, rec[r], res[(it - 1) + (size_t)nt * r], -1, f.px, m.kap);
    p_sum(m, f);
    store_interior(m, f.p, sp + ni * (it - 1));
    v_step(m, f, 3, -1);
    vz_free_surface(m, f);
    store_interior(m, f.vx, svx + ni * (it - 1));
    store_interior(m, f.vz, svz + ni * (it - 1));
  }
}

// Stage B: forward stepping driven by the time-reversed stage-A history as a
// dense extended source (:1104-1194; :760-855 for the esource variant whose
// pressure source covers interior indices 2..n-1 only).  wavefieldp may be
// null.
template <typename T>
void stage_b(const Medium<T>& m, int nt, const T* sp, const T* svx, const T* svz,
             const std::vector<Station>& rec, int nr, int type_rec, bool esource,
             T* sis, T* wavefieldp) {
  const size_t ni = (size_t)m.n1 * m.n2;
  const int n1e = m.n1e, npml = m.npml;
  Fields<T> f((size_t)n1e * m.n2e);
  std::fill(sis, sis + (size_t)nt * nr, (T)0);
  const T ss = (T)-1;
  const int lo1 = esource ? 2 : 1, hi1 = esource ? m.n1 - 1 : m.n1;
  const int lo2 = esource ? 2 : 1, hi2 = esource ? m.n2 - 1 : m.n2;
  for (int it = 1; it <= nt; ++it) {
    p_step(m, f, 3, +1);
    const int ic = nt - it + 1;
    const T* spc = sp + ni * (ic - 1);
    for (int i2 = lo2; i2 <= hi2; ++i2)
      for (int i1 = lo1; i1 <= hi1; ++i1) {
        size_t k = (i1 + npml - 1) + (size_t)n1e * (i2 + npml - 1);
        f.px[k] = f.px[k] + ss * m.dt * spc[(i1 - 1) + (size_t)m.n1 * (i2 - 1)] * m.kap[k];
      }
    p_sum(m, f);
    if (type_rec == 0) {
      if (wavefieldp) store_interior(m, f.p, wavefieldp + ni * (it - 1));
      for (int r = 0; r < nr; ++r) sis[(it - 1) + (size_t)nt * r] = hicks_gather(m, rec[r], f.p);
    }
    v_step(m, f, 3, +1);
    const T* svxc = svx + ni * (ic - 1);
    const T* svzc = svz + ni * (ic - 1);
    for (int i2 = 1; i2 <= m.n2; ++i2)
      for (int i1 = 1; i1 <= m.n1; ++i1) {
        size_t k = (i1 + npml - 1) + (size_t)n1e * (i2 + npml - 1);
        f.vx[k] = f.vx[k] + ss * m.dt * svxc[(i1 - 1) + (size_t)m.n1 * (i2 - 1)] * m.bue[k];
      }
    for (int i2 = 1; i2 <= m.n2; ++i2)
      for (int i1 = 1; i1 <= m.n1; ++i1) {
        size_t k = (i1 + npml - 1) + (size_t)n1e * (i2 + npml - 1);
        f.vz[k] = f.vz[k] + ss * m.dt * svzc[(i1 - 1) + (size_t)m.n1 * (i2 - 1)] * m.bue[k];
      }
    vz_free_surface(m, f);
  }
}

// submodeling_adjoint_esource_data (:880-1217).
template <typename T>
void esource_data(const Medium<T>& m, int nt, const T* res, int type_rec, const int* ir,
                  int nr, T* sis) {
  const size_t ni = (size_t)m.n1 * m.n2;
  std::vector<Station> rec = stations(ir, nr);
  std::vector<T> sp(ni * nt), svx(ni * nt), svz(ni * nt);
  stage_a(m, nt, res, rec, nr, sp.data(), svx.data(), svz.data());
  stage_b(m, nt, sp.data(), svx.data(), svz.data(), rec, nr, type_rec, false, sis, (T*)nullptr);
}

// submodeling_adjoint_esource (:523-878); also returns the printed cost
// (sequential sum of 0.5*sp^2, :734-744).
template <typename T>
T esource(const Medium<T>& m, int nt, const T* res, int type_rec, const int* ir, int nr,
          T* sis, T* wavefieldp) {
  const size_t ni = (size_t)m.n1 * m.n2;
  std::vector<Station> rec = stations(ir, nr);
  std::vector<T> sp(ni * nt), svx(ni * nt), svz(ni * nt);
  stage_a(m, nt, res, rec, nr, sp.data(), svx.data(), svz.data());
  T cost = 0;
  for (size_t k = 0; k < ni * nt; ++k) cost = cost + (T)0.5 * sp[k] * sp[k];
  if (wavefieldp) std::fill(wavefieldp, wavefieldp + ni * nt, (T)0);
  stage_b(m, nt, sp.data(), svx.data(), svz.data(), rec, nr, type_rec, true, sis, wavefieldp);
  return cost;
}

// subwavefieldresample (src/subwavefieldresample.f90:1-41): Hicks gather of a
// physical-grid wavefield history, support clipped to the physical grid.
template <typename T>
void resample(int n1, int n2, int npml, int nt, const int* ir, int nr, const T* wavefield,
              T* sis) {
  std::vector<Station> rec = stations(ir, nr);
  const size_t ni = (size_t)n1 * n2;
  std::fill(sis, sis + (size_t)nt * nr, (T)0);
  for (int it = 1; it <= nt; ++it)
    for (int r = 0; r < nr; ++r) {
      const int ix1 = rec[r].ix1 - npml, ix2 = rec[r].ix2 - npml;
      Support sp = clip(ix1, ix2, n1, n2);
      T acc = 0;
      for (int i1 = sp.r1min; i1 <= sp.r1max; ++i1)
        for (int i2 = sp.r2min; i2 <= sp.r2max; ++i2) {
          T c = (T)rec[r].tile[(i1 + kRad) + kTap * (i2 + kRad)];
          acc = acc + c * wavefield[(ix1 + i1 - 1) + (size_t)n1 * (ix2 + i2 - 1) + ni * (it - 1)];
        }
      sis[(it - 1) + (size_t)nt * r] = acc;
    }
}

// ---------------------------------------------------------------------------
// MINRES (src/minresModule.f90:10-403, src/sublinearminres.f90:7-133)
// ---------------------------------------------------------------------------

template <typename T>
T dotp(const std::vector<T>& a, const std::vector<T>& b) {
  T s = 0;
  for (size_t i = 0; i < a.size(); ++i) s = s + a[i] * b[i];
  return s;
}

// blurring: A x = time-reverse(esource_data(x)) (minresModule.f90:363-403).
template <typename T>
void blurring(const Medium<T>& m, int nt, int type_rec, const int* ir, int nr,
              const std::vector<T>& x, std::vector<T>& y) {
  std::vector<T> tmp((size_t)nt * nr);
  esource_data(m, nt, x.data(), type_rec, ir, nr, tmp.data());
  for (int r = 0; r < nr; ++r)
    for (int j = 0; j < nt; ++j)
      y[j + (size_t)nt * r] = tmp[(nt - 1 - j) + (size_t)nt * r];
}

struct MinresLog {
  int32_t istop, itn, nlog;
  int32_t pad;
  double anorm, acond, rnorm, arnorm, ynorm, shift;
  // per iteration (<= capacity): itn, x(1), qrnorm/beta1, Anorm, Acond
  double* rows;  // 5 * capacity
  int32_t capacity;
};

// sublinearminres + MINRES with the reference's actual call: x0 = 0,
// precon = .false., checkA = .false. (sublinearminres.f90:37-76).
template <typename T>
void linear_minres(const Medium<T>& m, int nt, int type_rec, const int* ir, int nr,
                   const T* deltadr, float mu, int itnlim, float rtol_f, T* deltade,
                   MinresLog* log) {
  const size_t n = (size_t)nt * nr;
  std::vector<T> b(deltadr, deltadr + n);
  // fac = ||b|| / ||GG^T b|| * mu; datanorm sums i over nt outer (:117-133).
  std::vector<T> gb(n);
  esource_data(m, nt, b.data(), type_rec, ir, nr, gb.data());
  auto datanorm = [&](const std::vector<T>& d) {
    T s = 0;
    for (int i = 0; i < nt; ++i)
      for (int j = 0; j < nr; ++j) s = s + d[i + (size_t)nt * j] * d[i + (size_t)nt * j];
    return (T)std::sqrt(s);
  };
  const T fac = datanorm(b) / datanorm(gb) * (T)mu;
  const T shift = -fac;
  const T rtol = (T)rtol_f;
  const T eps = std::numeric_limits<T>::epsilon();
  const T zero = 0, one = 1, ten = 10;

  std::vector<T> x(n, 0), r1(n), r2(n), v(n), w(n), w1(n), w2(n), y(n);
  int istop = 0, itn = 0;
  T anorm = 0, acond = 0, rnorm = 0, ynorm = 0, arnorml = 0;
  if (log) { log->nlog = 0; log->shift = (double)shift; }
  y = b; r1 = b;
  T beta1 = dotp(b, y);
  T oldb, beta, dbar, epsln, qrnorm, phibar, rhs1, rhs2, tnorm2, ynorm2, cs, sn;
  T gmax = 0, gmin = 0;
  if (beta1 <= zero) {
    istop = beta1 < zero ? 8 : 0;
    goto done;
  }
  beta1 = std::sqrt(beta1);
  // Unused operator application kept as in the reference (:132-133).
  blurring(m, nt, type_rec, ir, nr, y, w);
  arnorml = std::sqrt(dotp(w, w));
  oldb = 0; beta = beta1; dbar = 0; epsln = 0; qrnorm = beta1; phibar = beta1;
  rhs1 = beta1; rhs2 = 0; tnorm2 = 0; ynorm2 = 0; cs = -one; sn = 0;
  std::fill(w.begin(), w.end(), zero);
  std::fill(w2.begin(), w2.end(), zero);
  r2 = r1;
  for (;;) {
    ++itn;
    T s = one / beta;
    for (size_t i = 0; i < n; ++i) v[i] = s * y[i];
    blurring(m, nt, type_rec, ir, nr, v, y);
    for (size_t i = 0; i < n; ++i) y[i] = y[i] - shift * v[i];
    if (itn >= 2) {
      T q = beta / oldb;
      for (size_t i = 0; i < n; ++i) y[i] = y[i] - q * r1[i];
    }
    T alfa = dotp(v, y);
    T q = alfa / beta;
    for (size_t i = 0; i < n; ++i) y[i] = y[i] - q * r2[i];
    r1 = r2;
    r2 = y;
    oldb = beta;
    beta = dotp(r2, y);
    if (beta < zero) { istop = 6; break; }
    beta = std::sqrt(beta);
    tnorm2 = tnorm2 + alfa * alfa + oldb * oldb + beta * beta;
    if (itn == 1) {
      if (beta / beta1 <= ten * eps) istop = -1;
      gmax = std::fabs(alfa);
      gmin = gmax;
    }
    T oldeps = epsln;
    T delta = cs * dbar + sn * alfa;
    T gbar = sn * dbar - cs * alfa;
    epsln = sn * beta;
    dbar = -cs * beta;
    T gamma = std::sqrt(gbar * gbar + beta * beta);
    cs = gbar / gamma;
    sn = beta / gamma;
    T phi = cs * phibar;
    phibar = sn * phibar;
    T denom = one / gamma;
    for (size_t i = 0; i < n; ++i) {
      w1[i] = w2[i];
      w2[i] = w[i];
      w[i] = (v[i] - oldeps * w1[i] - delta * w2[i]) * denom;
      x[i] = x[i] + phi * w[i];
    }
    gmax = std::max(gmax, gamma);
    gmin = std::min(gmin, gamma);
    T z = rhs1 / gamma;
    ynorm2 = z * z + ynorm2;
    rhs1 = rhs2 - delta * z;
    rhs2 = -epsln * z;
    anorm = std::sqrt(tnorm2);
    ynorm = std::sqrt(ynorm2);
    qrnorm = phibar;
    T rnorml = rnorm;
    rnorm = qrnorm;
    T rootl = std::sqrt(gbar * gbar + dbar * dbar);
    arnorml = rnorml * rootl;
    acond = gmax / gmin;
    if (istop == 0) {
      if (itn >= itnlim) istop = 5;
      if (qrnorm / beta1 <= rtol) istop = 1;
    }
    if (log && log->nlog < log->capacity) {
      double* row = log->rows + 5 * (size_t)log->nlog;
      row[0] = itn; row[1] = (double)x[0]; row[2] = (double)(qrnorm / beta1);
      row[3] = (double)anorm; row[4] = (double)acond;
      log->nlog++;
    }
    if (istop != 0) break;
  }
done:
  std::copy(x.begin(), x.end(), deltade);
  if (log) {
    log->istop = istop; log->itn = itn; log->anorm = (double)anorm;
    log->acond = (double)acond; log->rnorm = (double)rnorm;
    log->arnorm = (double)arnorml; log->ynorm = (double)ynorm;
  }
}

// ---------------------------------------------------------------------------
// filmartin2d (src/minresModule.f90:486-632) with the Numerical-Recipes real
// FFT of src/libfourier.f90:199-331, keeping its single-precision temporaries
// (implicitly typed REAL C1, C2, H1R, H1I, H2R, H2I, WRS, WIS).
// ---------------------------------------------------------------------------

// Complex radix-2 FFT on interleaved data[0..2nn) (four2, libfourier.f90:282-331).
void four2(double* data, int nn, int isign) {
  const int n = 2 * nn;
  int j = 1;
  for (int i = 1; i <= n; i += 2) {
    if (j > i) {
      std::swap(data[j - 1], data[i - 1]);
      std::swap(data[j], data[i]);
    }
    int m = n / 2;
    while (m >= 2 && j > m) { j -= m; m /= 2; }
    j += m;
  }
  int mmax = 2;
  while (n > mmax) {
    const int istep = 2 * mmax;
    const double theta = 6.28318530717959 / (double)(isign * mmax);
    const double st = std::sin(0.5 * theta);
    const double wpr = -2.0 * st * st, wpi = std::sin(theta);
    double wr = 1.0, wi = 0.0;
    for (int m = 1; m <= mmax; m += 2) {
      for (int i = m; i <= n; i += istep) {
        const int jj = i + mmax;
        double tr = wr * data[jj - 1] - wi * data[jj];
        double ti = wr * data[jj] + wi * data[jj - 1];
        data[jj - 1] = data[i - 1] - tr;
        data[jj] = data[i] - ti;
        data[i - 1] = data[i - 1] + tr;
        data[i] = data[i] + ti;
      }
      double wt = wr;
      wr = wr * wpr - wi * wpi + wr;
      wi = wi * wpr + wt * wpi + wi;
    }
    mmax = istep;
  }
}

// REALFT2S (libfourier.f90:199-276); isign1 = 2 forward, else inverse.
void realft2s(int n1, int isign1, double* data, double* datai, double* buf) {
  const int n = n1 / 2;
  const int isign = (isign1 == 2) ? 1 : -1;
  double theta = 3.141592653589793 / (double)n;
  const float c1 = 0.5f;
  float c2;
  if (isign == -1) {
    for (int i = 0; i < n; ++i) buf[i] = data[i];
    for (int k = 0; k < n; ++k) { data[2 * k] = buf[k]; data[2 * k + 1] = datai[k]; }
  }
  if (isign == 1) {
    c2 = -0.5f;
    four2(data, n, +1);
  } else {
    c2 = 0.5f;
    theta = -theta;
  }
  const double sh = std::sin(0.5 * theta);
  const double wpr = -2.0 * sh * sh, wpi = std::sin(theta);
  double wr = 1.0 + wpr, wi = wpi;
  const int n2p3 = 2 * n + 3;
  for (int i = 2; i <= n / 2; ++i) {
    const int i1 = 2 * i - 1, i2 = i1 + 1, i3 = n2p3 - i2, i4 = i3 + 1;
    const float wrs = (float)wr, wis = (float)wi;
    const float h1r = (float)((double)c1 * (data[i1 - 1] + data[i3 - 1]));
    const float h1i = (float)((double)c1 * (data[i2 - 1] - data[i4 - 1]));
    const float h2r = (float)((double)(-c2) * (data[i2 - 1] + data[i4 - 1]));
    const float h2i = (float)((double)c2 * (data[i1 - 1] - data[i3 - 1]));
    data[i1 - 1] = (double)(h1r + wrs * h2r - wis * h2i);
    data[i2 - 1] = (double)(h1i + wrs * h2i + wis * h2r);
    data[i3 - 1] = (double)(h1r - wrs * h2r + wis * h2i);
    data[i4 - 1] = (double)(-h1i + wrs * h2i + wis * h2r);
    const double wt = wr;
    wr = wr * wpr - wi * wpi + wr;
    wi = wi * wpr + wt * wpi + wi;
  }
  if (isign == 1) {
    const float h1r = (float)data[0];
    data[0] = (double)h1r + data[1];
    data[1] = (double)h1r - data[1];
  } else {
    const float h1r = (float)data[0];
    data[0] = (double)c1 * ((double)h1r + data[1]);
    data[1] = (double)c1 * ((double)h1r - data[1]);
    four2(data, n, -1);
  }
  if (isign == 1) {
    for (int k = 0; k < n; ++k) { datai[k] = data[2 * k + 1]; data[k] = data[2 * k]; }
  } else {
    for (int i = 0; i < 2 * n; ++i) data[i] = data[i] / (double)(float)n;
  }
}

// Hanning branch (sphanning, minresModule.f90:619-632); han[0..nf].
void sphanning(float* han, int nf, int nord) {
  const float pi = 3.14159265f;
  for (int j = 1; j <= nf + 1; ++j) {
    float a = 2.0f * pi * (float)(j - 1) / (float)(2 * nf);
    float b = (std::cos(a) + 1.0f) / 2.0f + 0.000001f;
    float c = std::log(b) * (float)nord;
    han[j - 1] = std::exp(c);
  }
}

// Returns 0 on success, -1 if nt exceeds the largest transform (65536).
int filmartin2d(const float* in, int nr, int nt, float dt, float* flow, float* fhig,
                float* llow, float* lhig, float* out, int* nto_out) {
  static const int sizes[] = {8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096,
                              8192, 16384, 32768, 65536};
  int nto = 0;
  for (int s : sizes) if (nt <= s) { nto = s; break; }
  if (nto == 0) return -1;
  if (nto_out) *nto_out = nto;
  const int nord = 2, nf = nto;
  const float fe = 1.0f / dt;
  const float fmax = fe / 2.0f;
  if (*fhig > fmax) { *fhig = fmax; *lhig = 0.0f; }
  const int conv = (int)((float)nto / fe);
  const int iflow = (int)(*flow * (float)conv) + 1;
  const int ifhig = (int)(*fhig * (float)conv) + 1;
  int illow = (int)(*llow * (float)conv) + 1;
  int ilhig = (int)(*lhig * (float)conv) + 1;
  if (iflow - illow < 1 && iflow > 0) illow = iflow - 1;
  if (ifhig + ilhig > nf) ilhig = nf - ifhig;
  std::vector<float> fm(nf + 1, 0.0f);
  if (illow > 0) {
    std::vector<float> han(illow + 1);
    sphanning(han.data(), illow, nord);
    for (int j = 1; j <= illow; ++j) fm[iflow - j] = han[j - 1];
  }
  if (ilhig > 0) {
    std::vector<float> han(ilhig + 1);
    sphanning(han.data(), ilhig, nord);
    for (int j = 1; j <= ilhig; ++j) fm[ifhig + j - 2] = han[j - 1];
  }
  for (int j = iflow; j <= ifhig; ++j) fm[j - 1] = 1.0f;
  std::vector<double> dm(nf + 1);
  for (int j = 0; j <= nf; ++j) dm[j] = (double)(fm[j] + 0.0001f);
  std::vector<double> pr(nto), pi(nto), buf(nto);
  for (int r = 0; r < nr; ++r) {
    std::fill(pi.begin(), pi.end(), 0.0);
    std::fill(pr.begin(), pr.end(), 0.0);
    for (int j = 0; j < nt; ++j) pr[j] = (double)in[j + (size_t)nt * r];
    realft2s(nto, 2, pr.data(), pi.data(), buf.data());
    for (int j = 0; j < nto; ++j) { pr[j] *= dm[j]; pi[j] *= dm[j]; }
    realft2s(nto, 1, pr.data(), pi.data(), buf.data());
    for (int j = 0; j < nt; ++j) out[j + (size_t)nt * r] = (float)pr[j];
  }
  return 0;
}

// Filter coefficients as used per spectral bin (for product parity tests).
int filmartin_weights(int nt, float dt, float flow, float fhig, float llow, float lhig,
                      double* w /* nto+1 */, int* nto_out) {
  static const int sizes[] = {8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096,
                              8192, 16384, 32768, 65536};
  int nto = 0;
  for (int s : sizes) if (nt <= s) { nto = s; break; }
  if (nto == 0) return -1;
  *nto_out = nto;
  if (!w) return 0;
  std::vector<float> in(nt, 0.0f), out(nt);
  // Recompute the same trapezoid by running the filter construction.
  const int nord = 2, nf = nto;
  const float fe = 1.0f / dt, fmax = fe / 2.0f;
  if (fhig > fmax) { fhig = fmax; lhig = 0.0f; }
  const int conv = (int)((float)nto / fe);
  const int iflow = (int)(flow * (float)conv) + 1;
  const int ifhig = (int)(fhig * (float)conv) + 1;
  int illow = (int)(llow * (float)conv) + 1;
  int ilhig = (int)(lhig * (float)conv) + 1;
  if (iflow - illow < 1 && iflow > 0) illow = iflow - 1;
  if (ifhig + ilhig > nf) ilhig = nf - ifhig;
  std::vector<float> fm(nf + 1, 0.0f);
  if (illow > 0) {
    std::vector<float> han(illow + 1);
    sphanning(han.data(), illow, nord);
    for (int j = 1; j <= illow; ++j) fm[iflow - j] = han[j - 1];
  }
  if (ilhig > 0) {
    std::vector<float> han(ilhig + 1);
    sphanning(han.data(), ilhig, nord);
    for (int j = 1; j <= ilhig; ++j) fm[ifhig + j - 2] = han[j - 1];
  }
  for (int j = iflow; j <= ifhig; ++j) fm[j - 1] = 1.0f;
  for (int j = 0; j <= nf; ++j) w[j] = (double)(fm[j] + 0.0001f);
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points (ctypes).  Suffix _f32: reference arithmetic; _f64: FP64.
// ---------------------------------------------------------------------------

extern "C" void oracle_set_rho(const float* rho, int n1, int n2) {
  if (!rho || n1 <= 0 || n2 <= 0) {
    g_rho.clear();
    g_rho_n1 = g_rho_n2 = 0;
    return;
  }
  g_rho.assign(rho, rho + (size_t)n1 * n2);
  g_rho_n1 = n1;
  g_rho_n2 = n2;
}

extern "C" {

void oracle_kws_tile(int ia1, int ia2, int nfs, float* tile) { kws_tile(ia1, ia2, nfs, tile); }

void oracle_kws_table1d(float* c /* 21 x 100, n fastest */) {
  const Kws1D& t = kws1d();
  for (int ia = 0; ia < kNAlpha; ++ia)
    for (int n = 0; n < kTap; ++n) c[n + kTap * ia] = t.c[n][ia];
}

float oracle_bessi0(float x) { return bessel_i0(x); }

void oracle_subsourcekws(float z, float x, float dz, int ifs, int* out5) {
  float xs[2] = {z, x};
  int ix[2], ia[2], nfs;
  source_kws(xs, dz, ifs, ix, ia, &nfs);
  out5[0] = ix[0]; out5[1] = ix[1]; out5[2] = ia[0]; out5[3] = ia[1]; out5[4] = nfs;
}

void oracle_sponges(int npml, int n, float* a, float* a1, float* b, float* b1) {
  std::vector<float> d, d1;
  sponge_a(npml, n, d, d1);
  std::copy(d.begin(), d.end(), a); std::copy(d1.begin(), d1.end(), a1);
  sponge_b(npml, n, d, d1);
  std::copy(d.begin(), d.end(), b); std::copy(d1.begin(), d1.end(), b1);
}

#define ORACLE_FORWARD(SUF, T)                                                              \
  void oracle_submodeling_##SUF(const float* vp, int n1, int n2, int npml, float h, int ofs, \
                                int nt, float dt, const float* s, int type_src,             \
                                int type_rec, const int* is, const int* ir, int nr, T* sis, \
                                T* wavefield) {                                             \
    Medium<T> m = make_medium<T>(vp, n1, n2, npml, h, dt, ofs);                             \
    forward(m, nt, s, type_src, type_rec, is, ir, nr, sis, wavefield);                      \
  }
ORACLE_FORWARD(f32, float)
ORACLE_FORWARD(f64, double)

#define ORACLE_ESD(SUF, T)                                                                   \
  void oracle_esource_data_##SUF(const float* vp, int n1, int n2, int npml, float h, int ofs, \
                                 int nt, float dt, const T* res, int type_rec, int nr,        \
                                 const int* ir, T* sis) {                                     \
    Medium<T> m = make_medium<T>(vp, n1, n2, npml, h, dt, ofs);                              \
    esource_data(m, nt, res, type_rec, ir, nr, sis);                                         \
  }
ORACLE_ESD(f32, float)
ORACLE_ESD(f64, double)

#define ORACLE_ES(SUF, T)                                                                    \
  double oracle_esource_##SUF(const float* vp, int n1, int n2, int npml, float h, int ofs,    \
                              int nt, float dt, const T* res, int type_rec, int nr,           \
                              const int* ir, T* sis, T* wavefieldp) {                         \
    Medium<T> m = make_medium<T>(vp, n1, n2, npml, h, dt, ofs);                              \
    return (double)esource(m, nt, res, type_rec, ir, nr, sis, wavefieldp);                   \
  }
ORACLE_ES(f32, float)
ORACLE_ES(f64, double)

#define ORACLE_RS(SUF, T)                                                                    \
  void oracle_resample_##SUF(int n1, int n2, int npml, int nt, const int* ir, int nr,         \
                             const T* wavefield, T* sis) {                                    \
    resample(n1, n2, npml, nt, ir, nr, wavefield, sis);                                      \
  }
ORACLE_RS(f32, float)
ORACLE_RS(f64, double)

#define ORACLE_MINRES(SUF, T)                                                                 \
  void oracle_minres_##SUF(const float* vp, int n1, int n2, int npml, float h, int ofs,        \
                           int nt, float dt, int type_rec, int nr, const int* ir,              \
                           const T* deltadr, float mu, int itnlim, float rtol, T* deltade,     \
                           int32_t* istat /*istop,itn,nlog*/, double* scal /*anorm,acond,     \
                           rnorm,arnorm,ynorm,shift*/, double* rows, int capacity) {           \
    Medium<T> m = make_medium<T>(vp, n1, n2, npml, h, dt, ofs);                               \
    MinresLog lg{};                                                                           \
    lg.rows = rows; lg.capacity = rows ? capacity : 0;                                        \
    linear_minres(m, nt, type_rec, ir, nr, deltadr, mu, itnlim, rtol, deltade, &lg);         \
    istat[0] = lg.istop; istat[1] = lg.itn; istat[2] = lg.nlog;                               \
    scal[0] = lg.anorm; scal[1] = lg.acond; scal[2] = lg.rnorm; scal[3] = lg.arnorm;          \
    scal[4] = lg.ynorm; scal[5] = lg.shift;                                                   \
  }
ORACLE_MINRES(f32, float)
ORACLE_MINRES(f64, double)

int oracle_filmartin2d(const float* in, int nr, int nt, float dt, float* flow, float* fhig,
                       float* llow, float* lhig, float* out) {
  return filmartin2d(in, nr, nt, dt, flow, fhig, llow, lhig, out, nullptr);
}

int oracle_filmartin_weights(int nt, float dt, float flow, float fhig, float llow, float lhig,
                             double* w, int* nto) {
  return filmartin_weights(nt, dt, flow, fhig, llow, lhig, w, nto);
}

// One mode-1 shot followed by the mode-2 resampling and filter at the new
// datum (src/sub_redatum_DAW.f90:82-145 then :238-240).  Outputs are T
// except `redatumed` (the filtered, single-precision mode-2 output).  The
// wavefield sums of :143 are formed explicitly (n1*n2*nt values).
#define ORACLE_SHOT(SUF, T)                                                                     \
  int oracle_daw_shot_##SUF(const float* vp, int n1, int n2, int npml, float h, int ofs,         \
                            int nt, float dt, const float* s, int type_src, int type_rec,        \
                            const int* is, const int* ir, int nr, const float* dobs, float mu,  \
                            int itnlim, float rtol, const int* ird, int nd, float flow,         \
                            float fhig, float llow, float lhig, T* datar, T* deltadr,           \
                            T* deltade, T* dataesc, T* datae, T* redatumed_raw,                  \
                            float* redatumed, int32_t* istat, double* scal) {                   \
    Medium<T> m = make_medium<T>(vp, n1, n2, npml, h, dt, ofs);                                \
    const size_t ni = (size_t)n1 * n2, nd_ = (size_t)nt * nr;                                    \
    std::vector<T> wr(ni * nt), we(ni * nt);                                                     \
    forward(m, nt, s, type_src, type_rec, is, ir, nr, datar, wr.data());                         \
    for (int r = 0; r < nr; ++r)                                                                 \
      for (int it = 0; it < nt; ++it)                                                            \
        deltadr[(nt - 1 - it) + (size_t)nt * r] =                                                \
            (T)dobs[it + (size_t)nt * r] - datar[it + (size_t)nt * r];                           \
    MinresLog lg{};                                                                              \
    linear_minres(m, nt, type_rec, ir, nr, deltadr, mu, itnlim, rtol, deltade, &lg);            \
    esource(m, nt, deltade, type_rec, ir, nr, dataesc, we.data());                               \
    for (size_t k = 0; k < nd_; ++k) datae[k] = datar[k] + dataesc[k];                           \
    for (size_t k = 0; k < ni * nt; ++k) wr[k] = wr[k] + we[k];                                  \
    resample(n1, n2, npml, nt, ird, nd, wr.data(), redatumed_raw);                               \
    std::vector<float> raw32((size_t)nt * nd);                                                   \
    for (size_t k = 0; k < raw32.size(); ++k) raw32[k] = (float)redatumed_raw[k];               \
    int rc = filmartin2d(raw32.data(), nd, nt, dt, &flow, &fhig, &llow, &lhig, redatumed,       \
                         nullptr);                                                               \
    istat[0] = lg.istop; istat[1] = lg.itn; istat[2] = lg.nlog;                                  \
    scal[0] = lg.anorm; scal[1] = lg.acond; scal[2] = lg.rnorm; scal[3] = lg.arnorm;             \
    scal[4] = lg.ynorm; scal[5] = lg.shift;                                                      \
    return rc;                                                                                   \
  }
ORACLE_SHOT(f32, float)
ORACLE_SHOT(f64, double)

// Bounded CPU-baseline sample: one truncated mode-1 shot in reference (FP32)
// arithmetic with `iters` MINRES iterations and no file output; returns the
// number of extended-grid point updates performed so callers can scale.
double oracle_baseline_sample(const float* vp, int n1, int n2, int npml, float h, int ofs,
                              int nt, float dt, const float* s, const int* is, const int* ir,
                              int nr, const float* dobs, float mu, int iters) {
  Medium<float> m = make_medium<float>(vp, n1, n2, npml, h, dt, ofs);
  const size_t nd_ = (size_t)nt * nr;
  std::vector<float> datar(nd_), deltadr(nd_), deltade(nd_), dataesc(nd_);
  forward(m, nt, s, 0, 0, is, ir, nr, datar.data(), (float*)nullptr);
  for (int r = 0; r < nr; ++r)
    for (int it = 0; it < nt; ++it)
      deltadr[(nt - 1 - it) + (size_t)nt * r] = dobs[it + (size_t)nt * r] - datar[it + (size_t)nt * r];
  MinresLog lg{};
  linear_minres(m, nt, 0, ir, nr, deltadr.data(), mu, iters, 0.0f, deltade.data(), &lg);
  esource(m, nt, deltade.data(), 0, ir, nr, dataesc.data(), (float*)nullptr);
  const double sims = 1.0 + 2.0 + 2.0 + 2.0 * lg.itn + 2.0;
  return sims * (double)nt * (double)m.n1e * (double)m.n2e;
}

}  // extern "C"
