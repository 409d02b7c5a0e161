// Host-side Hicks (Kaiser-windowed sinc) coefficients and the reference's
// input formats: redatum.par and the acquisition file.
//
// Hicks: G. J. Hicks, "Arbitrary source and receiver positioning in
// finite-difference schemes using Kaiser windowed sinc functions",
// Geophysics 67 (2002).  The reference tabulates 21x21x100x100x11
// coefficients (src/kwsinc.f90:212-378, ~194 MB per table); only the 21x21
// tile of each station is ever read, so the library builds per-station tiles
// with the same single-precision arithmetic instead.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "daw_internal.h"

namespace daw {
namespace {

// Modified Bessel I0 by the polynomial fits of Abramowitz & Stegun 9.8.1 and
// 9.8.2 (the fit BESSI0 uses, src/kwsinc.f90:612-635), with its precisions:
// single-precision argument and result, double-precision polynomial.
float i0_poly(float x) {
  if (std::fabs(x) < 3.75f) {
    const float t = x / 3.75f;
    const double y = (double)(t * t);
    return (float)(1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 +
                   y * (0.2659732 + y * (0.0360768 + y * 0.0045813))))));
  }
  const float ax = std::fabs(x);
  const double y = (double)(3.75f / ax);
  const float lead = std::exp(ax) / std::sqrt(ax);
  return (float)((double)lead * (0.39894228 + y * (0.01328592 + y * (0.00225319 +
                 y * (-0.00157565 + y * (0.00916281 + y * (-0.02057706 +
                 y * (0.02635537 + y * (-0.01647633 + y * 0.00392377)))))))));
}

// 1-D monopole weights w[n+10][ia-1] (src/kwsinc.f90:94-179): Kaiser window
// with b = 14.18 (bhicks0 for irad = 10) times sinc, sampled at offsets
// n + alpha with alpha = 0.5 - (ia-1)/100.
struct Weights1D {
  float w[kTap][kNAlpha];
  Weights1D() {
    const float pi = 3.14159265359f;
    const float b = 14.18f;
    const float i0b = i0_poly(b);
    for (int ia = 0; ia < kNAlpha; ++ia) {
      const float alpha = 0.5f - (float)ia / (float)kNAlpha;
      for (int n = -kRad; n <= kRad; ++n) {
        const float xn = (float)n + alpha;
        float v = 0.0f;
        if (std::fabs(xn) <= (float)kRad) {
          if (std::fabs(xn) > 1e-15f) {
            const float arg = b * std::sqrt(1.0f - xn * xn / (float)(kRad * kRad));
            const float win = i0_poly(arg) / i0b;
            v = win * std::sin(pi * xn) / (pi * xn);
            if (std::fabs(v) < 1e-15f) v = 0.0f;
          } else {
            v = 1.0f;
          }
        }
        w[n + kRad][ia] = v;
      }
    }
  }
};

const Weights1D& weights() {
  static const Weights1D tab;
  return tab;
}

int nearest(float v) { return (int)std::lround(v); }  // Fortran NINT

}  // namespace

void hicks_tile(int ia1, int ia2, int nfs, float* tile) {
  const Weights1D& W = weights();
  float base[kTap][kTap];  // [i1][i2], product of the two 1-D weights
  for (int i2 = 0; i2 < kTap; ++i2)
    for (int i1 = 0; i1 < kTap; ++i1) {
      base[i1][i2] = W.w[i2][ia2 - 1] * W.w[i1][ia1 - 1];
      tile[i1 + kTap * i2] = base[i1][i2];
    }
  if (nfs <= 0) return;
  // nfs grid nodes of the support lie above the free surface (row -10+nfs of
  // the tile): zero the surface node and subtract the mirror images of the
  // nodes above it from the nodes below it (src/kwsinc.f90:316-364).
  const int surf = nfs;  // tile row index (0-based) of the free surface
  for (int i2 = 0; i2 < kTap; ++i2) {
    tile[surf + kTap * i2] = 0.0f;
    for (int k = 1; k <= nfs; ++k)
      tile[(surf + k) + kTap * i2] = base[surf + k][i2] - base[surf - k][i2];
  }
}

void hicks_locate(float z, float x, float h, int ofs, int32_t out[5]) {
  const float pos[2] = {z, x};
  for (int d = 0; d < 2; ++d) {
    const int ix = nearest(pos[d] / h) + 1;
    const float alpha = ((float)(ix - 1) * h - pos[d]) / h;
    const int ia = nearest((0.5f - alpha) * (float)kNAlpha) + 1;
    out[d] = ix;
    out[2 + d] = std::min(ia, kNAlpha);
  }
  int above = kRad - nearest(z / h);
  out[4] = (ofs == 0) ? 0 : std::max(above, 0);
}

std::string shot_name(int i) {
  char buf[32];
  if (i < 0 || i >= 100000) return std::string();
  std::snprintf(buf, sizeof buf, "%05d", i);
  return buf;
}

// ---------------------------------------------------------------------------
// Fortran list-directed input (as gfortran reads redatum.par and the
// acquisition file): every READ starts a new record, items are separated by
// blanks or commas, a READ that needs more items continues on the next
// records, the rest of its last record is discarded, and '/' ends it.
// ---------------------------------------------------------------------------
namespace {

class ListReader {
 public:
  explicit ListReader(std::istream& in) : in_(in) {}
  // Reads `count` raw items (strings) for one READ statement.
  bool read(int count, std::vector<std::string>* items, std::string* err) {
    items->clear();
    std::string line;
    while ((int)items->size() < count) {
      if (!std::getline(in_, line)) {
        *err = "end of file while reading " + std::to_string(count) + " items";
        return false;
      }
      size_t i = 0;
      const size_t n = line.size();
      while (i < n && (int)items->size() < count) {
        while (i < n && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) ++i;
        if (i >= n) break;
        if (line[i] == '/') return true;  // slash terminates the READ
        std::string tok;
        if (line[i] == '\'' || line[i] == '"') {
          const char q = line[i++];
          while (i < n && line[i] != q) tok += line[i++];
          ++i;
        } else {
          while (i < n && line[i] != ' ' && line[i] != '\t' && line[i] != ',' &&
                 line[i] != '\r' && line[i] != '/')
            tok += line[i++];
        }
        while (i < n && (line[i] == ' ' || line[i] == '\t')) ++i;
        if (i < n && line[i] == ',') ++i;
        // repeat count r*c
        const size_t star = tok.find('*');
        if (star != std::string::npos && star > 0 &&
            std::all_of(tok.begin(), tok.begin() + star, ::isdigit)) {
          const int rep = std::atoi(tok.substr(0, star).c_str());
          const std::string val = tok.substr(star + 1);
          for (int r = 0; r < rep && (int)items->size() < count; ++r) items->push_back(val);
        } else {
          items->push_back(tok);
        }
      }
    }
    return true;
  }

 private:
  std::istream& in_;
};

bool to_int(const std::string& s, int* v) {
  if (s.empty()) return false;
  char* end = nullptr;
  long r = std::strtol(s.c_str(), &end, 10);
  if (*end != '\0') return false;
  *v = (int)r;
  return true;
}

bool to_real(const std::string& s, float* v) {
  if (s.empty()) return false;
  std::string t = s;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'e';  // Fortran double exponent letter
  char* end = nullptr;
  double r = std::strtod(t.c_str(), &end);
  if (*end != '\0') return false;
  *v = (float)r;
  return true;
}

}  // namespace

bool read_parfile(const std::string& path, ParFile* pf, std::string* err) {
  std::ifstream f(path);
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  ListReader rd(f);
  std::vector<std::string> it;
  auto fail = [&](const char* what) {
    *err = std::string("redatum.par: bad ") + what;
    return false;
  };
  // Fixed order of src/subreadpar.f90:9-21.
  if (!rd.read(1, &it, err) || !to_int(it[0], &pf->mode)) return fail("mode (line 1)");
  if (!rd.read(2, &it, err)) return fail("model names (line 2)");
  pf->name_true = it[0];
  pf->name_init = it[1];
  if (!rd.read(1, &it, err)) return fail("acquisition name (line 3)");
  pf->name_acqui = it[0];
  if (!rd.read(1, &it, err)) return fail("wavelet name (line 4)");
  pf->name_src = it[0];
  if (!rd.read(4, &it, err) || !to_real(it[0], &pf->flow) || !to_real(it[1], &pf->fhig) ||
      !to_real(it[2], &pf->llow) || !to_real(it[3], &pf->lhig))
    return fail("flow fhig llow lhig (line 5, four reals)");
  if (!rd.read(7, &it, err) || !to_int(it[0], &pf->n1) || !to_int(it[1], &pf->n2) ||
      !to_int(it[2], &pf->npml) || !to_real(it[3], &pf->h) || !to_int(it[4], &pf->nt) ||
      !to_real(it[5], &pf->dt) || !to_real(it[6], &pf->dto))
    return fail("n1 n2 npml h nt dt dto (line 6)");
  if (!rd.read(2, &it, err) || !to_int(it[0], &pf->type_src) || !to_int(it[1], &pf->type_rec))
    return fail("type_src type_rec (line 7)");
  if (!rd.read(1, &it, err) || !to_int(it[0], &pf->ofs)) return fail("ofs (line 8)");
  if (!rd.read(1, &it, err) || !to_real(it[0], &pf->mu)) return fail("mu (line 9)");
  if (!rd.read(1, &it, err) || !to_int(it[0], &pf->oio)) return fail("oio (line 10)");
  if (!rd.read(2, &it, err) || !to_real(it[0], &pf->error) || !to_real(it[1], &pf->maxiter))
    return fail("error maxiter (line 11)");
  return true;
}

bool read_acquisition(const std::string& path_in, float h, int npml, int ofs,
                      std::vector<int32_t>* src_tab, int* nsrc,
                      std::vector<int32_t>* rec_tab, int* nrec, std::string* err) {
  // The counts are read through the full name (main_redatum_DAW.f90:135-137),
  // the positions through a CHARACTER(len=26) dummy (subacqui.f90:22), i.e.
  // the first 26 characters of the name.
  std::ifstream f0(path_in);
  if (!f0) {
    *err = "cannot open acquisition file " + path_in;
    return false;
  }
  ListReader r0(f0);
  std::vector<std::string> it;
  if (!r0.read(2, &it, err) || !to_int(it[0], nsrc) || !to_int(it[1], nrec) || *nsrc < 0 ||
      *nrec < 0) {
    *err = "acquisition: bad 'nsrc nrec' header";
    return false;
  }
  std::string path = path_in;
  const size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? "" : path.substr(0, slash + 1);
  std::string base = slash == std::string::npos ? path : path.substr(slash + 1);
  if (base.size() > 26) base = base.substr(0, 26);
  path = dir + base;
  std::ifstream f(path);
  if (!f) {
    *err = "cannot open acquisition file " + path + " (name truncated to 26 characters)";
    return false;
  }
  ListReader rd(f);
  if (!rd.read(1, &it, err)) return false;  // header record skipped (subacqui.f90:28)
  auto read_set = [&](int n, std::vector<int32_t>* tab) {
    tab->assign((size_t)n * 5, 0);
    for (int i = 0; i < n; ++i) {
      float z, x;
      if (!rd.read(2, &it, err) || !to_real(it[0], &z) || !to_real(it[1], &x)) {
        *err = "acquisition: bad position record " + std::to_string(i + 1);
        return false;
      }
      int32_t o[5];
      hicks_locate(z, x, h, ofs, o);
      (*tab)[i + 0 * (size_t)n] = o[0] + npml;
      (*tab)[i + 1 * (size_t)n] = o[1] + npml;
      (*tab)[i + 2 * (size_t)n] = o[2];
      (*tab)[i + 3 * (size_t)n] = o[3];
      (*tab)[i + 4 * (size_t)n] = (ofs == 0) ? 0 : o[4];
    }
    return true;
  };
  return read_set(*nsrc, src_tab) && read_set(*nrec, rec_tab);
}

}  // namespace daw

extern "C" {
// Exposed for the Python host mirror (kwsinc2d/subsourcekws equivalents).
void daw_hicks_tile(int32_t ia1, int32_t ia2, int32_t nfs, float* tile) {
  daw::hicks_tile(ia1, ia2, nfs, tile);
}
void daw_hicks_locate(float z, float x, float h, int32_t ofs, int32_t* out5) {
  daw::hicks_locate(z, x, h, ofs, out5);
}
}
