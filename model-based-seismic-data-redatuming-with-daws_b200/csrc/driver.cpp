// Reference workflow on top of the C ABI: main_redatum_DAW + sub_redatum_DAW
// (src/main_redatum_DAW.f90:47-168, src/sub_redatum_DAW.f90:1-266) with the
// same input files, output file names and raw float32 formats.
//
// One extension, invisible to the reference: an optional 12th record of
// redatum.par naming a datum acquisition file.  The reference reads exactly
// 11 records, so the extra line does not change its behaviour; when present,
// mode 1 also writes dataobs_redatum_NNNNN.bin directly (the mode-2 result)
// from the datum gathers taken during the simulations, without storing the
// n1*n2*nt wavefields.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "daw_internal.h"

extern "C" void daw_internal_set_error(daw_handle* h, const char* msg);

namespace {

struct Fail {
  int code;
  std::string msg;
};

std::string join(const std::string& dir, const std::string& name) {
  if (dir.empty() || (!name.empty() && name[0] == '/')) return name;
  return dir + "/" + name;
}

void read_raw(const std::string& path, float* dst, size_t count) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Fail{DAW_ERR_IO, "cannot open " + path};
  f.read(reinterpret_cast<char*>(dst), (std::streamsize)(count * sizeof(float)));
  if ((size_t)f.gcount() != count * sizeof(float))
    throw Fail{DAW_ERR_IO, path + ": expected " + std::to_string(count) + " float32 values"};
}

void write_raw(const std::string& path, const float* src, size_t count) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) throw Fail{DAW_ERR_IO, "cannot create " + path};
  f.write(reinterpret_cast<const char*>(src), (std::streamsize)(count * sizeof(float)));
  if (!f) throw Fail{DAW_ERR_IO, "write failed: " + path};
}

// deltadr_/deltade_ files hold each trace in forward time (the arrays are
// time reversed in memory; sub_redatum_DAW.f90:109-113).
void write_reversed(const std::string& path, const std::vector<float>& a, int nt, int nr) {
  std::vector<float> t((size_t)nt * nr);
  for (int r = 0; r < nr; ++r)
    for (int j = 0; j < nt; ++j) t[j + (size_t)nt * r] = a[(nt - 1 - j) + (size_t)nt * r];
  write_raw(path, t.data(), t.size());
}

void check(daw_handle* h, int rc, const char* what) {
  if (rc != DAW_OK) throw Fail{rc, std::string(what) + ": " + daw_last_error(h)};
}

// MINRES log in the reference's layout (minresModule.f90:66-68, 321-358).
void write_minres_log(const std::string& path, int n, int itnlim, float rtol,
                      const daw_minres_info& info) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw Fail{DAW_ERR_IO, "cannot create " + path};
  std::fprintf(f, "\n\n Enter MINRES.       Solution of symmetric   Ax = b\n");
  std::fprintf(f, " n      =%7d     checkA =   F            precon =   F\n", n);
  std::fprintf(f, " itnlim =%7d     rtol   =%11.2E     shift  =%23.14E\n", itnlim, rtol, info.shift);
  std::fprintf(f, "\n\n     itn        x(1)          norm(r)   norm(A)   cond(A)\n");
  const double eps = 1.1920928955078125e-07;
  for (int i = 0; i < info.nlog; ++i) {
    const double* r = info.log + 5 * i;
    const int itn = (int)r[0];
    const bool last = (i == info.nlog - 1);
    bool prnt = n <= 40 || itn <= 10 || itn >= itnlim - 10 || itn % 10 == 0 || last ||
                r[4] >= 1.0e-2 / eps;
    if (prnt) {
      std::fprintf(f, "%8d%19.10E%10.2E%10.2E%10.2E\n", itn, r[1], r[2], r[3], r[4]);
      if (itn % 10 == 0) std::fprintf(f, "\n");
    }
  }
  static const char* msg[] = {"beta2 = 0.  If M = I, b and x are eigenvectors of A",
                              "beta1 = 0.  The exact solution is  x = 0           ",
                              "Requested accuracy achieved, as determined by rtol ",
                              "Reasonable accuracy achieved, given eps            ",
                              "x has converged to an eigenvector                  ",
                              "Acond has exceeded 0.1/eps                         ",
                              "The iteration limit was reached                    ",
                              "Aprod  does not define a symmetric matrix          ",
                              "Msolve does not define a symmetric matrix          ",
                              "Msolve does not define a pos-def preconditioner    "};
  std::fprintf(f, "\n Exit  MINRES.      istop =%3d              itn   =%8d\n", info.istop, info.itn);
  std::fprintf(f, " Exit  MINRES.      Anorm =%12.4E     Acond =%12.4E\n", info.anorm, info.acond);
  std::fprintf(f, " Exit  MINRES.      rnorm =%12.4E     ynorm =%12.4E     Arnorml=%12.4E\n",
               info.rnorm, info.ynorm, info.arnorm);
  const int k = info.istop + 1;
  std::fprintf(f, " Exit  MINRES.      %s\n", (k >= 0 && k < 10) ? msg[k] : "");
  std::fclose(f);
}

// Optional 12th record: datum acquisition file name.
std::string datum_record(const std::string& parpath) {
  std::ifstream f(parpath);
  std::string line;
  for (int i = 0; i < 11 && std::getline(f, line); ++i) {
  }
  if (!std::getline(f, line)) return std::string();
  size_t a = line.find_first_not_of(" \t'\"");
  if (a == std::string::npos || line[a] == '!') return std::string();
  size_t b = line.find_first_of(" \t,'\"!", a);
  return line.substr(a, b == std::string::npos ? std::string::npos : b - a);
}

}  // namespace

extern "C" int daw_run_parfile(daw_handle* h, const char* workdir_c, int32_t first, int32_t last) {
  if (!h) return DAW_ERR_ARG;
  try {
    const std::string dir = workdir_c ? workdir_c : ".";
    const std::string parpath = join(dir, "redatum.par");
    daw::ParFile pf;
    std::string err;
    if (!daw::read_parfile(parpath, &pf, &err)) throw Fail{DAW_ERR_IO, err};
    if (pf.mode < 0 || pf.mode > 3) throw Fail{DAW_ERR_ARG, "redatum.par: mode must be 0..3"};
    const int n1 = pf.n1, n2 = pf.n2, nt = pf.nt;
    if (n1 <= 0 || n2 <= 0 || nt <= 0 || pf.npml <= 0) throw Fail{DAW_ERR_ARG, "redatum.par: bad grid"};
    std::vector<float> s(nt), ctrue((size_t)n1 * n2), c0((size_t)n1 * n2);
    read_raw(join(dir, pf.name_src), s.data(), s.size());
    for (float& v : s) v = v / (pf.h * pf.h);  // main_redatum_DAW.f90:111
    std::vector<int32_t> src_tab, rec_tab;
    int nsrc = 0, nrec = 0;
    if (!daw::read_acquisition(join(dir, pf.name_acqui), pf.h, pf.npml, pf.ofs, &src_tab, &nsrc,
                               &rec_tab, &nrec, &err))
      throw Fail{DAW_ERR_IO, err};
    if (pf.mode == 0) read_raw(join(dir, pf.name_true), ctrue.data(), ctrue.size());
    if (pf.mode == 1 || pf.mode == 3) read_raw(join(dir, pf.name_init), c0.data(), c0.size());
    const std::vector<float>& model = (pf.mode == 0) ? ctrue : c0;
    std::vector<float> dummy((size_t)n1 * n2, 1500.0f);
    check(h, daw_set_model(h, pf.mode == 2 ? dummy.data() : model.data(), n1, n2, pf.npml, pf.h,
                           pf.dt, pf.ofs),
          "daw_set_model");
    // optional datum receivers for the fused mode-1 redatuming
    std::vector<int32_t> dsrc, dtab;
    int dn_src = 0, dn = 0;
    const std::string dname = datum_record(parpath);
    if (!dname.empty() && pf.mode == 1) {
      if (!daw::read_acquisition(join(dir, dname), pf.h, pf.npml, pf.ofs, &dsrc, &dn_src, &dtab,
                                 &dn, &err))
        throw Fail{DAW_ERR_IO, err};
      check(h, daw_set_datum(h, dtab.data(), dn), "daw_set_datum");
    }
    int a = first > 0 ? first : 1, b = last > 0 ? last : nsrc;
    b = std::min(b, nsrc);
    float band[4] = {pf.flow, pf.fhig, pf.llow, pf.lhig};
    const size_t nd = (size_t)nt * nrec, ni = (size_t)n1 * n2;
    // Without wavefield files (oio != 1), modes 0 and 1 run shots in batches
    // through the batched entry points; the files written are the same.
    if ((pf.mode == 0 || pf.mode == 1) && pf.oio != 1) {
      const int chunk = pf.mode == 0 ? 32 : 8;
      for (int c0 = a; c0 <= b; c0 += chunk) {
        const int cnt = std::min(b, c0 + chunk - 1) - c0 + 1;
        std::vector<daw_shot_desc> descs(cnt);
        std::vector<std::vector<float>> data(cnt), reds(cnt);
        std::vector<std::string> names(cnt);
        for (int k = 0; k < cnt; ++k) {
          const int isrc = c0 + k;
          names[k] = daw::shot_name(isrc);
          if (names[k].empty()) throw Fail{DAW_ERR_ARG, "i too big (subroutine subname)"};
          daw_shot_desc& d = descs[k];
          d = daw_shot_desc{};
          d.shot = isrc;
          d.nt = nt;
          d.s = s.data();
          for (int q = 0; q < 5; ++q) d.src_tab[q] = src_tab[(isrc - 1) + (size_t)nsrc * q];
          d.rec_tab = rec_tab.data();
          d.nrec = nrec;
          d.type_src = pf.type_src;
          d.type_rec = pf.type_rec;
          d.mu = pf.mu;
          d.maxiter = (int)pf.maxiter;
          d.rtol = pf.error;
          std::memcpy(d.band, band, sizeof band);
          data[k].resize(nd);
          if (pf.mode == 1) {
            read_raw(join(dir, "dataobs_org_" + names[k] + ".bin"), data[k].data(), nd);
            d.dobs = data[k].data();
          }
        }
        if (pf.mode == 0) {
          std::vector<float*> outs(cnt);
          for (int k = 0; k < cnt; ++k) outs[k] = data[k].data();
          check(h, daw_submodeling_shots(h, cnt, descs.data(), outs.data()),
                "daw_submodeling_shots");
          for (int k = 0; k < cnt; ++k)
            write_raw(join(dir, "dataobs_" + names[k] + ".bin"), data[k].data(), nd);
        } else {
          std::vector<daw_shot_out> outs(cnt);
          for (int k = 0; k < cnt; ++k) {
            outs[k] = daw_shot_out{};
            if (dn) {
              reds[k].resize((size_t)nt * dn);
              outs[k].redatumed = reds[k].data();
            }
          }
          check(h, daw_shots(h, cnt, descs.data(), outs.data()), "daw_shots");
          for (int k = 0; k < cnt; ++k)
            if (dn)
              write_raw(join(dir, "dataobs_redatum_" + names[k] + ".bin"), reds[k].data(),
                        reds[k].size());
        }
      }
      return DAW_OK;
    }
    for (int isrc = a; isrc <= b; ++isrc) {
      const std::string nm = daw::shot_name(isrc);
      if (nm.empty()) throw Fail{DAW_ERR_ARG, "i too big (subroutine subname)"};
      int32_t src5[5];
      for (int k = 0; k < 5; ++k) src5[k] = src_tab[(isrc - 1) + (size_t)nsrc * k];
      if (pf.mode == 0) {
        std::vector<float> dobs(nd), wf;
        if (pf.oio == 1) wf.resize(ni * nt);
        check(h, daw_submodeling(h, s.data(), nt, src5, pf.type_src, pf.type_rec, rec_tab.data(),
                                 nrec, dobs.data(), pf.oio == 1 ? wf.data() : nullptr),
              "daw_submodeling");
        write_raw(join(dir, "dataobs_" + nm + ".bin"), dobs.data(), nd);
        if (pf.oio == 1) write_raw(join(dir, "wavefield_obs" + nm + ".bin"), wf.data(), wf.size());
      } else if (pf.mode == 2) {
        std::vector<float> wf(ni * nt), sis(nd), out(nd);
        read_raw(join(dir, "wavefield_exd" + nm + ".bin"), wf.data(), wf.size());
        check(h, daw_wavefield_resample(h, wf.data(), nt, rec_tab.data(), nrec, sis.data()),
              "daw_wavefield_resample");
        check(h, daw_filmartin2d(h, sis.data(), nrec, nt, pf.dt, &band[0], &band[1], &band[2],
                                 &band[3], out.data()),
              "daw_filmartin2d");
        write_raw(join(dir, "dataobs_redatum_" + nm + ".bin"), out.data(), nd);
      } else {
        std::vector<float> dobs(nd);
        read_raw(join(dir, "dataobs_org_" + nm + ".bin"), dobs.data(), nd);
        std::vector<double> logrows(5 * (size_t)std::max(1, (int)pf.maxiter));
        daw_minres_info info{};
        info.log = logrows.data();
        info.log_capacity = (int)logrows.size() / 5;
        std::vector<float> datar(nd, 0.f), deltadr(nd), deltade(nd), dataesc(nd), datae(nd);
        std::vector<float> wr, we;
        if (pf.mode == 1) {
          wr.resize(ni * nt);
          check(h, daw_submodeling(h, s.data(), nt, src5, pf.type_src, pf.type_rec,
                                   rec_tab.data(), nrec, datar.data(), wr.data()),
                "daw_submodeling");
          if (pf.oio == 1) {
            write_raw(join(dir, "datar_" + nm + ".bin"), datar.data(), nd);
            write_raw(join(dir, "wavefield_ini" + nm + ".bin"), wr.data(), wr.size());
          }
          for (int r = 0; r < nrec; ++r)  // subresiduals.f90:12-16
            for (int it = 0; it < nt; ++it)
              deltadr[(nt - 1 - it) + (size_t)nt * r] = dobs[it + (size_t)nt * r] - datar[it + (size_t)nt * r];
        } else {  // mode 3: reversed observed data (sub_redatum_DAW.f90:175-179)
          for (int r = 0; r < nrec; ++r)
            for (int j = 0; j < nt; ++j)
              deltadr[(nt - 1 - j) + (size_t)nt * r] = dobs[j + (size_t)nt * r];
        }
        if (pf.oio == 1) write_reversed(join(dir, "deltadr_" + nm + ".bin"), deltadr, nt, nrec);
        check(h, daw_linear_minres(h, deltadr.data(), nt, pf.type_rec, rec_tab.data(), nrec,
                                   pf.mu, (int)pf.maxiter, pf.error, deltade.data(), &info),
              "daw_linear_minres");
        if (pf.oio == 1) {
          write_minres_log(join(dir, "MINRES_" + nm + ".txt"), (int)nd, (int)pf.maxiter, pf.error, info);
          write_reversed(join(dir, "deltade_" + nm + ".bin"), deltade, nt, nrec);
        }
        we.resize(ni * nt);
        double cost = 0;
        check(h, daw_esource(h, deltade.data(), nt, pf.type_rec, rec_tab.data(), nrec,
                             dataesc.data(), we.data(), &cost),
              "daw_esource");
        std::printf(" cost= %g\n", cost);
        if (pf.oio == 1) write_raw(join(dir, "dataesc_" + nm + ".bin"), dataesc.data(), nd);
        if (pf.mode == 1) {
          for (size_t k = 0; k < ni * nt; ++k) wr[k] = wr[k] + we[k];
          for (size_t k = 0; k < nd; ++k) datae[k] = datar[k] + dataesc[k];
          if (pf.oio == 1) {
            write_raw(join(dir, "datae_" + nm + ".bin"), datae.data(), nd);
            write_raw(join(dir, "wavefield_exd" + nm + ".bin"), wr.data(), wr.size());
          }
          if (dn) {
            std::vector<float> raw((size_t)nt * dn), red((size_t)nt * dn);
            check(h, daw_wavefield_resample(h, wr.data(), nt, dtab.data(), dn, raw.data()),
                  "daw_wavefield_resample");
            check(h, daw_filmartin2d(h, raw.data(), dn, nt, pf.dt, &band[0], &band[1], &band[2],
                                     &band[3], red.data()),
                  "daw_filmartin2d");
            write_raw(join(dir, "dataobs_redatum_" + nm + ".bin"), red.data(), red.size());
          }
        } else if (pf.oio == 1) {
          write_raw(join(dir, "wavefield_exd" + nm + ".bin"), we.data(), we.size());
        }
      }
    }
    return DAW_OK;
  } catch (const Fail& f) {
    daw_internal_set_error(h, f.msg.c_str());
    return f.code;
  } catch (const std::bad_alloc&) {
    daw_internal_set_error(h, "host allocation failed");
    return DAW_ERR_OOM;
  }
}
