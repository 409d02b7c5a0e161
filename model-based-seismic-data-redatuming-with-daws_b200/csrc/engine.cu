// libdaw_b200 engine: handle, model set-up, Hicks maps, the simulation
// drivers (plain port and fused path), the G G^T operator, the device MINRES
// driver, the mode-1 shot pipeline with on-the-fly datum extraction, and the
// C ABI of include/daw_b200.h.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "daw_internal.h"
#include "fused.cuh"
#include "kernels.cuh"

using namespace daw;

namespace daw {
void minres_log_f32(MinresDev<float>* d, double* log, const float* x, cudaStream_t st);
void minres_log_f64(MinresDev<double>* d, double* log, const float* x, cudaStream_t st);
void history_cost(const void* hist, int fp16, const unsigned* amax, int nt, int n1, int n2,
                  int inner_ld, int inner_off, size_t field_stride, double* out,
                  cudaStream_t st);
}  // namespace daw

namespace {

struct DawError {
  int code;
  std::string msg;
};

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess)                                                                 \
      throw DawError{DAW_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)};       \
  } while (0)

void check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw DawError{DAW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// Grow-only named device buffers owned by a handle.
struct Pool {
  std::map<std::string, DevBuf> bufs;
  size_t total = 0;
  void* get(const std::string& name, size_t bytes) {
    if (bytes == 0) bytes = 16;
    DevBuf& b = bufs[name];
    if (b.bytes < bytes) {
      if (b.p) {
        cudaFree(b.p);
        total -= b.bytes;
      }
      b.p = nullptr;
      b.bytes = 0;
      if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        throw DawError{DAW_ERR_OOM, "device allocation of " + std::to_string(bytes) +
                                        " bytes for '" + name + "' failed"};
      }
      b.bytes = bytes;
      total += bytes;
    }
    return b.p;
  }
  template <typename T>
  T* get_t(const std::string& name, size_t count) {
    return static_cast<T*>(get(name, count * sizeof(T)));
  }
  void release_prefix(const std::string& prefix) {
    for (auto it = bufs.begin(); it != bufs.end();) {
      if (it->first.compare(0, prefix.size(), prefix) == 0) {
        if (it->second.p) cudaFree(it->second.p);
        total -= it->second.bytes;
        it = bufs.erase(it);
      } else {
        ++it;
      }
    }
  }
  void clear() {
    for (auto& kv : bufs)
      if (kv.second.p) cudaFree(kv.second.p);
    bufs.clear();
    total = 0;
  }
};

// ---------------------------------------------------------------------------
// Host-side medium set-up (src/submodeling2.f90:54-113, 1227-1393).
// ---------------------------------------------------------------------------
const float kSponge = 0.12f;  // xxfac

// cspongea: exp(-(0.12 x)^2) over the npml cells of each side, x = npml-i.
void sponge_a(int npml, int n, std::vector<float>& d, std::vector<float>& d1) {
  d.assign(n + 2 * npml, 1.0f);
  d1.assign(n + 2 * npml, 1.0f);
  for (int i = 1; i <= npml; ++i) {
    const float q = kSponge * (float)(npml - i);
    const float v = std::exp(-(q * q)), v1 = std::exp(-(0.5f * (q * q)));
    d[i - 1] = v;
    d1[i - 1] = v1;
    d[npml + n + (npml - i + 1) - 1] = v;  // mirrored: damp(npml+n+j) = spg(npml-j+1)
    d1[npml + n + (npml - i + 1) - 1] = v1;
  }
}

// cspongeb: the half-cell-shifted profile of the staggered velocity grid.
void sponge_b(int npml, int n, std::vector<float>& d, std::vector<float>& d1) {
  d.assign(n + 2 * npml, 1.0f);
  d1.assign(n + 2 * npml, 1.0f);
  for (int i = 1; i <= npml - 1; ++i) {
    const float q = kSponge * ((float)(npml - 1 - i) + 0.5f);
    d[i - 1] = std::exp(-(q * q));
    d1[i - 1] = std::exp(-(0.5f * (q * q)));
  }
  for (int i = 1; i <= npml; ++i) {
    const float q = kSponge * ((float)(i - 1) + 0.5f);
    d[npml + n + i - 1] = std::exp(-(q * q));
    d1[npml + n + i - 1] = std::exp(-(0.5f * (q * q)));
  }
}

// Per-shot device context of the pipeline.
struct ShotCtx {
  int shot = 0, nt = 0, nr = 0, nd = 0;
  int type_src = 0, type_rec = 0;
  float mu = 0, rtol = 0;
  int maxiter = 0;
  float band[4] = {0, 0, 0, 0};
  int32_t src5[5] = {0, 0, 0, 0, 0};
  std::string tag;
  StationsDev rec, src;
  InjMapDev recmap, srcmap;
  float *d_s = nullptr, *d_dobs = nullptr, *d_datar = nullptr, *d_deltadr = nullptr;
  float *d_deltade = nullptr, *d_dataesc = nullptr, *d_datae = nullptr;
  float *d_redF = nullptr, *d_redE = nullptr, *d_red = nullptr, *d_redf = nullptr;
  float* d_wf = nullptr;
  float* d_ampT = nullptr;  // stage-A residual in step-major order [nt][nr]
  // simulation state: a block of 9 fields [px, pz, vx, vz, p, px2, pz2, vx2,
  // vz2]; the one-kernel-per-step path alternates between {px, pz, vx, vz}
  // (set 0) and {px2, pz2, vx2, vz2} (set 1), and `par` is the set that holds
  // the current state.
  float* state = nullptr;
  float *px = nullptr, *pz = nullptr, *vx = nullptr, *vz = nullptr, *p = nullptr;
  float *px2 = nullptr, *pz2 = nullptr, *vx2 = nullptr, *vz2 = nullptr;
  int par = 0;
  void set_state(float* s9, size_t ne) {
    state = s9;
    px = s9; pz = s9 + ne; vx = s9 + 2 * ne; vz = s9 + 3 * ne; p = s9 + 4 * ne;
    px2 = s9 + 5 * ne; pz2 = s9 + 6 * ne; vx2 = s9 + 7 * ne; vz2 = s9 + 8 * ne;
  }
  void* hist = nullptr;
  int hist_steps = 0;  // steps the history buffer holds
  // Checkpointed stage A (hist_win > 0): the history buffer holds a window of
  // hist_win steps; ckpt holds the states before windows 1 .. nwin-1 and st_b
  // stage B's own state.
  int hist_win = 0;
  float* ckpt = nullptr;
  float* st_b = nullptr;
  unsigned* amax = nullptr;
  double* d_cost = nullptr;
  // operator I/O for the current application
  const float* op_in = nullptr;
  float* op_out = nullptr;
  int op_reverse = 0;
  bool active = true;
  // MINRES
  float *x = nullptr, *y = nullptr, *v = nullptr, *r1 = nullptr, *r2 = nullptr;
  float *w = nullptr, *w1 = nullptr, *w2 = nullptr, *gb = nullptr;
  void* partials = nullptr;
  void* mdev = nullptr;
  double* dlog = nullptr;
  int log_cap = 0;
  daw_minres_info info{};
  double cost = 0;
};

}  // namespace

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
struct daw_handle {
  int device = 0;
  cudaStream_t st = nullptr;
  std::string err;
  Options opt;
  bool has_model = false;
  Grid g{};
  ModelDev md;
  Pool model_pool, pool;
  std::vector<int32_t> datum_tab;
  int ndatum = 0;
  StationsDev datum;
  daw_timing tim{};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // graphs: key -> exec
  std::map<std::string, cudaGraphExec_t> graphs;
  // staged shots (device-resident runs)
  std::vector<daw_shot_desc> staged;
  std::vector<std::vector<float>> staged_s, staged_dobs;
  std::vector<std::vector<int32_t>> staged_rec;
  std::vector<ShotCtx> staged_ctx;
  int staged_ready = 0;
  // TMA kernels: persistent grid sizes and the bounded-wait error flag
  int persist_p = 0, persist_v = 0;
  int persist_v_mode[8] = {};  // velocity kernel grid per (mode, FP16 history)
  unsigned* d_err = nullptr;
  // One-kernel-per-step path: SMs, resident CTAs per SM of each (mode, FP16,
  // tile width) [mode][fp16][tc == 32], the tile-queue counter and the
  // autotuned configurations by (mode, FP16, grid, shots) key.
  int sms = 0;
  int step_occ[4][2][2] = {};
  unsigned* d_qctr = nullptr;
  struct Tuned {
    int family;            // 0: split pressure / velocity kernels, 1: one kernel per step
    int tile_cols;         // columns per tile (the split kernels' tiles are 32 wide)
    int ctas_per_sm;       // CTAs per SM (split: of the pressure kernel)
    int ctas_per_sm_v;     // split: CTAs per SM of the velocity kernel
    int sub;               // split: shots per launch (the batch's time loops run in
                           // groups of `sub` shots); 0 = the whole batch
    float us_per_step;     // measured device time of one step per shot (0: not measured)
  };
  std::map<std::string, Tuned> tuned;
};

namespace {

void drop_graphs(daw_handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

void sync(daw_handle* h) {
  CK(cudaStreamSynchronize(h->st));
}

void upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
}
void download(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes && dst) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
}

void require_model(daw_handle* h) {
  if (!h->has_model) throw DawError{DAW_ERR_STATE, "no model: call daw_set_model first"};
  // a density other than 1 runs on the plain and the split TMA kernels only
  if (h->md.rbw1 && h->opt.fused && (h->opt.chunk != 0 || h->opt.step == 1))
    throw DawError{DAW_ERR_ARG,
                   "a model with density runs on the plain or the split TMA kernels "
                   "(DAW_OPT_CHUNK = 0, DAW_OPT_STEP_KERNEL != 1)"};
}

void check_table(const daw_handle* h, const int32_t* tab, int n, bool extended, const char* what) {
  if (n < 0 || (n > 0 && !tab)) throw DawError{DAW_ERR_ARG, std::string(what) + ": bad table"};
  for (int i = 0; i < n; ++i) {
    const int ix1 = tab[i], ix2 = tab[i + n], a1 = tab[i + 2 * n], a2 = tab[i + 3 * n],
              fs = tab[i + 4 * n];
    const int lo = extended ? 1 : 1 + h->g.npml;
    const int hi1 = extended ? h->g.n1e : h->g.n1 + h->g.npml;
    const int hi2 = extended ? h->g.n2e : h->g.n2 + h->g.npml;
    (void)lo;
    if (ix1 < 1 - kRad || ix1 > hi1 + kRad || ix2 < 1 - kRad || ix2 > hi2 + kRad || a1 < 1 ||
        a1 > kNAlpha || a2 < 1 || a2 > kNAlpha || fs < 0 || fs > kRad)
      throw DawError{DAW_ERR_ARG, std::string(what) + ": entry " + std::to_string(i + 1) +
                                      " out of range"};
  }
}

StationsDev make_stations(daw_handle* h, Pool& pool, const std::string& name, const int32_t* tab,
                          int n) {
  StationsDev s;
  s.n = n;
  if (n == 0) return s;
  std::vector<int> ix1(n), ix2(n);
  std::vector<float> tiles((size_t)n * kTile);
  for (int i = 0; i < n; ++i) {
    ix1[i] = tab[i];
    ix2[i] = tab[i + n];
    hicks_tile(tab[i + 2 * n], tab[i + 3 * n], tab[i + 4 * n], tiles.data() + (size_t)i * kTile);
  }
  s.ix1 = pool.get_t<int>(name + ".ix1", n);
  s.ix2 = pool.get_t<int>(name + ".ix2", n);
  s.tile = pool.get_t<float>(name + ".tile", (size_t)n * kTile);
  upload(s.ix1, ix1.data(), n * sizeof(int), h->st);
  upload(s.ix2, ix2.data(), n * sizeof(int), h->st);
  upload(s.tile, tiles.data(), tiles.size() * sizeof(float), h->st);
  sync(h);  // host vectors go out of scope
  return s;
}

// Gather-form injection map of stations `tab` on the extended grid.
InjMapDev make_map(daw_handle* h, Pool& pool, const std::string& name, const int32_t* tab, int n) {
  const Grid& g = h->g;
  struct E {
    long long pt;
    int sta;
    float c;
  };
  std::vector<E> es;
  es.reserve((size_t)n * kTile);
  std::vector<float> tile(kTile);
  for (int s = 0; s < n; ++s) {
    const int ix1 = tab[s], ix2 = tab[s + n];
    hicks_tile(tab[s + 2 * n], tab[s + 3 * n], tab[s + 4 * n], tile.data());
    const int r1a = std::max(1 - ix1, -kRad), r1b = std::min(g.n1e - ix1, kRad);
    const int r2a = std::max(1 - ix2, -kRad), r2b = std::min(g.n2e - ix2, kRad);
    for (int i1 = r1a; i1 <= r1b; ++i1)
      for (int i2 = r2a; i2 <= r2b; ++i2) {
        const long long pt = (long long)(ix1 + i1 - 1) + (long long)g.ld * (ix2 + i2 - 1);
        es.push_back({pt, s, tile[(i1 + kRad) + kTap * (i2 + kRad)]});
      }
  }
  std::stable_sort(es.begin(), es.end(), [](const E& a, const E& b) { return a.pt < b.pt; });
  std::vector<int> pt, ptr, sta;
  std::vector<float> coef;
  for (size_t i = 0; i < es.size(); ++i) {
    if (i == 0 || es[i].pt != es[i - 1].pt) {
      pt.push_back((int)es[i].pt);
      ptr.push_back((int)i);
    }
    sta.push_back(es[i].sta);
    coef.push_back(es[i].c);
  }
  ptr.push_back((int)es.size());
  // column bands
  std::vector<int> clo(g.n2e, INT_MAX), chi(g.n2e, -1), cbase(g.n2e, 0), rowptr;
  for (size_t q = 0; q < pt.size(); ++q) {
    const int c = pt[q] / g.ld, r = pt[q] % g.ld;
    clo[c] = std::min(clo[c], r);
    chi[c] = std::max(chi[c], r);
  }
  {
    size_t q = 0;
    for (int c = 0; c < g.n2e; ++c) {
      cbase[c] = (int)rowptr.size();
      if (chi[c] < clo[c]) continue;
      for (int r = clo[c]; r <= chi[c]; ++r) {
        // entries of (r, c) are those of touched point pt == r + ld*c
        const long long want = (long long)r + (long long)g.ld * c;
        while (q < pt.size() && pt[q] < want) ++q;
        if (q < pt.size() && pt[q] == want)
          rowptr.push_back(ptr[q]);
        else
          rowptr.push_back(q < pt.size() ? ptr[q] : ptr.back());
      }
    }
    rowptr.push_back(ptr.back());
  }
  // rowptr[i+1] must close row i: rebuild as explicit begin/end pairs.
  std::vector<int> rp;
  rp.reserve(rowptr.size());
  {
    size_t q = 0;
    int idx = 0;
    for (int c = 0; c < g.n2e; ++c) {
      if (chi[c] < clo[c]) continue;
      for (int r = clo[c]; r <= chi[c]; ++r, ++idx) {
        const long long want = (long long)r + (long long)g.ld * c;
        while (q < pt.size() && pt[q] < want) ++q;
        if (q < pt.size() && pt[q] == want) {
          rp.push_back(ptr[q]);
          rp.push_back(ptr[q + 1]);
        } else {
          rp.push_back(0);
          rp.push_back(0);
        }
      }
    }
  }
  // cbase indexes pairs
  {
    int idx = 0;
    for (int c = 0; c < g.n2e; ++c) {
      cbase[c] = idx;
      if (chi[c] >= clo[c]) idx += chi[c] - clo[c] + 1;
    }
  }
  InjMapDev m;
  m.npts = (int)pt.size();
  m.nent = (int)sta.size();
  m.pt = pool.get_t<int>(name + ".pt", std::max<size_t>(1, pt.size()));
  m.ptr = pool.get_t<int>(name + ".ptr", ptr.size());
  m.sta = pool.get_t<int>(name + ".sta", std::max<size_t>(1, sta.size()));
  m.coef = pool.get_t<float>(name + ".coef", std::max<size_t>(1, coef.size()));
  m.col_lo = pool.get_t<int>(name + ".clo", g.n2e);
  m.col_hi = pool.get_t<int>(name + ".chi", g.n2e);
  m.col_base = pool.get_t<int>(name + ".cbase", g.n2e);
  m.rowptr = pool.get_t<int>(name + ".rp", std::max<size_t>(2, rp.size()));
  upload(m.pt, pt.data(), pt.size() * sizeof(int), h->st);
  upload(m.ptr, ptr.data(), ptr.size() * sizeof(int), h->st);
  upload(m.sta, sta.data(), sta.size() * sizeof(int), h->st);
  upload(m.coef, coef.data(), coef.size() * sizeof(float), h->st);
  upload(m.col_lo, clo.data(), g.n2e * sizeof(int), h->st);
  upload(m.col_hi, chi.data(), g.n2e * sizeof(int), h->st);
  upload(m.col_base, cbase.data(), g.n2e * sizeof(int), h->st);
  upload(m.rowptr, rp.data(), rp.size() * sizeof(int), h->st);
  std::vector<float2> ent(sta.size());
  for (size_t i = 0; i < sta.size(); ++i) {
    float sbits;
    std::memcpy(&sbits, &sta[i], sizeof sbits);
    ent[i] = make_float2(coef[i], sbits);
  }
  m.ent = pool.get_t<float2>(name + ".ent", std::max<size_t>(1, ent.size()));
  upload(m.ent, ent.data(), ent.size() * sizeof(float2), h->st);
  m.nsta = n;
  sync(h);
  return m;
}

// ---------------------------------------------------------------------------
// Simulation state and histories
// ---------------------------------------------------------------------------
int hist_ld(const daw_handle* h) {
  // interior rows per column, padded to 8 elements (16 B of FP16)
  return h->g.hist_rows();
}
size_t hist_bytes_per_step(const daw_handle* h, bool fp16) {
  return (size_t)3 * hist_ld(h) * h->g.n2 * (fp16 ? 2 : 4);
}

// Fields of a shot's state block (see ShotCtx).
constexpr int kStateFields = 9;

// State and history of a shot of nt_alloc steps; win > 0 (less than
// nt_alloc) keeps the history in windows of win steps.
void alloc_state(daw_handle* h, ShotCtx& c, int slot, int nt_alloc, bool fp16, int win = 0) {
  const size_t ne = h->g.ext_elems();
  const std::string p = "slot" + std::to_string(slot) + ".";
  c.set_state(h->pool.get_t<float>(p + "state", kStateFields * ne), ne);
  c.par = 0;
  const int hs = (win > 0 && win < nt_alloc) ? win : nt_alloc;
  c.hist = h->pool.get(p + "hist", hist_bytes_per_step(h, fp16) * (size_t)hs);
  c.hist_steps = hs;
  c.amax = h->pool.get_t<unsigned>(p + "amax", (size_t)(hs + 1) * 3 * kAmaxSlots);
  c.d_cost = h->pool.get_t<double>(p + "cost", 1);
  c.hist_win = hs < nt_alloc ? hs : 0;
  if (c.hist_win) {
    const size_t nwin = (size_t)(nt_alloc + hs - 1) / hs;
    c.st_b = h->pool.get_t<float>(p + "stateB", kStateFields * ne);
    c.ckpt = h->pool.get_t<float>(p + "ckpt", (nwin - 1) * 5 * ne);
  }
}

void zero_state(daw_handle* h, ShotCtx& c) {
  CK(cudaMemsetAsync(c.state, 0, kStateFields * h->g.ext_elems() * sizeof(float), h->st));
  c.par = 0;
}

// ---------------------------------------------------------------------------
// Plain-port simulations (one shot, one kernel per reference loop nest).
// Plain histories are FP32 [it][3][n2][n1h].
// ---------------------------------------------------------------------------
float* hist32(daw_handle* h, ShotCtx& c, int it1, int field) {
  const size_t ni = (size_t)hist_ld(h) * h->g.n2;
  return static_cast<float*>(c.hist) + ((size_t)(it1 - 1) * 3 + field) * ni;
}

// Device time of one time loop (events on the library stream).
struct SimClock {
  daw_handle* h;
  explicit SimClock(daw_handle* hh) : h(hh) { CK(cudaEventRecord(h->ev0, h->st)); }
  void stop(double* ms, double* steps, double nsteps, double shot_steps) {
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaEventSynchronize(h->ev1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms += t;
    *steps += nsteps;
    h->tim.shot_steps += shot_steps;
  }
};

void plain_forward(daw_handle* h, ShotCtx& c, float* sis, float* wf, float* red) {
  const Grid& g = h->g;
  PlainFields f{c.p, c.px, c.pz, c.vx, c.vz};
  zero_state(h, c);
  CK(cudaMemsetAsync(sis, 0, (size_t)c.nt * c.nr * sizeof(float), h->st));
  if (red) CK(cudaMemsetAsync(red, 0, (size_t)c.nt * h->ndatum * sizeof(float), h->st));
  const size_t ni = g.int_elems();
  SimClock clk(h);
  for (int it = 1; it <= c.nt; ++it) {
    plain_p_update(g, h->md, f, 2, +1, h->st);
    if (c.type_src == 0) plain_inject(c.srcmap, c.px, h->md.kap, g.dt, c.d_s + (it - 1), 0, +1, h->st);
    plain_psum(g, f, h->st);
    if (c.type_rec == 0) {
      if (wf) plain_store_interior(g, wf + ni * (it - 1), c.p, false, h->st);
      hicks_gather(c.rec, c.p, g.ld, 0, g.n1e, g.n2e, sis, c.nt, it - 1, 1, 0, h->st);
      if (red && h->ndatum)
        hicks_gather(h->datum, c.p + g.npml + (size_t)g.ld * g.npml, g.ld, g.npml, g.n1, g.n2,
                     red, c.nt, it - 1, 1, 0, h->st);
    }
    plain_v_update(g, h->md, f, 2, +1, h->st);
    if (c.type_src == 1) plain_inject(c.srcmap, c.vz, h->md.rbue, g.dt, c.d_s + (it - 1), 0, +1, h->st);
    plain_vz_free_surface(g, c.vz, h->st);
    h->tim.kernel_launches += 6;
  }
  check_launch("plain forward");
  clk.stop(&h->tim.sim_fwd_ms, &h->tim.steps_fwd, c.nt, c.nt);
  h->tim.point_updates += (double)c.nt * g.n1e * g.n2e;
}

void plain_stage_a(daw_handle* h, ShotCtx& c, const float* res) {
  const Grid& g = h->g;
  PlainFields f{c.p, c.px, c.pz, c.vx, c.vz};
  zero_state(h, c);
  SimClock clk(h);
  for (int it = 1; it <= c.nt; ++it) {
    plain_p_update(g, h->md, f, 3, -1, h->st);
    plain_inject(c.recmap, c.px, h->md.kap, g.dt, res + (it - 1), c.nt, -1, h->st);
    plain_psum(g, f, h->st);
    plain_store_interior(g, hist32(h, c, it, 0), c.p, false, h->st);
    plain_v_update(g, h->md, f, 3, -1, h->st);
    plain_vz_free_surface(g, c.vz, h->st);
    plain_store_interior(g, hist32(h, c, it, 1), c.vx, false, h->st);
    plain_store_interior(g, hist32(h, c, it, 2), c.vz, false, h->st);
    h->tim.kernel_launches += 8;
  }
  check_launch("plain stage A");
  clk.stop(&h->tim.sim_a_ms, &h->tim.steps_a, c.nt, c.nt);
  h->tim.point_updates += (double)c.nt * g.n1e * g.n2e;
  h->tim.hist_bytes += (double)c.nt * 3 * g.int_elems() * 4;
}

void plain_stage_b(daw_handle* h, ShotCtx& c, bool esource, float* out, int reverse, float* wf,
                   float* red) {
  const Grid& g = h->g;
  PlainFields f{c.p, c.px, c.pz, c.vx, c.vz};
  zero_state(h, c);
  CK(cudaMemsetAsync(out, 0, (size_t)c.nt * c.nr * sizeof(float), h->st));
  if (red) CK(cudaMemsetAsync(red, 0, (size_t)c.nt * h->ndatum * sizeof(float), h->st));
  const size_t ni = g.int_elems();
  SimClock clk(h);
  for (int it = 1; it <= c.nt; ++it) {
    const int ic = c.nt - it + 1;
    plain_p_update(g, h->md, f, 3, +1, h->st);
    plain_psrc(g, h->md, c.px, hist32(h, c, ic, 0), esource, h->st);
    plain_psum(g, f, h->st);
    if (c.type_rec == 0) {
      if (wf) plain_store_interior(g, wf + ni * (it - 1), c.p, true, h->st);
      hicks_gather(c.rec, c.p, g.ld, 0, g.n1e, g.n2e, out, c.nt, reverse ? c.nt - it : it - 1, 1,
                   0, h->st);
      if (red && h->ndatum)
        hicks_gather(h->datum, c.p + g.npml + (size_t)g.ld * g.npml, g.ld, g.npml, g.n1, g.n2,
                     red, c.nt, it - 1, 1, 0, h->st);
    }
    plain_v_update(g, h->md, f, 3, +1, h->st);
    plain_vsrc(g, h->md, c.vx, c.vz, hist32(h, c, ic, 1), hist32(h, c, ic, 2), h->st);
    plain_vz_free_surface(g, c.vz, h->st);
    h->tim.kernel_launches += 7;
  }
  check_launch("plain stage B");
  clk.stop(&h->tim.sim_b_ms, &h->tim.steps_b, c.nt, c.nt);
  h->tim.point_updates += (double)c.nt * g.n1e * g.n2e;
  h->tim.hist_bytes += (double)c.nt * 3 * g.int_elems() * 4;
}

// ---------------------------------------------------------------------------
// Fused-path simulations (batch of shots, two kernels per step).
// ---------------------------------------------------------------------------
struct Batch {
  std::vector<ShotCtx*> shots;
  ShotDevice* d_shots = nullptr;
  TmaMaps* d_maps = nullptr;
  StepMaps* d_smaps = nullptr;
  std::vector<ShotDevice> h_shots;
  int max_nt = 0, max_rec = 0, max_datum = 0;
  bool no_datum = false;  // forward-only batches: no datum gathers
  int slot0 = 0;
};

// A window of a checkpointed shot's record: steps s0+1 .. s0+len.
struct Window {
  int s0 = 0, len = 0;
};

// 0: TMA-pipelined persistent kernels (default); 1, 2, 4: register kernels
// with that many columns per thread.
int chunk_of(const daw_handle* h) { return h->opt.chunk; }
// Tensor maps needed by the TMA kernels: the split kernels' unless the
// one-kernel-per-step family is pinned, the step kernels' unless the split
// family is pinned (DAW_OPT_STEP_KERNEL 0 / 1; 2 = autotuned needs both).
bool tma_path(const daw_handle* h) { return h->opt.fused && h->opt.chunk == 0; }
bool split_maps(const daw_handle* h) { return tma_path(h) && h->opt.step != 1; }
bool step_maps(const daw_handle* h) { return tma_path(h) && h->opt.step != 0; }
// Family of the windows of a checkpointed shot (not tuned): the step kernels
// only when pinned.
bool windowed_step(const daw_handle* h) { return tma_path(h) && h->opt.step == 1; }

// Device descriptors (and tensor maps) of the batch's shots for `mode`.  With
// a window, stage A sees the window as a record of w->len steps whose
// amplitudes start at step w->s0 + 1.
void fill_shot_devices(daw_handle* h, Batch& b, int mode, const Window* w = nullptr) {
  b.h_shots.resize(b.shots.size());
  for (size_t i = 0; i < b.shots.size(); ++i) {
    ShotCtx& c = *b.shots[i];
    ShotDevice& d = b.h_shots[i];
    std::memset(&d, 0, sizeof d);
    d.px = c.px; d.pz = c.pz; d.vx = c.vx; d.vz = c.vz; d.p = c.p;
    d.px2 = c.px2; d.pz2 = c.pz2; d.vx2 = c.vx2; d.vz2 = c.vz2;
    d.hist = c.hist;
    d.amax = c.amax;
    d.nt = c.nt;
    d.type_src = c.type_src;
    d.type_rec = c.type_rec;
    d.active = c.active ? 1 : 0;
    d.rec = c.rec;
    if (h->ndatum > 0 && !b.no_datum) d.datum = h->datum;  // else n = 0: no datum gathers
    d.cost = nullptr;
    if (mode == FM_FWD) {
      d.amp = c.d_s;
      d.amp_stride = 0;
      d.inj = c.srcmap;
      d.out = c.d_datar;
      d.out_reverse = 0;
      d.red = h->ndatum > 0 && !b.no_datum ? c.d_redF : nullptr;
      d.wf = c.d_wf;
      d.wf_acc = 0;
    } else if (mode == FM_STAGE_A) {
      d.amp = c.op_in + (w ? w->s0 : 0);
      d.amp_stride = c.nt;
      d.inj = c.recmap;
      if (w) d.nt = w->len;
    } else {
      d.out = c.op_out;
      d.out_reverse = c.op_reverse;
      if (mode == FM_STAGE_B_ES) {
        d.red = h->ndatum > 0 ? c.d_redE : nullptr;
        d.wf = c.d_wf;
        d.wf_acc = 1;
      }
    }
  }
  upload(b.d_shots, b.h_shots.data(), b.h_shots.size() * sizeof(ShotDevice), h->st);
  if (step_maps(h)) {
    // tensor maps of every shot for both tile widths: [tile width 16 | 32][shot]
    const size_t n = b.shots.size();
    std::vector<StepMaps> maps(2 * n);
    for (size_t i = 0; i < n; ++i) {
      const ShotCtx& c = *b.shots[i];
      float* const st[2][4] = {{c.px, c.pz, c.vx, c.vz}, {c.px2, c.pz2, c.vx2, c.vz2}};
      for (int t = 0; t < 2; ++t)
        if (!step_encode_maps(h->g, st, h->md.kap, c.hist, h->opt.history_fp16, hist_ld(h),
                              c.hist_steps, t ? 32 : 16, &maps[t * n + i]))
          throw DawError{DAW_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    }
    b.d_smaps = static_cast<StepMaps*>(h->pool.get(
        "batch.smaps" + std::to_string(b.slot0) + "." + std::to_string(mode),
        maps.size() * sizeof(StepMaps)));
    upload(b.d_smaps, maps.data(), maps.size() * sizeof(StepMaps), h->st);
    sync(h);  // `maps` goes out of scope
  }
  if (split_maps(h)) {
    // tensor maps of every shot's fields (the TMA kernels' operands)
    std::vector<TmaMaps> maps(b.shots.size());
    for (size_t i = 0; i < b.shots.size(); ++i) {
      const ShotCtx& c = *b.shots[i];
      if (!tma_encode_maps(h->g, c.vx, c.vz, c.px, c.pz, c.p, h->md.kap, c.hist,
                           h->opt.history_fp16, hist_ld(h), c.hist_steps, &maps[i]))
        throw DawError{DAW_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    }
    // one buffer per mode: a buffer's contents then never change between the
    // launches of a run or a cached graph (windowed runs switch the state
    // pointers between stage A and stage B)
    b.d_maps = static_cast<TmaMaps*>(
        h->pool.get("batch.maps" + std::to_string(b.slot0) + "." + std::to_string(mode),
                    maps.size() * sizeof(TmaMaps)));
    upload(b.d_maps, maps.data(), maps.size() * sizeof(TmaMaps), h->st);
    sync(h);  // `maps` goes out of scope
  }
}

FusedLaunch launch_of(daw_handle* h, Batch& b) {
  FusedLaunch L{};  // nparam = 0: no per-shot parameters unless set
  L.shots = b.d_shots;
  L.nshots = (int)b.shots.size();
  L.hist_fp16 = h->opt.history_fp16;
  L.n1h = hist_ld(h);
  L.chunk = chunk_of(h);
  L.max_rec = b.max_rec;
  L.max_datum = b.max_datum;
  L.maps = b.d_maps;
  L.err = h->d_err;
  L.persist_p = h->persist_p;
  L.persist_v = h->persist_v;
  L.pdl = h->opt.pdl;
  return L;
}

void check_device_error(daw_handle* h) {
  unsigned e = 0;
  CK(cudaMemcpy(&e, h->d_err, sizeof e, cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(h->d_err, 0, sizeof(unsigned)));
    if (e & kErrTimeout)
      throw DawError{DAW_ERR_TIMEOUT,
                     "a bounded device wait ran out (TMA tile copy did not complete)"};
    throw DawError{DAW_ERR_NAN, "non-finite value (NaN or Inf) in a stage-A wavefield history"};
  }
}

void stop_clock(daw_handle* h, SimClock& clk, Batch& b, int mode, const Window* w, int lo = 0,
                int hi = -1) {
  if (hi < 0) hi = (int)b.shots.size();
  double shot_steps = 0;
  int gmax = 0;
  for (int i = lo; i < hi; ++i) {
    const ShotCtx* c = b.shots[i];
    if (c->active) shot_steps += w ? w->len : c->nt;
    gmax = std::max(gmax, c->nt);
  }
  double* ms = mode == FM_FWD ? &h->tim.sim_fwd_ms : mode == FM_STAGE_A ? &h->tim.sim_a_ms : &h->tim.sim_b_ms;
  double* st = mode == FM_FWD ? &h->tim.steps_fwd : mode == FM_STAGE_A ? &h->tim.steps_a : &h->tim.steps_b;
  (mode == FM_FWD ? h->tim.shot_steps_fwd : mode == FM_STAGE_A ? h->tim.shot_steps_a
                                                                : h->tim.shot_steps_b) += shot_steps;
  clk.stop(ms, st, w ? w->len : gmax, shot_steps);
}

// Autotuner of the TMA time-step kernels, per (mode, history precision,
// grid, batch).  Candidates are timed over the run's first six steps (at
// least two, so the one-kernel-per-step family's work deferred to the next
// launch is counted; six, so a 20-40 us step is timed well above the event
// resolution), median of 3 after a warm-up, and compared by device time per
// shot step:
//   - separate pressure and velocity kernels (64 x 32 tiles): the shots per
//     launch -- an HBM-admitted batch can run its time loops in groups of k
//     shots, and the fastest k is often below the batch because the groups'
//     wavefield state then stays in L2 -- and then, for that k, 1 ..
//     occupancy CTAs per SM of each kernel;
//   - with DAW_OPT_STEP_KERNEL = 2 or 1, one kernel per step with 16- or
//     32-column tiles and 1 .. occupancy CTAs per SM (whole batch).
// Only runs that start from the zero state are tuned; the windows of a
// checkpointed shot take the family DAW_OPT_STEP_KERNEL names with default
// shapes.  The trials change only what the run itself then overwrites: the
// state (zeroed again afterwards, and the stage-A max-|x| slots cleared), the
// first history slots and the first rows of the outputs.  The final esource,
// whose first step also accumulates into the wavefield output, tunes as stage
// B (same kernel shapes) and takes stage B's choice.
daw_handle::Tuned tune_run(daw_handle* h, Batch& b, int mode, FusedLaunch L, int first,
                           int last_step, bool may_time) {
  const int tmode = mode == FM_STAGE_B_ES ? FM_STAGE_B : mode;
  const int f = L.hist_fp16 ? 1 : 0;
  const int occ_p = std::max(1, std::min(h->persist_p / h->sms, 3));
  const int occ_v = std::max(1, std::min(h->persist_v_mode[tmode * 2 + f] / h->sms, 3));
  std::vector<int> act;  // active shots (indices < 64)
  for (size_t i = 0; i < b.shots.size() && i < 64; ++i)
    if (b.shots[i]->active) act.push_back((int)i);
  const int nact = std::max<int>(1, (int)act.size());
  const daw_handle::Tuned split_default{0, 32, occ_p, occ_v, 0, 0.f};
  if (!may_time) {  // checkpointed windows: the named family, default shapes
    if (h->opt.step == 1) {
      const int tc = h->opt.tile_cols ? h->opt.tile_cols : 32;
      const int occ = std::max(1, std::min(h->step_occ[tmode][f][tc == 32 ? 1 : 0], 3));
      return {1, tc, h->opt.ctas_per_sm ? std::min(h->opt.ctas_per_sm, occ) : occ, 0, 0, 0.f};
    }
    return split_default;
  }
  char key[192];
  std::snprintf(key, sizeof key, "m%d.f%d.g%dx%d.p%d.s%d.a%d.r%d.d%d.k%d.t%d.c%d.rho%d", tmode,
                f, h->g.n1, h->g.n2, h->g.npml, L.nshots, nact, L.max_rec, L.max_datum,
                h->opt.step, h->opt.tile_cols, h->opt.ctas_per_sm, h->md.rbw1 ? 1 : 0);
  auto found = h->tuned.find(key);
  if (found != h->tuned.end()) return found->second;
  const size_t n = b.shots.size();
  auto trial = [&](const daw_handle::Tuned& cd) -> float {  // us per shot step
    FusedLaunch T = L;
    const int k = cd.family == 0 && cd.sub > 0 ? std::min(cd.sub, nact) : nact;
    if (cd.family == 0) {
      T.nlive = 0;
      for (int i = 0; i < k && i < (int)act.size(); ++i) T.live[T.nlive++] = (unsigned char)act[i];
      T.persist_p = cd.ctas_per_sm * h->sms;
      T.persist_v = cd.ctas_per_sm_v * h->sms;
    } else {
      T.tile_cols = cd.tile_cols;
      T.smaps = b.d_smaps + (cd.tile_cols == 32 ? n : 0);
    }
    const int nst = std::min(first + 5, last_step) - first + 1;
    float ms[3];
    for (int r = 0; r < 4; ++r) {
      if (cd.family == 1) CK(cudaMemsetAsync(h->d_qctr, 0, sizeof(unsigned), h->st));
      if (r > 0) CK(cudaEventRecord(h->ev0, h->st));
      for (int st = first; st < first + nst; ++st) {
        if (cd.family == 1) {
          step_launch(h->g, h->md, T, tmode, st, cd.ctas_per_sm * h->sms, h->st);
        } else {
          tma_p_step(h->g, h->md, T, tmode, st, h->st);
          tma_v_step(h->g, h->md, T, tmode, st, h->st);
        }
      }
      if (r > 0) {
        CK(cudaEventRecord(h->ev1, h->st));
        CK(cudaEventSynchronize(h->ev1));
        CK(cudaEventElapsedTime(&ms[r - 1], h->ev0, h->ev1));
      }
    }
    check_launch("time-step kernels (tuning)");
    h->tim.kernel_launches += 4 * nst * (cd.family == 1 ? 1 : 2);
    std::sort(ms, ms + 3);
    return ms[1] * 1e3f / (float)(nst * k);
  };
  daw_handle::Tuned best = split_default;
  best.us_per_step = 1e30f;
  bool timed = false;
  auto consider = [&](daw_handle::Tuned cd) {
    cd.us_per_step = trial(cd);
    timed = true;
    if (cd.us_per_step < best.us_per_step) best = cd;
  };
  if (h->opt.step != 1) {
    // shots per launch (default shapes), then the CTAs per SM for the best
    std::vector<int> ks;
    for (int k : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64})
      if (k < nact) ks.push_back(k);
    ks.push_back(nact);
    if (ks.size() > 1)
      for (int k : ks) consider({0, 32, occ_p, occ_v, k == nact ? 0 : k, 0.f});
    const int kbest = best.family == 0 ? best.sub : 0;
    if (occ_p * occ_v > 1)
      for (int pc = 1; pc <= occ_p; ++pc)
        for (int vc = 1; vc <= occ_v; ++vc)
          if (!(timed && pc == occ_p && vc == occ_v)) consider({0, 32, pc, vc, kbest, 0.f});
  }
  if (h->opt.step != 0 && !h->md.rbw1)  // the step family has no density variant
    for (int tc : {16, 32}) {
      if (h->opt.tile_cols && h->opt.tile_cols != tc) continue;
      // a pinned CTA count above what fits is clamped to the occupancy
      const int occ = std::min(h->step_occ[tmode][f][tc == 32 ? 1 : 0], 3);
      const int pin = h->opt.ctas_per_sm ? std::min(h->opt.ctas_per_sm, occ) : 0;
      for (int c = 1; c <= occ; ++c)
        if (!pin || pin == c) consider({1, tc, c, 0, 0, 0.f});
    }
  if (!timed) best = split_default;
  if (timed) {
    // undo the trials: the run starts from the zero state and clear slots
    for (ShotCtx* c : b.shots) {
      if (!c->active) continue;
      zero_state(h, *c);
      if (mode == FM_STAGE_A)
        CK(cudaMemsetAsync(c->amax, 0, (size_t)(c->nt + 1) * 3 * kAmaxSlots * sizeof(unsigned),
                           h->st));
    }
    check_device_error(h);
  }
  h->tuned[key] = best;
  return best;
}

// Runs `nsteps` steps of `mode`, captured once per batch/mode in a CUDA
// graph when enabled (kernel arguments are constant; per-shot pointers live in
// the device-side ShotDevice array, refreshed before each replay).
//
// With a window (one shot, checkpointed stage A): stage A runs the window as a
// record of w->len steps; stage B runs the record steps that read the
// window's history, nt-s0-len+1 .. nt-s0, with history slot 0 = step s0+1.
// Windowed runs are captured in graphs too, keyed by the window's first and
// last step, its history offset and the state set the run starts from; each
// mode has its own tensor-map buffer, whose contents stay fixed for a stage.
void run_fused(daw_handle* h, Batch& b, int mode, const Window* w = nullptr) {
  const Grid& g = h->g;
  if (w && b.shots.size() != 1) throw DawError{DAW_ERR_STATE, "a windowed run holds one shot"};
  FusedLaunch L = launch_of(h, b);
  L.persist_v = h->persist_v_mode[mode * 2 + (L.hist_fp16 ? 1 : 0)];
  L.nparam = std::min<int>((int)b.shots.size(), FusedLaunch::kParamShots);
  unsigned long long phash = 1469598103934665603ull;  // FNV-1a of the per-shot parameters
  auto mix = [&](unsigned long long v) { phash = (phash ^ v) * 1099511628211ull; };
  for (int i = 0; i < FusedLaunch::kParamShots; ++i) {
    const ShotCtx* c = i < L.nparam ? b.shots[i] : nullptr;
    L.shot_amax[i] = c ? c->amax : nullptr;
    L.shot_amp[i] = !c ? nullptr
                    : mode == FM_FWD ? c->d_s
                    : mode == FM_STAGE_A ? c->d_ampT + (w ? (size_t)w->s0 * c->nr : 0)
                                         : nullptr;
    L.shot_nt[i] = !c ? 0 : (w && mode == FM_STAGE_A) ? w->len : c->nt;
    L.shot_nsta[i] = !c ? 0 : mode == FM_FWD ? 1 : mode == FM_STAGE_A ? c->nr : 0;
    mix((unsigned long long)(uintptr_t)L.shot_amax[i]);
    mix((unsigned long long)(uintptr_t)L.shot_amp[i]);
    mix((unsigned long long)L.shot_nt[i] << 32 | (unsigned)L.shot_nsta[i]);
  }
  // steps first..last; the velocity kernel runs for it <= nt_v
  int first = 1, nt_v = b.max_nt;
  if (w && mode == FM_STAGE_A) {
    nt_v = w->len;
  } else if (w) {
    first = b.max_nt - w->s0 - w->len + 1;
    nt_v = b.max_nt - w->s0;
    L.hist_step0 = w->s0;
  }
  const bool tma = L.chunk == 0;
  L.first = first;
  L.step_last = nt_v;
  L.qctr = h->d_qctr;  // tile queue of the one-kernel-per-step path
  L.ngath = mode == FM_STAGE_A ? 0 : (L.max_rec + (b.no_datum ? 0 : L.max_datum) + 7) / 8;
  L.active_mask = 0;
  for (size_t i = 0; i < b.shots.size() && i < 64; ++i)
    if (b.shots[i]->active) L.active_mask |= 1ull << i;
  // shots with work at step it: active, and it within the record (the split
  // pressure kernel's stage-A flush step included)
  auto live_of = [&](FusedLaunch& T, int it, bool velocity, int lo = 0, int hi = 64) {
    T.nlive = 0;
    for (size_t i = lo; i < b.shots.size() && (int)i < std::min(hi, 64); ++i) {
      const ShotCtx* c = b.shots[i];
      if (!c->active) continue;
      const int nts = (w && mode == FM_STAGE_A) ? w->len : c->nt;
      const int lim = nts + ((mode == FM_STAGE_A && !velocity) ? 1 : 0);
      if (it <= lim) T.live[T.nlive++] = (unsigned char)i;
    }
  };
  live_of(L, first, false);
  daw_handle::Tuned tn{0, 32, 0, 0, 0, 0.f};
  if (tma) {
    tn = tune_run(h, b, mode, L, first, nt_v, w == nullptr);
    h->tim.kernel_family[mode] = tn.family;
    h->tim.tile_cols[mode] = tn.tile_cols;
    h->tim.ctas_per_sm[mode] = tn.ctas_per_sm;
    h->tim.ctas_per_sm_v[mode] = tn.ctas_per_sm_v;
    h->tim.shots_per_launch[mode] = tn.family == 0 && tn.sub ? tn.sub : (int)b.shots.size();
    if (tn.family == 0) {
      L.persist_p = tn.ctas_per_sm * h->sms;
      L.persist_v = tn.ctas_per_sm_v * h->sms;
    }
  }
  const bool step = tma && tn.family == 1;
  // the step path's extra launch does the last step's deferred work; the
  // split kernels' extra stage-A launch flushes its history
  const int last = step ? nt_v + 1 : (mode == FM_STAGE_A) ? nt_v + 1 : nt_v;
  int grid = 0;
  if (step) {
    int par0 = -1;
    for (ShotCtx* c : b.shots) {
      if (!c->active) continue;
      if (par0 >= 0 && c->par != par0)
        throw DawError{DAW_ERR_STATE, "shots of a batch start from different state sets"};
      par0 = c->par;
    }
    L.par0 = std::max(par0, 0);
    L.tile_cols = tn.tile_cols;
    L.smaps = b.d_smaps + (tn.tile_cols == 32 ? b.shots.size() : 0);
    grid = tn.ctas_per_sm * h->sms;
  }
  // The time loop of shots [lo, hi) of the batch (the split kernels run an
  // admitted batch in groups of the tuned shots per launch; the other paths
  // take the whole batch).
  auto run_group = [&](int lo, int hi) {
    auto body = [&]() {
      if (step) {
        CK(cudaMemsetAsync(h->d_qctr, 0, sizeof(unsigned), h->st));
        for (int it = first; it <= last; ++it) step_launch(g, h->md, L, mode, it, grid, h->st);
        return;
      }
      for (int it = first; it <= last; ++it) {
        if (tma) {
          FusedLaunch T = L;
          live_of(T, it, false, lo, hi);
          if (T.nlive) tma_p_step(g, h->md, T, mode, it, h->st);
          live_of(T, it, true, lo, hi);
          if (it <= nt_v && T.nlive) tma_v_step(g, h->md, T, mode, it, h->st);
        } else {
          fused_p_step(g, h->md, L, mode, it, h->st);
          if (it <= nt_v) fused_v_step(g, h->md, L, mode, it, h->st);
        }
      }
    };
    if (h->opt.graph) {
      char key[360];
      std::snprintf(key, sizeof key,
                    "m%d.n%d.s%zu.p%p.q%p.z%p.c%d.f%d.r%d.d%d.h%llx.w%d.%d.%d.%d.%d.%d.%d.a%llx.l%d"
                    ".g%d.%d.v%d",
                    mode, b.max_nt, b.shots.size(), (void*)b.d_shots, (void*)b.d_maps,
                    (void*)b.d_smaps, L.chunk, L.hist_fp16, L.max_rec, L.max_datum, phash, step,
                    first, last, L.hist_step0, L.par0, L.tile_cols, grid, L.active_mask, L.pdl,
                    lo, hi, L.persist_p * 1000 + L.persist_v);
      auto it = h->graphs.find(key);
      if (it == h->graphs.end()) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        body();
        CK(cudaStreamEndCapture(h->st, &graph));
        cudaGraphExec_t exec;
        CK(cudaGraphInstantiate(&exec, graph, 0));
        cudaGraphDestroy(graph);
        it = h->graphs.emplace(key, exec).first;
      }
      SimClock clk(h);
      CK(cudaGraphLaunch(it->second, h->st));
      stop_clock(h, clk, b, mode, w, lo, hi);
    } else {
      SimClock clk(h);
      body();
      stop_clock(h, clk, b, mode, w, lo, hi);
    }
  };
  const int nsteps = nt_v - first + 1;
  long long launches = 0;
  const int nb = (int)b.shots.size();
  const int k = (tma && !step && tn.sub > 0) ? tn.sub : nb;
  for (int lo = 0; lo < nb; lo += k) {
    run_group(lo, std::min(nb, lo + k));
    launches += step ? (long long)nsteps + 1 : 2LL * nsteps + (mode == FM_STAGE_A ? 1 : 0);
  }
  check_launch("fused steps");
  check_device_error(h);
  h->tim.kernel_launches += launches;
  for (ShotCtx* c : b.shots) {
    if (!c->active) continue;
    const int steps = w ? (mode == FM_STAGE_A ? w->len : nt_v - first + 1) : c->nt;
    if (step) c->par = (c->par + steps) & 1;  // the set holding the state after the run
    h->tim.point_updates += (double)steps * g.n1e * g.n2e;
    if (mode != FM_FWD)
      h->tim.hist_bytes += (double)steps * 3 * g.int_elems() * (h->opt.history_fp16 ? 2 : 4);
  }
}

void clear_amax(daw_handle* h, Batch& b) {
  for (ShotCtx* c : b.shots)
    CK(cudaMemsetAsync(c->amax, 0, (size_t)(c->nt + 1) * 3 * kAmaxSlots * sizeof(unsigned), h->st));
}

// ---------------------------------------------------------------------------
// Operators over a batch.  op_in/op_out/op_reverse are set per shot.
// ---------------------------------------------------------------------------
void batch_forward(daw_handle* h, Batch& b) {
  if (!h->opt.fused) {
    for (ShotCtx* c : b.shots)
      plain_forward(h, *c, c->d_datar, c->d_wf, h->ndatum && !b.no_datum ? c->d_redF : nullptr);
    return;
  }
  for (ShotCtx* c : b.shots) {
    CK(cudaMemsetAsync(c->d_datar, 0, (size_t)c->nt * c->nr * sizeof(float), h->st));
    if (h->ndatum)
      CK(cudaMemsetAsync(c->d_redF, 0, (size_t)c->nt * h->ndatum * sizeof(float), h->st));
    zero_state(h, *c);
  }
  fill_shot_devices(h, b, FM_FWD);
  run_fused(h, b, FM_FWD);
}

// G G^T (stage A + stage B) of one shot whose stage-A history is kept in
// windows of K = hist_win steps.  Stage A runs once over the record, window
// by window, saving its state before each window; the last window's history
// stays in the buffer.  Stage B then takes the windows in reverse order and,
// before each window but the last, re-runs stage A over that window from the
// saved state.  Stage A's kernels see a window as a record of its own length
// whose amplitudes start at the window's first step, and the history flush
// step leaves the state unchanged, so every history value comes from the same
// operations as in the whole-record run: the outputs are equal bit for bit
// (the FP64 cost sum aside, whose order is unspecified in both).
void shot_operator_windowed(daw_handle* h, Batch& b, bool esource) {
  ShotCtx& c = *b.shots[0];
  if (!c.active) return;
  const size_t ne = h->g.ext_elems();
  // a saved state: the four fields of the current set (one-kernel-per-step
  // path) or px, pz, vx, vz, p (split kernels); ckpt slots hold 5 fields
  const bool step = windowed_step(h);
  const size_t save_bytes = (step ? 4 : 5) * ne * sizeof(float);
  const int K = c.hist_win, nwin = (c.nt + K - 1) / K;
  float* const st_a = c.state;  // the slot's state block
  auto use_state = [&](float* s9, int par) {
    c.set_state(s9, ne);
    c.par = par;
  };
  auto cur_fields = [&]() { return (step && c.par) ? c.px2 : c.px; };
  struct Restore {  // the ShotCtx points at stage A's state again on every exit
    std::function<void()> f;
    ~Restore() { f(); }
  } restore{[&] { use_state(st_a, 0); }};
  auto window = [&](int w) { return Window{w * K, std::min(K, c.nt - w * K)}; };
  auto stage_a = [&](int w) {
    const Window win = window(w);
    CK(cudaMemsetAsync(c.amax, 0, (size_t)(win.len + 1) * 3 * kAmaxSlots * sizeof(unsigned), h->st));
    fill_shot_devices(h, b, FM_STAGE_A, &win);
    run_fused(h, b, FM_STAGE_A, &win);
  };
  if (c.nr > 0) {
    transpose_traces(c.op_in, c.d_ampT, c.nt, c.nr, h->st);
    h->tim.kernel_launches += 1;
  }
  zero_state(h, c);
  for (int w = 0; w < nwin; ++w) {
    if (w > 0)
      CK(cudaMemcpyAsync(c.ckpt + (size_t)(w - 1) * 5 * ne, cur_fields(), save_bytes,
                         cudaMemcpyDeviceToDevice, h->st));
    stage_a(w);
  }
  const int mode = esource ? FM_STAGE_B_ES : FM_STAGE_B;
  use_state(c.st_b, 0);
  zero_state(h, c);
  CK(cudaMemsetAsync(c.op_out, 0, (size_t)c.nt * c.nr * sizeof(float), h->st));
  if (esource && h->ndatum)
    CK(cudaMemsetAsync(c.d_redE, 0, (size_t)c.nt * h->ndatum * sizeof(float), h->st));
  for (int w = nwin - 1; w >= 0; --w) {
    if (w < nwin - 1) {
      const int par_b = c.par;
      use_state(st_a, 0);
      if (w == 0)
        zero_state(h, c);
      else  // into set 0, which the restarted run starts from
        CK(cudaMemcpyAsync(c.px, c.ckpt + (size_t)(w - 1) * 5 * ne, save_bytes,
                           cudaMemcpyDeviceToDevice, h->st));
      stage_a(w);
      use_state(c.st_b, par_b);
    }
    const Window win = window(w);
    if (esource && c.d_cost)
      history_cost(c.hist, h->opt.history_fp16, c.amax, win.len, h->g.n1, h->g.n2, hist_ld(h),
                   h->g.npml - h->g.hist_base(), (size_t)hist_ld(h) * h->g.n2, c.d_cost, h->st);
    fill_shot_devices(h, b, mode, &win);
    run_fused(h, b, mode, &win);
  }
}

// Stage A + stage B.  esource: final simulation (interior 2..n-1 pressure
// source, datum gather, optional wavefield accumulation and cost).
void batch_operator(daw_handle* h, Batch& b, bool esource) {
  if (!h->opt.fused) {
    for (ShotCtx* c : b.shots) {
      if (!c->active) continue;
      plain_stage_a(h, *c, c->op_in);
      if (esource && c->d_cost) {
        history_cost(c->hist, 0, nullptr, c->nt, h->g.n1, h->g.n2, h->g.n1, 0,
                     (size_t)hist_ld(h) * h->g.n2, c->d_cost, h->st);
      }
      plain_stage_b(h, *c, esource, c->op_out, c->op_reverse, esource ? c->d_wf : nullptr,
                    esource && h->ndatum ? c->d_redE : nullptr);
    }
    return;
  }
  for (ShotCtx* c : b.shots)
    if (c->hist_win > 0) {
      if (b.shots.size() != 1)
        throw DawError{DAW_ERR_STATE, "a shot with a windowed history runs alone"};
      shot_operator_windowed(h, b, esource);
      return;
    }
  for (ShotCtx* c : b.shots) {
    if (!c->active) continue;
    zero_state(h, *c);
  }
  clear_amax(h, b);
  for (ShotCtx* c : b.shots)  // step-major residual for the fused kernels' amplitude staging
    if (c->active && c->nr > 0) {
      transpose_traces(c->op_in, c->d_ampT, c->nt, c->nr, h->st);
      h->tim.kernel_launches += 1;
    }
  fill_shot_devices(h, b, FM_STAGE_A);
  run_fused(h, b, FM_STAGE_A);
  for (ShotCtx* c : b.shots) {
    if (!c->active) continue;
    if (esource && c->d_cost)
      history_cost(c->hist, h->opt.history_fp16, c->amax, c->nt, h->g.n1, h->g.n2, hist_ld(h),
                   h->g.npml - h->g.hist_base(), (size_t)hist_ld(h) * h->g.n2, c->d_cost, h->st);
    zero_state(h, *c);
    CK(cudaMemsetAsync(c->op_out, 0, (size_t)c->nt * c->nr * sizeof(float), h->st));
    if (esource && h->ndatum)
      CK(cudaMemsetAsync(c->d_redE, 0, (size_t)c->nt * h->ndatum * sizeof(float), h->st));
  }
  fill_shot_devices(h, b, esource ? FM_STAGE_B_ES : FM_STAGE_B);
  run_fused(h, b, esource ? FM_STAGE_B_ES : FM_STAGE_B);
}

// ---------------------------------------------------------------------------
// Device MINRES over a batch (each shot its own Krylov state).
// ---------------------------------------------------------------------------
template <typename S>
void batch_minres(daw_handle* h, Batch& b) {
  using Ops = MinresOps<S>;
  cudaStream_t st = h->st;
  // buffers
  for (size_t i = 0; i < b.shots.size(); ++i) {
    ShotCtx& c = *b.shots[i];
    const size_t n = (size_t)c.nt * c.nr;
    const std::string p = "mr" + std::to_string(b.slot0 + i) + ".";
    float* base = h->pool.get_t<float>(p + "vec", 8 * n);
    c.y = base; c.v = base + n; c.r1 = base + 2 * n; c.r2 = base + 3 * n;
    c.w = base + 4 * n; c.w1 = base + 5 * n; c.w2 = base + 6 * n; c.gb = base + 7 * n;
    c.x = c.d_deltade;
    const int nblk = minres_blocks(n);
    c.partials = h->pool.get(p + "part", 4 * nblk * sizeof(S));
    c.mdev = h->pool.get(p + "state", sizeof(MinresDev<S>));
    c.log_cap = std::max(1, c.maxiter);
    c.dlog = h->pool.get_t<double>(p + "log", 5 * (size_t)c.log_cap);
    MinresDev<S> init{};
    init.log_capacity = c.log_cap;
    upload(c.mdev, &init, sizeof init, st);
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float op_ms = 0, ms = 0;
  auto timed_op = [&](bool esource) {
    CK(cudaEventRecord(e0, st));
    batch_operator(h, b, esource);
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(&ms, e0, e1));
    op_ms += ms;
  };
  // fac: G G^T applied to deltadr, not time reversed (sublinearminres.f90:64)
  for (ShotCtx* c : b.shots) {
    c->active = true;
    c->op_in = c->d_deltadr;
    c->op_out = c->gb;
    c->op_reverse = 0;
  }
  timed_op(false);
  for (ShotCtx* c : b.shots) {
    const size_t n = (size_t)c->nt * c->nr;
    const int nblk = minres_blocks(n);
    S* P = static_cast<S*>(c->partials);
    Ops::dot(c->d_deltadr, c->d_deltadr, n, P, nblk, st);
    Ops::dot(c->gb, c->gb, n, P + nblk, nblk, st);
    Ops::init(static_cast<MinresDev<S>*>(c->mdev), P, P + nblk, P, nblk, c->mu, c->maxiter,
              c->rtol, st);
    // y = b, r1 = b, r2 = b, x = 0, w = 0, w2 = 0
    CK(cudaMemcpyAsync(c->y, c->d_deltadr, n * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c->r1, c->d_deltadr, n * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c->r2, c->d_deltadr, n * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(c->x, 0, n * 4, st));
  }
  // stop flags
  std::vector<MinresDev<S>> hs(b.shots.size());
  auto fetch = [&]() {
    for (size_t i = 0; i < b.shots.size(); ++i)
      download(&hs[i], b.shots[i]->mdev, sizeof(MinresDev<S>), st);
    sync(h);
  };
  fetch();
  // Unused operator application of the reference (minresModule.f90:132-133).
  if (!h->opt.skip_dead_op) {
    bool any = false;
    for (size_t i = 0; i < b.shots.size(); ++i) {
      ShotCtx* c = b.shots[i];
      c->active = !hs[i].done;
      any |= c->active;
      c->op_in = c->y;
      c->op_out = c->w;
      c->op_reverse = 1;
    }
    if (any) {
      timed_op(false);
      for (ShotCtx* c : b.shots) {
        if (!c->active) continue;
        const size_t n = (size_t)c->nt * c->nr;
        const int nblk = minres_blocks(n);
        S* P = static_cast<S*>(c->partials);
        Ops::dot(c->w, c->w, n, P, nblk, st);
        Ops::arnorm0(static_cast<MinresDev<S>*>(c->mdev), P, nblk, st);
      }
    }
  }
  for (ShotCtx* c : b.shots) {
    const size_t n = (size_t)c->nt * c->nr;
    CK(cudaMemsetAsync(c->w, 0, n * 4, st));
    CK(cudaMemsetAsync(c->w2, 0, n * 4, st));
  }
  float vec_ms = 0;
  // Buffers: r2 holds the current Lanczos vector (the reference's y after
  // `r2 = y`), r1 the previous one, y is the spare the operator writes A v
  // into; after each iteration (r1, r2, y) <- (r2, y, r1).
  for (;;) {
    bool any = false;
    for (size_t i = 0; i < b.shots.size(); ++i) {
      b.shots[i]->active = !hs[i].done;
      any |= b.shots[i]->active;
    }
    if (!any) break;
    for (ShotCtx* c : b.shots) {
      if (!c->active) continue;
      const size_t n = (size_t)c->nt * c->nr;
      Ops::v_from_y(static_cast<MinresDev<S>*>(c->mdev), c->v, c->r2, n, st);
      c->op_in = c->v;
      c->op_out = c->y;
      c->op_reverse = 1;
    }
    timed_op(false);
    CK(cudaEventRecord(e0, st));
    for (ShotCtx* c : b.shots) {
      if (!c->active) continue;
      const size_t n = (size_t)c->nt * c->nr;
      const int nblk = minres_blocks(n);
      S* P = static_cast<S*>(c->partials);
      MinresDev<S>* d = static_cast<MinresDev<S>*>(c->mdev);
      Ops::y1(d, c->y, c->v, c->r1, n, P, nblk, st);
      Ops::alfa(d, P, nblk, st);
      Ops::y2(d, c->y, c->r2, n, P, nblk, st);
      float* old_r1 = c->r1;
      c->r1 = c->r2;
      c->r2 = c->y;
      c->y = old_r1;
      Ops::scal(d, P, nblk, c->dlog, c->x, st);
      float* old_w1 = c->w1;
      c->w1 = c->w2;
      c->w2 = c->w;
      c->w = old_w1;
      Ops::xw(d, c->w, c->w1, c->w2, c->v, c->x, n, st);
      if (sizeof(S) == sizeof(float))
        minres_log_f32(reinterpret_cast<MinresDev<float>*>(d), c->dlog, c->x, st);
      else
        minres_log_f64(reinterpret_cast<MinresDev<double>*>(d), c->dlog, c->x, st);
    }
    CK(cudaEventRecord(e1, st));
    check_launch("minres vector kernels");
    fetch();
    CK(cudaEventElapsedTime(&ms, e0, e1));
    vec_ms += ms;
  }
  h->tim.operator_ms += op_ms;
  h->tim.minres_vec_ms += vec_ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // info
  for (size_t i = 0; i < b.shots.size(); ++i) {
    ShotCtx& c = *b.shots[i];
    const MinresDev<S>& d = hs[i];
    c.info.istop = d.istop;
    c.info.itn = d.itn;
    c.info.nlog = d.nlog;
    c.info.anorm = (double)d.anorm;
    c.info.acond = (double)d.acond;
    c.info.rnorm = (double)d.rnorm;
    c.info.arnorm = (double)d.arnorml;
    c.info.ynorm = (double)d.ynorm;
    c.info.shift = (double)d.shift;
    c.info.beta1 = (double)d.beta1;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Filter weights (src/minresModule.f90:505-586), host side.
// ---------------------------------------------------------------------------
namespace {

// Element j (1-based, j <= nf + 1) of sphanning's Hanning branch of order
// nord over nf + 1 points (src/minresModule.f90:619-632).
float hanning_at(int j, int nf, int nord) {
  const float pi = 3.14159265f;
  const float a = 2.0f * pi * (float)(j - 1) / (float)(2 * nf);
  const float b = (std::cos(a) + 1.0f) / 2.0f + 0.000001f;
  return std::exp(std::log(b) * (float)nord);
}

}  // namespace

namespace daw {

int filter_nto(int nt) {
  for (int s = 8; s <= 65536; s *= 2)
    if (nt <= s) return s;
  return 0;
}

int filter_weights_into(int nt, float dt, float* flow, float* fhig, float* llow, float* lhig,
                        float* fm, double* w) {
  const int nto = filter_nto(nt);
  if (nto == 0) return 0;
  std::fill(fm, fm + nto + 1, 0.0f);
  const float fe = 1.0f / dt, fmax = fe / 2.0f;
  if (*fhig > fmax) {
    *fhig = fmax;
    *lhig = 0.0f;
  }
  // The reference stores nto/fe in an INTEGER (minresModule.f90:492,529).
  const int conv = (int)((float)nto / fe);
  const int iflow = (int)(*flow * (float)conv) + 1;
  const int ifhig = (int)(*fhig * (float)conv) + 1;
  int illow = (int)(*llow * (float)conv) + 1;
  int ilhig = (int)(*lhig * (float)conv) + 1;
  if (iflow - illow < 1 && iflow > 0) illow = iflow - 1;
  if (ifhig + ilhig > nto) ilhig = nto - ifhig;
  // Taper branches: only the taps that land on bins 0..nto are evaluated.
  if (illow > 0) {
    const int j0 = std::max(1, iflow - nto), j1 = std::min(illow, iflow);
    for (int j = j0; j <= j1; ++j) fm[iflow - j] = hanning_at(j, illow, 2);
  }
  if (ilhig > 0) {
    const int j0 = std::max(1, 2 - ifhig), j1 = std::min(ilhig, nto + 2 - ifhig);
    for (int j = j0; j <= j1; ++j) fm[ifhig + j - 2] = hanning_at(j, ilhig, 2);
  }
  for (int j = std::max(iflow, 1); j <= std::min(ifhig, nto + 1); ++j) fm[j - 1] = 1.0f;
  for (int j = 0; j <= nto; ++j) w[j] = (double)(fm[j] + 0.0001f);
  return nto;
}

}  // namespace daw

namespace {

// Returns nto; fills w[0..nto] and applies the in-place fhig/lhig clamp.
int filter_weights(int nt, float dt, float* flow, float* fhig, float* llow, float* lhig,
                   std::vector<double>& w) {
  const int nto = filter_nto(nt);
  if (nto == 0) throw DawError{DAW_ERR_ARG, "filmartin2d: nt exceeds 65536"};
  std::vector<float> fm(nto + 1);
  w.resize(nto + 1);
  filter_weights_into(nt, dt, flow, fhig, llow, lhig, fm.data(), w.data());
  return nto;
}

void run_filter(daw_handle* h, const float* d_in, float* d_out, int nt, int nr, float dt,
                float band[4], const std::string& tag) {
  std::vector<double> w;
  const int nto = filter_weights(nt, dt, &band[0], &band[1], &band[2], &band[3], w);
  double* dw = h->pool.get_t<double>(tag + ".fw", w.size());
  upload(dw, w.data(), w.size() * sizeof(double), h->st);
  const size_t sb = filter_scratch_bytes(nr, nto);
  double* scratch = sb ? static_cast<double*>(h->pool.get(tag + ".fscr", sb)) : nullptr;
  filter_traces(d_in, d_out, nt, nr, nto, dw, scratch, h->st);
  check_launch("filmartin2d");
  h->tim.kernel_launches += 1;
  sync(h);  // w goes out of scope
}

// ---------------------------------------------------------------------------
// Shot preparation and the batched pipeline
// ---------------------------------------------------------------------------
// Device bytes of one shot.  win > 0 (less than nt): the history is kept in
// windows of win steps, and the states saved before the later windows plus
// stage B's own state take the place of the rest of the history.
size_t shot_bytes(const daw_handle* h, int nt, int nr, bool fp16, bool want_wf, int win = 0) {
  const Grid& g = h->g;
  const size_t state = (size_t)kStateFields * g.ext_elems() * 4;
  const size_t saved = (size_t)5 * g.ext_elems() * 4;
  const int hs = (win > 0 && win < nt) ? win : nt;
  size_t b = state;                                        // state
  b += hist_bytes_per_step(h, fp16) * (size_t)hs;          // history (window)
  b += (size_t)(hs + 1) * 3 * kAmaxSlots * 4;
  if (hs < nt) b += state + saved * (size_t)((nt + hs - 1) / hs - 1);  // stage-B state + saved states
  b += (size_t)(8 + 7) * nt * nr * 4;                      // MINRES + data arrays
  b += (size_t)6 * nt * std::max(h->ndatum, 1) * 4;        // datum gathers
  if (want_wf) b += g.int_elems() * (size_t)nt * 4;
  b += (size_t)nr * kTile * 12 * 2 + (size_t)g.n2e * 16 * 2;  // maps
  return b;
}

void prepare_shot(daw_handle* h, ShotCtx& c, const daw_shot_desc& d, int slot, bool want_wf,
                  bool fp16, bool forward_only = false, int win = 0) {
  const Grid& g = h->g;
  if (d.nt <= 0 || d.nrec < 0 || !d.s ||
      (d.nrec > 0 && (!d.rec_tab || (!forward_only && !d.dobs))))
    throw DawError{DAW_ERR_ARG, "shot " + std::to_string(d.shot) + ": bad descriptor"};
  c = ShotCtx();
  c.shot = d.shot;
  c.nt = d.nt;
  c.nr = d.nrec;
  c.nd = h->ndatum;
  c.type_src = d.type_src;
  c.type_rec = d.type_rec;
  c.mu = d.mu;
  c.maxiter = d.maxiter;
  c.rtol = d.rtol;
  std::memcpy(c.band, d.band, sizeof c.band);
  std::memcpy(c.src5, d.src_tab, sizeof c.src5);
  check_table(h, d.src_tab, 1, true, "src_tab");
  check_table(h, d.rec_tab, d.nrec, true, "rec_tab");
  const std::string p = "shot" + std::to_string(slot) + ".";
  c.tag = p;
  const size_t n = (size_t)d.nt * d.nrec, nd = (size_t)d.nt * std::max(h->ndatum, 1);
  float* a = h->pool.get_t<float>(p + "data", 7 * n + 5 * nd + d.nt);
  c.d_dobs = a; c.d_datar = a + n; c.d_deltadr = a + 2 * n; c.d_deltade = a + 3 * n;
  c.d_dataesc = a + 4 * n; c.d_datae = a + 5 * n;
  c.d_redF = a + 7 * n; c.d_redE = c.d_redF + nd; c.d_red = c.d_redE + nd;
  c.d_redf = c.d_red + nd;
  c.d_s = c.d_redf + nd + nd;
  upload(c.d_s, d.s, (size_t)d.nt * 4, h->st);
  if (d.dobs) upload(c.d_dobs, d.dobs, n * 4, h->st);
  c.rec = make_stations(h, h->pool, p + "rec", d.rec_tab, d.nrec);
  c.recmap = make_map(h, h->pool, p + "recmap", d.rec_tab, d.nrec);
  int32_t s5[5];
  std::memcpy(s5, d.src_tab, sizeof s5);
  c.src = make_stations(h, h->pool, p + "src", s5, 1);
  c.srcmap = make_map(h, h->pool, p + "srcmap", s5, 1);
  c.d_wf = want_wf ? h->pool.get_t<float>(p + "wf", g.int_elems() * (size_t)d.nt) : nullptr;
  c.d_ampT = h->pool.get_t<float>(p + "ampT", std::max<size_t>(n, 1));
  // forward-only shots keep no history: one step is allocated so that the
  // (unused) history tensor map describes real memory
  alloc_state(h, c, slot, forward_only ? 1 : d.nt, fp16, forward_only ? 0 : win);
}

// Device bytes of one forward-only shot (state, one history step, data, maps).
size_t shot_bytes_forward(const daw_handle* h, int nt, int nr) {
  const Grid& g = h->g;
  size_t b = (size_t)kStateFields * g.ext_elems() * 4 + hist_bytes_per_step(h, true) * 2 +
             2 * 3 * kAmaxSlots * 4;
  b += ((size_t)8 * nt * nr + (size_t)5 * nt * std::max(h->ndatum, 1) + nt) * 4;
  b += (size_t)nr * kTile * 12 * 2 + (size_t)g.n2e * 16 * 2;
  return b;
}

// Batched forward modelling (mode 0): many shots per launch, receiver data
// only.  At most kForwardBatch shots per batch.
constexpr int kForwardBatch = 64;
void run_forward_shots(daw_handle* h, int n, const daw_shot_desc* descs, float* const* sis) {
  require_model(h);
  if (n <= 0) return;
  int max_nt = 0, max_nr = 0;
  for (int i = 0; i < n; ++i) {
    max_nt = std::max(max_nt, descs[i].nt);
    max_nr = std::max(max_nr, descs[i].nrec);
    if (descs[i].nrec > 0 && !sis[i])
      throw DawError{DAW_ERR_ARG, "daw_submodeling_shots: output " + std::to_string(i) + " is NULL"};
  }
  int S = std::min(n, kForwardBatch);
  if (h->opt.fused) {
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const size_t per = shot_bytes_forward(h, max_nt, max_nr);
    const size_t avail = (size_t)((double)(free_b + h->pool.total) * 0.92);
    S = std::min<int>(S, (int)(avail / std::max<size_t>(per, 1)));
    if (S < 1) throw DawError{DAW_ERR_OOM, "HBM admission refused for a forward shot"};
  } else {
    S = 1;
  }
  if (h->opt.max_batch > 0) S = std::min(S, h->opt.max_batch);
  drop_graphs(h);
  for (int first = 0; first < n; first += S) {
    const int cnt = std::min(S, n - first);
    std::vector<ShotCtx> ctx(cnt);
    Batch b;
    b.slot0 = 0;
    b.no_datum = true;
    for (int i = 0; i < cnt; ++i) {
      prepare_shot(h, ctx[i], descs[first + i], i, false, h->opt.history_fp16 != 0, true);
      ctx[i].active = true;
      b.shots.push_back(&ctx[i]);
      b.max_nt = std::max(b.max_nt, ctx[i].nt);
      b.max_rec = std::max(b.max_rec, ctx[i].nr);
    }
    b.max_datum = 0;
    if (h->opt.fused)
      b.d_shots = static_cast<ShotDevice*>(h->pool.get("batch.shots0", cnt * sizeof(ShotDevice)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, h->st));
    batch_forward(h, b);
    CK(cudaEventRecord(e1, h->st));
    for (int i = 0; i < cnt; ++i)
      if (ctx[i].nr > 0)
        download(sis[first + i], ctx[i].d_datar, (size_t)ctx[i].nt * ctx[i].nr * sizeof(float),
                 h->st);
    sync(h);
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    h->tim.forward_ms += ms;
    h->tim.total_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(h);
  }
}

// An NVTX range around a scope (a pipeline phase), shown by nsys / ncu.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

void run_pipeline(daw_handle* h, Batch& b) {
  NvtxRange batch_range("daw shot batch");
  cudaStream_t st = h->st;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float ms = 0;
  b.max_nt = 0;
  b.max_rec = 0;
  for (ShotCtx* c : b.shots) {
    b.max_nt = std::max(b.max_nt, c->nt);
    b.max_rec = std::max(b.max_rec, c->nr);
    c->active = true;
  }
  b.max_datum = h->ndatum;
  if (h->opt.fused) {
    b.d_shots = static_cast<ShotDevice*>(
        h->pool.get("batch.shots" + std::to_string(b.slot0), b.shots.size() * sizeof(ShotDevice)));
  }
  // 1. forward modelling in c0 (sub_redatum_DAW.f90:82)
  nvtxRangePushA("daw forward");
  CK(cudaEventRecord(e0, st));
  batch_forward(h, b);
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(&ms, e0, e1));
  h->tim.forward_ms += ms;
  nvtxRangePop();
  // 2. time-reversed residuals (:103)
  for (ShotCtx* c : b.shots) residuals(c->d_dobs, c->d_datar, c->d_deltadr, c->nt, c->nr, st);
  check_launch("residuals");
  // 3. MINRES (:115)
  nvtxRangePushA("daw minres");
  if (h->opt.scalars_fp64)
    batch_minres<double>(h, b);
  else
    batch_minres<float>(h, b);
  nvtxRangePop();
  // 4. final extended-source simulation (:131) with the datum gather
  nvtxRangePushA("daw esource");
  for (ShotCtx* c : b.shots) {
    c->active = true;
    c->op_in = c->d_deltade;
    c->op_out = c->d_dataesc;
    c->op_reverse = 0;
    CK(cudaMemsetAsync(c->d_cost, 0, sizeof(double), st));
  }
  CK(cudaEventRecord(e0, st));
  batch_operator(h, b, true);
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(&ms, e0, e1));
  h->tim.esource_ms += ms;
  nvtxRangePop();
  // 5. DAW data and the redatumed data at the datum (:143-145, :238-240)
  nvtxRangePushA("daw datum and filter");
  CK(cudaEventRecord(e0, st));
  for (ShotCtx* c : b.shots) {
    vec_add(c->d_datar, c->d_dataesc, c->d_datae, (size_t)c->nt * c->nr, st);
    if (h->ndatum) {
      vec_add(c->d_redF, c->d_redE, c->d_red, (size_t)c->nt * h->ndatum, st);
      run_filter(h, c->d_red, c->d_redf, c->nt, h->ndatum, h->g.dt, c->band, c->tag);
    }
  }
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(&ms, e0, e1));
  h->tim.filter_ms += ms;
  nvtxRangePop();
  for (ShotCtx* c : b.shots) download(&c->cost, c->d_cost, sizeof(double), st);
  sync(h);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

void fetch_outputs(daw_handle* h, ShotCtx& c, daw_shot_out* o) {
  if (!o) return;
  const size_t n = (size_t)c.nt * c.nr, nd = (size_t)c.nt * h->ndatum;
  download(o->datar, c.d_datar, n * 4, h->st);
  download(o->deltadr, c.d_deltadr, n * 4, h->st);
  download(o->deltade, c.d_deltade, n * 4, h->st);
  download(o->dataesc, c.d_dataesc, n * 4, h->st);
  download(o->datae, c.d_datae, n * 4, h->st);
  if (h->ndatum) {
    download(o->redatumed_raw, c.d_red, nd * 4, h->st);
    download(o->redatumed, c.d_redf, nd * 4, h->st);
  }
  if (o->wavefield_exd && c.d_wf)
    download(o->wavefield_exd, c.d_wf, h->g.int_elems() * (size_t)c.nt * 4, h->st);
  double* user_log = o->minres.log;
  const int cap = o->minres.log_capacity;
  o->minres = c.info;
  o->minres.log = user_log;
  o->minres.log_capacity = cap;
  if (user_log && c.dlog && cap > 0) {
    const int nl = std::min(cap, c.info.nlog);
    download(user_log, c.dlog, (size_t)5 * nl * sizeof(double), h->st);
    o->minres.nlog = nl;
  }
  o->cost = c.cost;
  sync(h);
}

// Device bytes a batch may use: free memory plus the handle's reusable
// buffers, less a margin.
size_t admission_bytes(daw_handle* h) {
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  return (size_t)((double)(free_b + h->pool.total) * 0.92);
}

// Stage-A history window of a shot of nt steps (fused kernels only): 0 keeps
// the whole history; DAW_OPT_CHECKPOINT = K > 0 asks for windows of K steps;
// 0 picks the largest window that fits when the whole history does not.
int history_window(daw_handle* h, int nt, int nr, bool want_wf, size_t avail) {
  if (!h->opt.fused) return 0;
  const bool fp16 = h->opt.history_fp16 != 0;
  if (h->opt.checkpoint > 0) {
    // a requested window: its history plus ceil(nt/K) saved states must fit
    const int k = h->opt.checkpoint < nt ? h->opt.checkpoint : 0;
    const size_t need = shot_bytes(h, nt, nr, fp16, want_wf, k);
    if (need > avail)
      throw DawError{DAW_ERR_OOM, "HBM admission refused: one shot with history windows of " +
                                      std::to_string(h->opt.checkpoint) + " steps needs " +
                                      std::to_string(need) + " bytes, " + std::to_string(avail) +
                                      " available"};
    return k;
  }
  if (shot_bytes(h, nt, nr, fp16, want_wf) <= avail) return 0;
  for (int k = nt - 1; k >= 1; --k)
    if (shot_bytes(h, nt, nr, fp16, want_wf, k) <= avail) return k;
  throw DawError{DAW_ERR_OOM, "HBM admission refused: one shot needs " +
                                  std::to_string(shot_bytes(h, nt, nr, fp16, want_wf, 1)) +
                                  " bytes with the smallest history window, " +
                                  std::to_string(avail) + " available"};
}

// Shots of the next batch: the longest prefix of d[0..n) whose shots -- each
// with its own record length and receiver count -- fit the admission bound
// together (at most DAW_OPT_MAX_BATCH).  *win is the stage-A history window,
// set when the first shot alone needs one; a shot with a window runs alone.
int admit_batch(daw_handle* h, int n, const daw_shot_desc* d, bool want_wf, int* win) {
  *win = 0;
  if (!h->opt.fused || n <= 0) return std::min(n, 1);
  const size_t avail = admission_bytes(h);
  *win = history_window(h, d[0].nt, d[0].nrec, want_wf, avail);
  if (*win > 0) return 1;
  const bool fp16 = h->opt.history_fp16 != 0;
  const int cap = std::min(h->opt.max_batch > 0 ? std::min(n, h->opt.max_batch) : n, 64);
  size_t sum = 0;
  int s = 0;
  while (s < cap) {
    const size_t b = shot_bytes(h, d[s].nt, d[s].nrec, fp16, want_wf);
    if (sum + b > avail) break;
    sum += b;
    ++s;
  }
  if (s < 1)
    throw DawError{DAW_ERR_OOM, "HBM admission refused: one shot needs " +
                                    std::to_string(shot_bytes(h, d[0].nt, d[0].nrec, fp16, want_wf)) +
                                    " bytes, " + std::to_string(avail) + " available"};
  return s;
}

// Frees the per-slot buffers (state, histories, data, MINRES vectors, maps)
// of the previous batch, so that a batch of differently sized shots
// allocates exactly what it needs; graphs that point at them go first.
void release_slots(daw_handle* h) {
  drop_graphs(h);
  for (const char* p : {"slot", "shot", "mr", "batch."}) h->pool.release_prefix(p);
}

// Shots run longest record first, so that the shots of a batch (and of its
// launch groups) have similar record lengths and few time steps run with
// part of a batch idle; outputs go to their own descriptors' slots.
void run_shots(daw_handle* h, int n, const daw_shot_desc* descs, daw_shot_out* outs) {
  require_model(h);
  if (n <= 0) return;
  bool want_wf = false;
  for (int i = 0; i < n; ++i) want_wf |= (outs && outs[i].wavefield_exd != nullptr);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return descs[a].nt > descs[b].nt; });
  std::vector<daw_shot_desc> sorted(n);
  for (int i = 0; i < n; ++i) sorted[i] = descs[order[i]];
  for (int first = 0; first < n;) {
    release_slots(h);
    int win = 0;
    const int cnt = admit_batch(h, n - first, sorted.data() + first, want_wf, &win);
    std::vector<ShotCtx> ctx(cnt);
    Batch b;
    b.slot0 = 0;
    for (int i = 0; i < cnt; ++i) {
      const int o = order[first + i];
      prepare_shot(h, ctx[i], descs[o], i, outs && outs[o].wavefield_exd,
                   h->opt.history_fp16 != 0, false, win);
      b.shots.push_back(&ctx[i]);
    }
    run_pipeline(h, b);
    for (int i = 0; i < cnt; ++i) fetch_outputs(h, ctx[i], outs ? &outs[order[first + i]] : nullptr);
    drop_graphs(h);
    first += cnt;
  }
}

// Single-shot operator helpers for the reference-routine mirrors.
// forward_only: no stage-A history (one step allocated for the unused map).
ShotCtx& single_ctx(daw_handle* h, ShotCtx& c, int nt, const int32_t* ir, int nr, int type_rec,
                    bool want_wf, bool forward_only = false) {
  if (nt <= 0 || nr < 0 || (nr > 0 && !ir)) throw DawError{DAW_ERR_ARG, "bad nt/nr/table"};
  check_table(h, ir, nr, true, "ir");
  c = ShotCtx();
  c.nt = nt;
  c.nr = nr;
  c.type_rec = type_rec;
  const std::string p = "shot0.";
  c.tag = p;
  const size_t n = (size_t)nt * nr;
  float* a = h->pool.get_t<float>(p + "data", 7 * n + 5 * (size_t)nt * std::max(h->ndatum, 1) + nt);
  c.d_dobs = a; c.d_datar = a + n; c.d_deltadr = a + 2 * n; c.d_deltade = a + 3 * n;
  c.d_dataesc = a + 4 * n; c.d_datae = a + 5 * n;
  const size_t nd = (size_t)nt * std::max(h->ndatum, 1);
  c.d_redF = a + 7 * n; c.d_redE = c.d_redF + nd; c.d_red = c.d_redE + nd; c.d_redf = c.d_red + nd;
  c.d_s = c.d_redf + nd + nd;
  c.rec = make_stations(h, h->pool, p + "rec", ir, nr);
  c.recmap = make_map(h, h->pool, p + "recmap", ir, nr);
  c.d_wf = want_wf ? h->pool.get_t<float>(p + "wf", h->g.int_elems() * (size_t)nt) : nullptr;
  c.d_ampT = h->pool.get_t<float>(p + "ampT", std::max<size_t>(n, 1));
  const int win = forward_only ? 0 : history_window(h, nt, nr, want_wf, admission_bytes(h));
  alloc_state(h, c, 0, forward_only ? 1 : nt, h->opt.history_fp16 != 0 && h->opt.fused != 0, win);
  return c;
}

void apply_preset(Options& o, int preset) {
  o.preset = preset;
  if (preset == 0) {
    o.history_fp16 = 0; o.scalars_fp64 = 0; o.fused = 0; o.graph = 0;
  } else {
    o.history_fp16 = 1; o.scalars_fp64 = 1; o.fused = 1; o.graph = 1;
  }
}

template <typename F>
int guarded(daw_handle* h, F&& f) {
  if (!h) return DAW_ERR_ARG;
  try {
    CK(cudaSetDevice(h->device));
    f();
    h->err.clear();
    return DAW_OK;
  } catch (const DawError& e) {
    h->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    h->err = "host allocation failed";
    return DAW_ERR_OOM;
  } catch (const std::exception& e) {
    h->err = e.what();
    return DAW_ERR_ARG;
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* daw_version(void) { return "daw_b200 1.0 (sm_100a)"; }

int daw_create(daw_handle** out, int32_t device) {
  if (!out) return DAW_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return DAW_ERR_NODEV;
  }
  if (device < 0 || device >= count) return DAW_ERR_NODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    cudaGetLastError();
    return DAW_ERR_NODEV;
  }
  daw_handle* h = new (std::nothrow) daw_handle();
  if (!h) return DAW_ERR_OOM;
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return DAW_ERR_CUDA;
  }
  apply_preset(h->opt, 1);
  if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(h->st);
    delete h;
    return DAW_ERR_CUDA;
  }
  tma_prepare(&h->persist_p, &h->persist_v, h->persist_v_mode);
  step_prepare();
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
  for (int mode = 0; mode < 4; ++mode)
    for (int f = 0; f < 2; ++f)
      for (int t = 0; t < 2; ++t) h->step_occ[mode][f][t] = step_occupancy(mode, f != 0, t ? 32 : 16);
  cudaGetLastError();
  // The device set-up of daw_filmartin2d_noalloc, while memory is still free
  // (not fatal here: a failure is reported again by that entry point).
  if (filter_noalloc_prepare(nullptr, 0) != DAW_OK) cudaGetLastError();
  if (cudaMalloc(&h->d_err, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(h->d_err, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&h->d_qctr, 2 * sizeof(unsigned)) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(h->st);
    delete h;
    return DAW_ERR_CUDA;
  }
  *out = h;
  return DAW_OK;
}

void daw_destroy(daw_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->st);
  drop_graphs(h);
  h->pool.clear();
  h->model_pool.clear();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->d_err) cudaFree(h->d_err);
  if (h->d_qctr) cudaFree(h->d_qctr);
  cudaStreamDestroy(h->st);
  delete h;
}

const char* daw_last_error(const daw_handle* h) { return h ? h->err.c_str() : "null handle"; }

void daw_internal_set_error(daw_handle* h, const char* msg) {
  if (h) h->err = msg ? msg : "";
}

int daw_set_option(daw_handle* h, int32_t key, double value) {
  return guarded(h, [&] {
    const int v = (int)value;
    switch (key) {
      case DAW_OPT_PRESET:
        if (v != 0 && v != 1) throw DawError{DAW_ERR_ARG, "preset must be 0 or 1"};
        apply_preset(h->opt, v);
        break;
      case DAW_OPT_HISTORY: h->opt.history_fp16 = v ? 1 : 0; break;
      case DAW_OPT_SCALARS: h->opt.scalars_fp64 = v ? 1 : 0; break;
      case DAW_OPT_FUSED: h->opt.fused = v ? 1 : 0; break;
      case DAW_OPT_GRAPH: h->opt.graph = v ? 1 : 0; break;
      case DAW_OPT_SKIP_DEAD_OP: h->opt.skip_dead_op = v ? 1 : 0; break;
      case DAW_OPT_MAX_BATCH: h->opt.max_batch = std::max(0, v); break;
      case DAW_OPT_CHUNK:
        if (v != 0 && v != 1 && v != 2 && v != 4)
          throw DawError{DAW_ERR_ARG, "points per thread must be 1, 2 or 4 (0 = default)"};
        h->opt.chunk = v;
        break;
      case DAW_OPT_CHECKPOINT:
        if (v < 0) throw DawError{DAW_ERR_ARG, "history window must be >= 0 (0 = automatic)"};
        h->opt.checkpoint = v;
        break;
      case DAW_OPT_STEP_KERNEL:
        if (v < 0 || v > 2)
          throw DawError{DAW_ERR_ARG, "step kernel: 0 split, 1 one per step, 2 autotuned"};
        h->opt.step = v;
        break;
      case DAW_OPT_PDL: h->opt.pdl = v ? 1 : 0; break;
      case DAW_OPT_TILE_COLS:
        if (v != 0 && v != 16 && v != 32)
          throw DawError{DAW_ERR_ARG, "tile columns must be 16 or 32 (0 = autotuned)"};
        h->opt.tile_cols = v;
        break;
      case DAW_OPT_CTAS_PER_SM:
        if (v < 0 || v > 3) throw DawError{DAW_ERR_ARG, "CTAs per SM must be 0..3 (0 = autotuned)"};
        h->opt.ctas_per_sm = v;
        break;
      default: throw DawError{DAW_ERR_ARG, "unknown option"};
    }
    if (!h->opt.fused && h->opt.history_fp16)
      throw DawError{DAW_ERR_ARG, "FP16 histories need the fused kernels (DAW_OPT_FUSED=1)"};
    drop_graphs(h);
  });
}

int daw_get_option(const daw_handle* h, int32_t key, double* value) {
  if (!h || !value) return DAW_ERR_ARG;
  const Options& o = h->opt;
  switch (key) {
    case DAW_OPT_PRESET: *value = o.preset; break;
    case DAW_OPT_HISTORY: *value = o.history_fp16; break;
    case DAW_OPT_SCALARS: *value = o.scalars_fp64; break;
    case DAW_OPT_FUSED: *value = o.fused; break;
    case DAW_OPT_GRAPH: *value = o.graph; break;
    case DAW_OPT_SKIP_DEAD_OP: *value = o.skip_dead_op; break;
    case DAW_OPT_MAX_BATCH: *value = o.max_batch; break;
    case DAW_OPT_CHUNK: *value = o.chunk; break;
    case DAW_OPT_CHECKPOINT: *value = o.checkpoint; break;
    case DAW_OPT_STEP_KERNEL: *value = o.step; break;
    case DAW_OPT_PDL: *value = o.pdl; break;
    case DAW_OPT_TILE_COLS: *value = o.tile_cols; break;
    case DAW_OPT_CTAS_PER_SM: *value = o.ctas_per_sm; break;
    default: return DAW_ERR_ARG;
  }
  return DAW_OK;
}

namespace {

// Model set-up of daw_set_model / daw_set_model_rho (submodeling2.f90:54-113).
void set_model(daw_handle* h, const float* vp, const float* rho, int32_t n1, int32_t n2,
               int32_t npml, float hgrid, float dt, int32_t ofs) {
    if (!vp || n1 < 4 || n2 < 4 || npml < 1 || !(hgrid > 0) || !(dt > 0))
      throw DawError{DAW_ERR_ARG, "daw_set_model: bad arguments"};
    sync(h);
    drop_graphs(h);
    h->pool.clear();
    h->model_pool.clear();
    h->has_model = false;
    Grid g{};
    g.n1 = n1; g.n2 = n2; g.npml = npml;
    g.n1e = n1 + 2 * npml; g.n2e = n2 + 2 * npml;
    g.ld = (g.n1e + 63) / 64 * 64;  // fused kernels: 64 rows (32 lanes x float2) per warp
    g.ofs = ofs;
    g.h = hgrid; g.dt = dt; g.dtdx = dt / hgrid;
    std::vector<float> d1a, d1a1, d1b, d1b1, d2a, d2a1, d2b, d2b1;
    sponge_a(npml, n2, d2a, d2a1);
    sponge_b(npml, n2, d2b, d2b1);
    sponge_a(npml, n1, d1a, d1a1);
    sponge_b(npml, n1, d1b, d1b1);
    std::vector<float> bw1(g.n1e), bw2(g.n2e);
    for (int i = 0; i < g.n1e; ++i) bw1[i] = (g.dtdx * 1.0f) * d1b1[i];
    for (int i = 0; i < g.n2e; ++i) bw2[i] = (g.dtdx * 1.0f) * d2b1[i];
    // kappa = rho vp^2, formed in double (submodeling2.f90:1235), on the
    // edge-replicated extended grid (submodext); rho = 1 unless given.
    std::vector<float> kap(g.ext_elems(), 0.0f);
    std::vector<float> bue(rho ? g.ext_elems() : 0, 1.0f);
    for (int j = 0; j < g.n2e; ++j) {
      const int sj = std::min(std::max(j - npml, 0), n2 - 1);
      for (int i = 0; i < g.n1e; ++i) {
        const int si = std::min(std::max(i - npml, 0), n1 - 1);
        const double v = (double)vp[si + (size_t)n1 * sj];
        const size_t k = i + (size_t)g.ld * j;
        if (rho) {
          const float r = rho[si + (size_t)n1 * sj];
          kap[k] = (float)((double)r * (v * v));
          bue[k] = r > 0.f ? 1.0f / r : 1e10f;  // substagger :1236-1240
        } else {
          kap[k] = (float)(v * v);
        }
      }
    }
    // Buoyancy averaged onto the staggered grids (substagger :1248-1266):
    // bu1 between rows i1 and i1+1, bu2 between columns i2 and i2+1, then
    // the update coefficients dtdx*bu*damp*b1 (:107-108).  The last row of
    // bu1 and the last column of bu2 are never read by the stencil (updates
    // stop two points short of the edge); they keep bu itself.
    std::vector<float> rbw1, rbw2;
    if (rho) {
      rbw1.assign(g.ext_elems(), 0.0f);
      rbw2.assign(g.ext_elems(), 0.0f);
      for (int j = 0; j < g.n2e; ++j)
        for (int i = 0; i < g.n1e; ++i) {
          const size_t k = i + (size_t)g.ld * j;
          const float bu1 = i + 1 < g.n1e ? 0.5f * (bue[k + 1] + bue[k]) : bue[k];
          const float bu2 = j + 1 < g.n2e ? 0.5f * (bue[k + g.ld] + bue[k]) : bue[k];
          rbw1[k] = (g.dtdx * bu1) * d1b1[i];
          rbw2[k] = (g.dtdx * bu2) * d2b1[j];
        }
    }
    Pool& P = h->model_pool;
    ModelDev m;
    m.kap = P.get_t<float>("kap", kap.size());
    m.d1a = P.get_t<float>("d1a", g.n1e); m.d1b = P.get_t<float>("d1b", g.n1e);
    m.d1a1 = P.get_t<float>("d1a1", g.n1e); m.bw1 = P.get_t<float>("bw1", g.n1e);
    m.d2a = P.get_t<float>("d2a", g.n2e); m.d2b = P.get_t<float>("d2b", g.n2e);
    m.d2a1 = P.get_t<float>("d2a1", g.n2e); m.bw2 = P.get_t<float>("bw2", g.n2e);
    upload(m.kap, kap.data(), kap.size() * 4, h->st);
    upload(m.d1a, d1a.data(), g.n1e * 4, h->st); upload(m.d1b, d1b.data(), g.n1e * 4, h->st);
    upload(m.d1a1, d1a1.data(), g.n1e * 4, h->st); upload(m.bw1, bw1.data(), g.n1e * 4, h->st);
    upload(m.d2a, d2a.data(), g.n2e * 4, h->st); upload(m.d2b, d2b.data(), g.n2e * 4, h->st);
    upload(m.d2a1, d2a1.data(), g.n2e * 4, h->st); upload(m.bw2, bw2.data(), g.n2e * 4, h->st);
    std::vector<float4> prow(g.n1e), pcol(g.n2e);
    for (int i = 0; i < g.n1e; ++i) prow[i] = make_float4(d1a[i], d1a1[i], d1b[i], bw1[i]);
    for (int j = 0; j < g.n2e; ++j) pcol[j] = make_float4(d2a[j], d2a1[j], d2b[j], bw2[j]);
    m.prow = P.get_t<float4>("prow", g.n1e);
    m.pcol = P.get_t<float4>("pcol", g.n2e);
    upload(m.prow, prow.data(), g.n1e * sizeof(float4), h->st);
    upload(m.pcol, pcol.data(), g.n2e * sizeof(float4), h->st);
    if (rho) {
      m.rbw1 = P.get_t<float>("rbw1", rbw1.size());
      m.rbw2 = P.get_t<float>("rbw2", rbw2.size());
      m.rbue = P.get_t<float>("rbue", bue.size());
      upload(m.rbw1, rbw1.data(), rbw1.size() * 4, h->st);
      upload(m.rbw2, rbw2.data(), rbw2.size() * 4, h->st);
      upload(m.rbue, bue.data(), bue.size() * 4, h->st);
    }
    sync(h);
    h->g = g;
    h->md = m;
    h->has_model = true;
    if (h->ndatum > 0) h->datum = make_stations(h, h->model_pool, "datum", h->datum_tab.data(), h->ndatum);
}

}  // namespace

int daw_set_model(daw_handle* h, const float* vp, int32_t n1, int32_t n2, int32_t npml,
                  float hgrid, float dt, int32_t ofs) {
  return guarded(h, [&] { set_model(h, vp, nullptr, n1, n2, npml, hgrid, dt, ofs); });
}

int daw_set_model_rho(daw_handle* h, const float* vp, const float* rho, int32_t n1, int32_t n2,
                      int32_t npml, float hgrid, float dt, int32_t ofs) {
  return guarded(h, [&] { set_model(h, vp, rho, n1, n2, npml, hgrid, dt, ofs); });
}

int daw_set_datum(daw_handle* h, const int32_t* tab, int32_t n) {
  return guarded(h, [&] {
    require_model(h);
    check_table(h, tab, n, true, "datum_tab");
    h->datum_tab.assign(tab, tab + (size_t)n * 5);
    h->ndatum = n;
    h->datum = make_stations(h, h->model_pool, "datum", tab, n);
    drop_graphs(h);
  });
}

int daw_submodeling(daw_handle* h, const float* s, int32_t nt, const int32_t* is5,
                    int32_t type_src, int32_t type_rec, const int32_t* ir, int32_t nr,
                    float* sis, float* wavefield) {
  return guarded(h, [&] {
    require_model(h);
    if (!s || !is5 || !sis) throw DawError{DAW_ERR_ARG, "daw_submodeling: null argument"};
    ShotCtx c;
    single_ctx(h, c, nt, ir, nr, type_rec, wavefield != nullptr, true);
    c.type_src = type_src;
    check_table(h, is5, 1, true, "is");
    std::memcpy(c.src5, is5, sizeof c.src5);
    c.src = make_stations(h, h->pool, "shot0.src", is5, 1);
    c.srcmap = make_map(h, h->pool, "shot0.srcmap", is5, 1);
    upload(c.d_s, s, (size_t)nt * 4, h->st);
    Batch b;
    b.shots.push_back(&c);
    b.max_nt = nt;
    b.max_rec = nr;
    b.max_datum = 0;
    const int nd_save = h->ndatum;
    h->ndatum = 0;  // plain routine: no datum gather
    try {
      if (h->opt.fused) b.d_shots = static_cast<ShotDevice*>(h->pool.get("batch.shots0", sizeof(ShotDevice)));
      batch_forward(h, b);
    } catch (...) {
      h->ndatum = nd_save;
      throw;
    }
    h->ndatum = nd_save;
    download(sis, c.d_datar, (size_t)nt * nr * 4, h->st);
    if (wavefield) download(wavefield, c.d_wf, h->g.int_elems() * (size_t)nt * 4, h->st);
    sync(h);
    drop_graphs(h);
  });
}

static int operator_call(daw_handle* h, const float* res, int32_t nt, int32_t type_rec,
                         const int32_t* ir, int32_t nr, float* sis, float* wavefieldp,
                         double* cost, bool esource) {
  return guarded(h, [&] {
    require_model(h);
    if (!res || !sis) throw DawError{DAW_ERR_ARG, "null argument"};
    ShotCtx c;
    single_ctx(h, c, nt, ir, nr, type_rec, wavefieldp != nullptr);
    upload(c.d_deltadr, res, (size_t)nt * nr * 4, h->st);
    if (c.d_wf) CK(cudaMemsetAsync(c.d_wf, 0, h->g.int_elems() * (size_t)nt * 4, h->st));
    c.op_in = c.d_deltadr;
    c.op_out = c.d_dataesc;
    c.op_reverse = 0;
    CK(cudaMemsetAsync(c.d_cost, 0, sizeof(double), h->st));
    Batch b;
    b.shots.push_back(&c);
    b.max_nt = nt;
    b.max_rec = nr;
    b.max_datum = 0;
    const int nd_save = h->ndatum;
    h->ndatum = 0;
    try {
      if (h->opt.fused) b.d_shots = static_cast<ShotDevice*>(h->pool.get("batch.shots0", sizeof(ShotDevice)));
      batch_operator(h, b, esource);
    } catch (...) {
      h->ndatum = nd_save;
      throw;
    }
    h->ndatum = nd_save;
    download(sis, c.d_dataesc, (size_t)nt * nr * 4, h->st);
    if (wavefieldp) download(wavefieldp, c.d_wf, h->g.int_elems() * (size_t)nt * 4, h->st);
    if (cost) download(cost, c.d_cost, sizeof(double), h->st);
    sync(h);
    drop_graphs(h);
  });
}

int daw_esource_data(daw_handle* h, const float* res, int32_t nt, int32_t type_rec,
                     const int32_t* ir, int32_t nr, float* sis) {
  return operator_call(h, res, nt, type_rec, ir, nr, sis, nullptr, nullptr, false);
}

int daw_esource(daw_handle* h, const float* res, int32_t nt, int32_t type_rec, const int32_t* ir,
                int32_t nr, float* sis, float* wavefieldp, double* cost) {
  return operator_call(h, res, nt, type_rec, ir, nr, sis, wavefieldp, cost, true);
}

int daw_linear_minres(daw_handle* h, const float* deltadr, int32_t nt, int32_t type_rec,
                      const int32_t* ir, int32_t nr, float mu, int32_t maxiter, float rtol,
                      float* deltade, daw_minres_info* info) {
  return guarded(h, [&] {
    require_model(h);
    if (!deltadr || !deltade || maxiter < 0) throw DawError{DAW_ERR_ARG, "null argument"};
    ShotCtx c;
    single_ctx(h, c, nt, ir, nr, type_rec, false);
    c.mu = mu;
    c.maxiter = maxiter;
    c.rtol = rtol;
    upload(c.d_deltadr, deltadr, (size_t)nt * nr * 4, h->st);
    Batch b;
    b.shots.push_back(&c);
    b.max_nt = nt;
    b.max_rec = nr;
    b.max_datum = 0;
    const int nd_save = h->ndatum;
    h->ndatum = 0;
    try {
      if (h->opt.fused) b.d_shots = static_cast<ShotDevice*>(h->pool.get("batch.shots0", sizeof(ShotDevice)));
      if (h->opt.scalars_fp64)
        batch_minres<double>(h, b);
      else
        batch_minres<float>(h, b);
    } catch (...) {
      h->ndatum = nd_save;
      throw;
    }
    h->ndatum = nd_save;
    download(deltade, c.d_deltade, (size_t)nt * nr * 4, h->st);
    if (info) {
      double* lg = info->log;
      const int cap = info->log_capacity;
      *info = c.info;
      info->log = lg;
      info->log_capacity = cap;
      if (lg && cap > 0) {
        const int nl = std::min(cap, c.info.nlog);
        download(lg, c.dlog, (size_t)5 * nl * sizeof(double), h->st);
        info->nlog = nl;
      }
    }
    sync(h);
    drop_graphs(h);
  });
}

int daw_wavefield_resample(daw_handle* h, const float* wavefield, int32_t nt, const int32_t* ir,
                           int32_t nr, float* sis) {
  return guarded(h, [&] {
    require_model(h);
    if (!wavefield || !sis || nt <= 0 || nr < 0 || nt > 65535)
      throw DawError{DAW_ERR_ARG, "daw_wavefield_resample: bad arguments"};
    check_table(h, ir, nr, true, "ir");
    const Grid& g = h->g;
    const size_t ni = g.int_elems();
    float* wf = h->pool.get_t<float>("resample.wf", ni * (size_t)nt);
    float* out = h->pool.get_t<float>("resample.out", (size_t)nt * std::max(nr, 1));
    upload(wf, wavefield, ni * (size_t)nt * 4, h->st);
    StationsDev st = make_stations(h, h->pool, "resample.st", ir, nr);
    CK(cudaMemsetAsync(out, 0, (size_t)nt * std::max(nr, 1) * 4, h->st));
    hicks_gather(st, wf, g.n1, g.npml, g.n1, g.n2, out, nt, 0, nt, ni, h->st);
    check_launch("resample");
    download(sis, out, (size_t)nt * nr * 4, h->st);
    sync(h);
  });
}

int daw_filmartin2d(daw_handle* h, const float* in, int32_t nr, int32_t nt, float dt,
                    float* flow, float* fhig, float* llow, float* lhig, float* out) {
  return guarded(h, [&] {
    if (!in || !out || !flow || !fhig || !llow || !lhig || nr < 0 || nt <= 0 || !(dt > 0))
      throw DawError{DAW_ERR_ARG, "daw_filmartin2d: bad arguments"};
    const size_t n = (size_t)nt * nr;
    float* din = h->pool.get_t<float>("filt.in", std::max<size_t>(n, 1));
    float* dout = h->pool.get_t<float>("filt.out", std::max<size_t>(n, 1));
    upload(din, in, n * 4, h->st);
    float band[4] = {*flow, *fhig, *llow, *lhig};
    run_filter(h, din, dout, nt, nr, dt, band, "filt");
    *flow = band[0]; *fhig = band[1]; *llow = band[2]; *lhig = band[3];
    download(out, dout, n * 4, h->st);
    sync(h);
  });
}

int daw_submodeling_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs,
                          float* const* sis) {
  return guarded(h, [&] {
    if (n < 0 || (n > 0 && (!descs || !sis)))
      throw DawError{DAW_ERR_ARG, "daw_submodeling_shots: bad arguments"};
    run_forward_shots(h, n, descs, sis);
  });
}

int daw_shot(daw_handle* h, const daw_shot_desc* desc, daw_shot_out* out) {
  return daw_shots(h, 1, desc, out);
}

int daw_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs, daw_shot_out* outs) {
  return guarded(h, [&] {
    if (n < 0 || (n > 0 && !descs)) throw DawError{DAW_ERR_ARG, "daw_shots: bad arguments"};
    run_shots(h, n, descs, outs);
  });
}

int daw_selftest_wait_timeout(daw_handle* h) {
  if (!h) return DAW_ERR_ARG;
  const int rc = guarded(h, [&] {
    tma_wait_selftest(h->d_err, 1LL << 20, h->st);  // ~0.5 ms at the SM clock
    check_launch("wait self-test");
    sync(h);
    check_device_error(h);
  });
  return rc;
}

int daw_get_timing(const daw_handle* h, daw_timing* t) {
  if (!h || !t) return DAW_ERR_ARG;
  *t = h->tim;
  return DAW_OK;
}

void daw_reset_timing(daw_handle* h) {
  if (h) h->tim = daw_timing{};
}

// Device-resident runs: inputs copied once into pinned-free host copies, then
// uploaded to the device by daw_stage_shots' first batch; daw_run_staged runs
// the whole pipeline with no host<->device traffic of shot data.
int daw_admit_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs, int32_t* count,
                    int32_t* window) {
  return guarded(h, [&] {
    require_model(h);
    if (n <= 0 || !descs || !count) throw DawError{DAW_ERR_ARG, "daw_admit_shots: bad arguments"};
    int win = 0;
    *count = admit_batch(h, n, descs, false, &win);
    if (window) *window = win;
  });
}

int daw_stage_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs) {
  return guarded(h, [&] {
    require_model(h);
    if (n <= 0 || !descs) throw DawError{DAW_ERR_ARG, "daw_stage_shots: bad arguments"};
    int win = 0;
    h->staged_ready = 0;
    h->staged_ctx.clear();
    release_slots(h);
    const int S = admit_batch(h, n, descs, false, &win);
    if (S < n)
      throw DawError{DAW_ERR_OOM, "staged shots must fit one batch (" + std::to_string(S) +
                                      " admitted of " + std::to_string(n) + ")"};
    h->staged_ctx.assign(n, ShotCtx());
    for (int i = 0; i < n; ++i)
      prepare_shot(h, h->staged_ctx[i], descs[i], i, false, h->opt.history_fp16 != 0, false, win);
    sync(h);
    h->staged_ready = n;
  });
}

int daw_run_staged(daw_handle* h, float* ms_out) {
  return guarded(h, [&] {
    if (!h->staged_ready) throw DawError{DAW_ERR_STATE, "no staged shots"};
    Batch b;
    for (ShotCtx& c : h->staged_ctx) b.shots.push_back(&c);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, h->st));
    run_pipeline(h, b);
    CK(cudaEventRecord(e1, h->st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    h->tim.total_ms += ms;
    if (ms_out) *ms_out = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

int daw_fetch_shots(daw_handle* h, daw_shot_out* outs) {
  return guarded(h, [&] {
    if (!h->staged_ready) throw DawError{DAW_ERR_STATE, "no staged shots"};
    for (size_t i = 0; i < h->staged_ctx.size(); ++i) fetch_outputs(h, h->staged_ctx[i], outs ? &outs[i] : nullptr);
  });
}

}  // extern "C"
