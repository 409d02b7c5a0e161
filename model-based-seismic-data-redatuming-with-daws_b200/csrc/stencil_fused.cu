// Fused time-step kernels for a batch of shots sharing one model.
//
// Thread mapping: a warp owns 32 consecutive depth rows (i1, the contiguous
// axis, so every field access of a warp is one 128-byte line) and streams
// along `chunk` columns (i2).  Values along i2 live in a four-entry register
// queue (one new load per point); the depth neighbours come from warp
// shuffles, with the three halo values at the warp edges loaded directly.
// Each CTA (8 warps) belongs to one shot, so per-shot reductions stay
// CTA-local.
//
// Arithmetic of every update is the reference's, operation by operation
// (separately rounded FP32), so with FP32 histories the fused path reproduces
// the plain port bit for bit.  FP16 histories carry one power-of-two scale per
// (shot, step, field): the kernel that produces a field reduces max|x| over
// the interior; the next kernel, which reads the field anyway for its
// stencil, encodes and stores it -- no extra pass over the grid.
#include "fused.cuh"

namespace daw {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;

// Power-of-two scale exponent for a step/field: values are stored as
// x * 2^(15-E) with E chosen so that max|x| < 2^E, i.e. |stored| < 2^15.
__device__ __forceinline__ int amax_exponent(unsigned bits) {
  const int ef = (int)(bits >> 23);
  const int e = (ef == 0) ? -126 : ef - 126;
  return max(min(e, 120), -100);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

__device__ __forceinline__ unsigned warp_amax_slots(const unsigned* slots) {
  const unsigned v = slots[threadIdx.x & 31];
  return __reduce_max_sync(0xffffffffu, v);
}

template <bool FP16>
struct Hist;
template <>
struct Hist<true> {
  using T = __half;
  static __device__ __forceinline__ void put(void* base, size_t off, float v, float inv) {
    static_cast<__half*>(base)[off] = __float2half_rn(v * inv);
  }
  static __device__ __forceinline__ float get(const void* base, size_t off, float scale) {
    return __half2float(static_cast<const __half*>(base)[off]) * scale;
  }
};
template <>
struct Hist<false> {
  using T = float;
  static __device__ __forceinline__ void put(void* base, size_t off, float v, float) {
    static_cast<float*>(base)[off] = v;
  }
  static __device__ __forceinline__ float get(const void* base, size_t off, float) {
    return static_cast<const float*>(base)[off];
  }
};

struct WarpPos {
  int shot, rw, cc;
  bool valid;
};

__device__ __forceinline__ int stencil_blocks_per_shot(const Grid& g, int chunk) {
  const int nrw = (g.n1e + 31) / 32, ncc = (g.n2e + chunk - 1) / chunk;
  return (nrw * ncc + kWarps - 1) / kWarps;
}

__device__ __forceinline__ WarpPos warp_pos(const Grid& g, int chunk, int block) {
  const int nrw = (g.n1e + 31) / 32, ncc = (g.n2e + chunk - 1) / chunk;
  const int bps = (nrw * ncc + kWarps - 1) / kWarps;
  WarpPos w;
  w.shot = block / bps;
  const int lw = (block % bps) * kWarps + (threadIdx.x >> 5);
  w.valid = lw < nrw * ncc;
  w.rw = lw % nrw;
  w.cc = lw / nrw;
  return w;
}

// Per-point Hicks injection in gather form: contributions of the stations
// covering point (i1, i2) in station order (the reference's order).
__device__ __forceinline__ float inject_point(const InjMapDev& m, float v, int i1, int i2,
                                              int clo, int chi, float dt, float w,
                                              const float* amp, int amp_stride, int sign) {
  if (i1 < clo || i1 > chi) return v;
  const int r = __ldg(m.col_base + i2) + (i1 - clo);
  const int e0 = __ldg(m.rowptr + 2 * r), e1 = __ldg(m.rowptr + 2 * r + 1);
  for (int e = e0; e < e1; ++e) {
    const float a = __ldg(amp + (size_t)__ldg(m.sta + e) * amp_stride);
    const float term = fmul(fmul(fmul(__ldg(m.coef + e), dt), a), w);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  return v;
}

// ---------------------------------------------------------------------------
// Pressure kernel
// ---------------------------------------------------------------------------
template <int MODE, bool FP16>
__global__ void __launch_bounds__(kThreads)
    k_fused_p(Grid g, ModelDev m, FusedLaunch L, int it) {
  using H = Hist<FP16>;
  __shared__ unsigned red_p[kWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const WarpPos wp = warp_pos(g, L.chunk, blockIdx.x);
  if (wp.shot >= L.nshots) return;  // whole CTA
  const ShotDevice& sd = L.shots[wp.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (MODE == FM_STAGE_A ? it > nt + 1 : it > nt) return;
  const bool flush = (MODE == FM_STAGE_A) && it == nt + 1;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int fsrows = g.ofs == 1 ? npml + 1 : 0;
  const size_t nih = (size_t)L.n1h * g.n2;  // history field slice
  const int i1 = wp.rw * 32 + lane;
  const bool row_ok = wp.valid && i1 < n1e;
  const int i1p = i1 - npml;
  const bool row_int = row_ok && i1p >= 0 && i1p < g.n1;

  // Scales: stage A stores the v history of step it-1; stage B reads p of ic.
  float inv_vx = 1.f, inv_vz = 1.f, sc_p = 1.f;
  const int ic = nt - it + 1;
  if (FP16) {
    if (MODE == FM_STAGE_A && it >= 2) {
      const unsigned* a = sd.amax + ((size_t)(it - 2) * 3) * kAmaxSlots;
      inv_vx = pow2f(15 - amax_exponent(warp_amax_slots(a + kAmaxSlots)));
      inv_vz = pow2f(15 - amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + ((size_t)(ic - 1) * 3) * kAmaxSlots;
      sc_p = pow2f(amax_exponent(warp_amax_slots(a)) - 15);
    }
  }
  const float dtdx = g.dtdx, dt = g.dt;
  const float mdt = fmul(-1.0f, dt);
  const float d1a = row_ok ? __ldg(m.d1a + i1) : 0.f;
  const float d1a1 = row_ok ? __ldg(m.d1a1 + i1) : 0.f;
  const int src_lo = (MODE == FM_STAGE_B_ES) ? 1 : 0;
  const int src_hi1 = (MODE == FM_STAGE_B_ES) ? g.n1 - 1 : g.n1;
  const int src_hi2 = (MODE == FM_STAGE_B_ES) ? g.n2 - 1 : g.n2;
  const bool do_inj = (MODE == FM_STAGE_A) || (MODE == FM_FWD && sd.type_src == 0);
  const float* amp = (MODE == FM_FWD) ? sd.amp + (it - 1) : sd.amp + (it - 1);
  const void* hist = sd.hist;
  float lmax = 0.f;

  const int c0 = wp.cc * L.chunk;
  const int c1 = min(c0 + L.chunk, n2e);
  const float* __restrict__ vx = sd.vx;
  const float* __restrict__ vz = sd.vz;
  float* __restrict__ px = sd.px;
  float* __restrict__ pz = sd.pz;
  float* __restrict__ pp = sd.p;
  const float* __restrict__ kap = m.kap;
  // register queue along i2: q0 = vx[i2-2] .. q3 = vx[i2+1]
  auto ldvx = [&](int c) -> float {
    return (wp.valid && c >= 0 && c < n2e) ? vx[i1 + (size_t)ld * c] : 0.f;
  };
  float q0 = ldvx(c0 - 2), q1 = ldvx(c0 - 1), q2 = ldvx(c0);
  for (int i2 = c0; i2 < c1; ++i2) {
    const float q3 = ldvx(i2 + 1);
    const size_t k = i1 + (size_t)ld * i2;
    const float vzc = wp.valid ? vz[k] : 0.f;
    const int i2p = i2 - npml;
    const bool interior = row_int && i2p >= 0 && i2p < g.n2;
    if (MODE == FM_STAGE_A && it >= 2 && interior) {
      // deferred velocity history of step it-1 (the current vx, vz)
      const size_t o = ((size_t)(it - 2) * 3) * nih + i1p + (size_t)L.n1h * i2p;
      H::put(sd.hist, o + nih, q2, inv_vx);
      H::put(sd.hist, o + 2 * nih, vzc, inv_vz);
    }
    if (!flush) {
      float vzm1 = __shfl_up_sync(0xffffffffu, vzc, 1);
      float vzm2 = __shfl_up_sync(0xffffffffu, vzc, 2);
      float vzp1 = __shfl_down_sync(0xffffffffu, vzc, 1);
      const bool upd = row_ok && i1 >= 2 && i1 < hi1 && i2 >= 2 && i2 < hi2;
      if (upd) {
        if (lane == 0) { vzm1 = vz[k - 1]; vzm2 = vz[k - 2]; }
        if (lane == 1) vzm2 = vz[k - 2];
        if (lane == 31) vzp1 = vz[k + 1];
      }
      if (row_ok) {
        float pxv = px[k], pzv = pz[k];
        if (upd) {
          const float der2 = dminus(q0, q1, q2, q3);
          const float der1 = dminus(vzm2, vzm1, vzc, vzp1);
          const float kd = fmul(dtdx, kap[k]);
          const float kw2 = fmul(kd, __ldg(m.d2a1 + i2));
          const float kw1 = fmul(kd, d1a1);
          const float ax = fmul(__ldg(m.d2a + i2), pxv), bx = fmul(kw2, der2);
          const float az = fmul(d1a, pzv), bz = fmul(kw1, der1);
          const bool fwd = (MODE != FM_STAGE_A);
          pxv = fwd ? fadd(ax, bx) : fsub(ax, bx);
          pzv = fwd ? fadd(az, bz) : fsub(az, bz);
        }
        if (do_inj) {
          const int clo = __ldg(sd.inj.col_lo + i2), chi = __ldg(sd.inj.col_hi + i2);
          if (i1 >= clo && i1 <= chi)
            pxv = inject_point(sd.inj, pxv, i1, i2, clo, chi, dt, kap[k], amp, sd.amp_stride,
                               MODE == FM_FWD ? +1 : -1);
        }
        if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
          if (interior && i1p >= src_lo && i1p < src_hi1 && i2p >= src_lo && i2p < src_hi2) {
            const size_t o = ((size_t)(ic - 1) * 3) * nih + i1p + (size_t)L.n1h * i2p;
            const float hv = H::get(hist, o, sc_p);
            pxv = fadd(pxv, fmul(fmul(mdt, hv), kap[k]));
          }
        }
        const float pv = i1 < fsrows ? 0.f : fadd(pxv, pzv);
        px[k] = pxv;
        pz[k] = pzv;
        pp[k] = pv;
        if (interior) {
          if (MODE == FM_STAGE_A) lmax = fmaxf(lmax, fabsf(pv));
          if (MODE == FM_FWD && sd.wf && sd.type_rec == 0)
            sd.wf[(size_t)(it - 1) * g.int_elems() + i1p + (size_t)g.n1 * i2p] = pv;
          if (MODE == FM_STAGE_B_ES && sd.wf && sd.type_rec == 0) {
            float* w = sd.wf + (size_t)(it - 1) * g.int_elems() + i1p + (size_t)g.n1 * i2p;
            *w = fadd(*w, pv);
          }
        }
      }
    }
    q0 = q1;
    q1 = q2;
    q2 = q3;
  }
  if (MODE == FM_STAGE_A && !flush) {
    // max |p| of step it over the interior -> amax slot (CTA-local first)
    unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(lmax));
    if (lane == 0) red_p[wib] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned r = 0;
      for (int w = 0; w < kWarps; ++w) r = max(r, red_p[w]);
      if (r) atomicMax(sd.amax + ((size_t)(it - 1) * 3) * kAmaxSlots + (blockIdx.x % kAmaxSlots), r);
    }
  }
}

// Sequential Hicks gather of one station by one warp (lane 0 sums in the
// reference's i1-outer order), used by the gather CTAs of k_fused_v.
__device__ float warp_gather(float* prod, const StationsDev& st, int s, const float* origin,
                             int ld, int shift, int hi1, int hi2) {
  const int lane = threadIdx.x & 31;
  const int ix1 = __ldg(st.ix1 + s) - shift, ix2 = __ldg(st.ix2 + s) - shift;
  const int r1a = max(1 - ix1, -kRad), r1b = min(hi1 - ix1, kRad);
  const int r2a = max(1 - ix2, -kRad), r2b = min(hi2 - ix2, kRad);
  const float* tile = st.tile + (size_t)s * kTile;
  for (int t = lane; t < kTile; t += 32) {
    const int a = t / kTap - kRad, b = t % kTap - kRad;
    float v = 0.f;
    if (a >= r1a && a <= r1b && b >= r2a && b <= r2b)
      v = fmul(__ldg(tile + (a + kRad) + kTap * (b + kRad)),
               origin[(ix1 + a - 1) + (size_t)ld * (ix2 + b - 1)]);
    prod[t] = v;
  }
  __syncwarp();
  float acc = 0.f;
  if (lane == 0)
    for (int a = r1a; a <= r1b; ++a)
      for (int b = r2a; b <= r2b; ++b) acc = fadd(acc, prod[(a + kRad) * kTap + (b + kRad)]);
  __syncwarp();
  return acc;
}

// ---------------------------------------------------------------------------
// Velocity kernel (+ gathers in the first `ngb` CTAs)
// ---------------------------------------------------------------------------
template <int MODE, bool FP16>
__global__ void __launch_bounds__(kThreads)
    k_fused_v(Grid g, ModelDev m, FusedLaunch L, int it, int ngb_per_shot) {
  using H = Hist<FP16>;
  __shared__ unsigned red_v[2][kWarps];
  __shared__ float prod[kWarps][kTile];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int ngb = ngb_per_shot * L.nshots;
  if ((int)blockIdx.x < ngb) {
    // ---- gather CTAs: receivers then datum stations of one shot
    if (MODE == FM_STAGE_A) return;
    const int shot = blockIdx.x / ngb_per_shot;
    const ShotDevice& sd = L.shots[shot];
    if (!sd.active || it > sd.nt || sd.type_rec != 0) return;
    const int s = (blockIdx.x % ngb_per_shot) * kWarps + wib;
    if (s < sd.rec.n) {
      if (sd.out) {
        const float v = warp_gather(prod[wib], sd.rec, s, sd.p, g.ld, 0, g.n1e, g.n2e);
        const int row = sd.out_reverse ? sd.nt - it : it - 1;
        if (lane == 0) sd.out[row + (size_t)sd.nt * s] = v;
      }
    } else if (s - sd.rec.n < sd.datum.n && sd.red &&
               (MODE == FM_FWD || MODE == FM_STAGE_B_ES)) {
      const int d = s - sd.rec.n;
      const float v = warp_gather(prod[wib], sd.datum, d, sd.p + g.npml + (size_t)g.ld * g.npml,
                                  g.ld, g.npml, g.n1, g.n2);
      if (lane == 0) sd.red[(it - 1) + (size_t)sd.nt * d] = v;
    }
    return;
  }
  const WarpPos wp = warp_pos(g, L.chunk, blockIdx.x - ngb);
  if (wp.shot >= L.nshots) return;
  const ShotDevice& sd = L.shots[wp.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (it > nt) return;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const size_t nih = (size_t)L.n1h * g.n2;
  const int i1 = wp.rw * 32 + lane;
  const bool row_ok = wp.valid && i1 < n1e;
  const int i1p = i1 - npml;
  const bool row_int = row_ok && i1p >= 0 && i1p < g.n1;
  const int ic = nt - it + 1;
  float inv_p = 1.f, sc_vx = 1.f, sc_vz = 1.f;
  if (FP16) {
    if (MODE == FM_STAGE_A) {
      const unsigned* a = sd.amax + ((size_t)(it - 1) * 3) * kAmaxSlots;
      inv_p = pow2f(15 - amax_exponent(warp_amax_slots(a)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + ((size_t)(ic - 1) * 3) * kAmaxSlots;
      sc_vx = pow2f(amax_exponent(warp_amax_slots(a + kAmaxSlots)) - 15);
      sc_vz = pow2f(amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)) - 15);
    }
  }
  const float dt = g.dt;
  const float mdt = fmul(-1.0f, dt);
  const float d1b = row_ok ? __ldg(m.d1b + i1) : 0.f;
  const float bw1 = row_ok ? __ldg(m.bw1 + i1) : 0.f;
  const bool fs_src_row = g.ofs == 1 && i1 == npml;      // writes vz(npml) too
  const bool fs_dst_row = g.ofs == 1 && i1 == npml - 1;  // vz overwritten
  const bool do_inj = (MODE == FM_FWD) && sd.type_src == 1;
  float lmx = 0.f, lmz = 0.f;
  const int c0 = wp.cc * L.chunk;
  const int c1 = min(c0 + L.chunk, n2e);
  const float* __restrict__ pp = sd.p;
  float* __restrict__ vx = sd.vx;
  float* __restrict__ vz = sd.vz;
  auto ldp = [&](int c) -> float {
    return (wp.valid && c >= 0 && c < n2e) ? pp[i1 + (size_t)ld * c] : 0.f;
  };
  // register queue along i2: q0 = p[i2-1] .. q3 = p[i2+2]
  float q0 = ldp(c0 - 1), q1 = ldp(c0), q2 = ldp(c0 + 1);
  for (int i2 = c0; i2 < c1; ++i2) {
    const float q3 = ldp(i2 + 2);
    const size_t k = i1 + (size_t)ld * i2;
    const float pc = q1;
    float pm1 = __shfl_up_sync(0xffffffffu, pc, 1);
    float pp1 = __shfl_down_sync(0xffffffffu, pc, 1);
    float pp2 = __shfl_down_sync(0xffffffffu, pc, 2);
    const bool upd = row_ok && i1 >= 2 && i1 < hi1 && i2 >= 2 && i2 < hi2;
    if (upd) {
      if (lane == 0) pm1 = pp[k - 1];
      if (lane == 31) pp1 = pp[k + 1];
      if (lane >= 30) pp2 = pp[k + 2];
    }
    const int i2p = i2 - npml;
    const bool interior = row_int && i2p >= 0 && i2p < g.n2;
    if (row_ok) {
      float vxv = vx[k], vzv = vz[k];
      if (upd) {
        const float der2 = dplus(q0, q1, q2, q3);
        const float der1 = dplus(pm1, pc, pp1, pp2);
        const float ax = fmul(__ldg(m.d2b + i2), vxv), bx = fmul(__ldg(m.bw2 + i2), der2);
        const float az = fmul(d1b, vzv), bz = fmul(bw1, der1);
        const bool fwd = (MODE != FM_STAGE_A);
        vxv = fwd ? fadd(ax, bx) : fsub(ax, bx);
        vzv = fwd ? fadd(az, bz) : fsub(az, bz);
      }
      if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
        if (interior) {
          const size_t o = ((size_t)(ic - 1) * 3) * nih + i1p + (size_t)L.n1h * i2p;
          vxv = fadd(vxv, fmul(fmul(mdt, H::get(sd.hist, o + nih, sc_vx)), 1.0f));
          vzv = fadd(vzv, fmul(fmul(mdt, H::get(sd.hist, o + 2 * nih, sc_vz)), 1.0f));
        }
      }
      if (do_inj) {
        const int clo = __ldg(sd.inj.col_lo + i2), chi = __ldg(sd.inj.col_hi + i2);
        if (i1 >= clo && i1 <= chi)
          vzv = inject_point(sd.inj, vzv, i1, i2, clo, chi, dt, 1.0f, sd.amp + (it - 1),
                             sd.amp_stride, +1);
      }
      vx[k] = vxv;
      if (!fs_dst_row) vz[k] = vzv;
      if (fs_src_row) vz[k - 1] = vzv;
      if (MODE == FM_STAGE_A && interior) {
        const size_t o = ((size_t)(it - 1) * 3) * nih + i1p + (size_t)L.n1h * i2p;
        H::put(sd.hist, o, pc, inv_p);  // deferred pressure history of step it
        lmx = fmaxf(lmx, fabsf(vxv));
        lmz = fmaxf(lmz, fabsf(vzv));
      }
    }
    q0 = q1;
    q1 = q2;
    q2 = q3;
  }
  if (MODE == FM_STAGE_A) {
    const unsigned bx = __reduce_max_sync(0xffffffffu, __float_as_uint(lmx));
    const unsigned bz = __reduce_max_sync(0xffffffffu, __float_as_uint(lmz));
    if (lane == 0) {
      red_v[0][wib] = bx;
      red_v[1][wib] = bz;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned rx = 0, rz = 0;
      for (int w = 0; w < kWarps; ++w) {
        rx = max(rx, red_v[0][w]);
        rz = max(rz, red_v[1][w]);
      }
      unsigned* a = sd.amax + ((size_t)(it - 1) * 3) * kAmaxSlots + (blockIdx.x % kAmaxSlots);
      if (rx) atomicMax(a + kAmaxSlots, rx);
      if (rz) atomicMax(a + 2 * kAmaxSlots, rz);
    }
  }
}

// Sum of 0.5*sp^2 over a stage-A history (the esource `cost`).
template <bool FP16>
__global__ void k_hist_cost(const void* hist, const unsigned* amax, int nt, int n1, int n2,
                            int inner_ld, size_t field_stride, double* out) {
  __shared__ double sh[256];
  double acc = 0;
  const size_t per = (size_t)n1 * n2;
  const size_t total = per * nt;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(q / per);
    const size_t r = q % per;
    const int i1 = (int)(r % n1), i2 = (int)(r / n1);
    const size_t o = (size_t)it * 3 * field_stride + i1 + (size_t)inner_ld * i2;
    float sc = 1.f;
    if (FP16) {
      unsigned b = 0;
      for (int s = 0; s < kAmaxSlots; ++s) b = max(b, amax[(size_t)it * 3 * kAmaxSlots + s]);
      sc = pow2f(amax_exponent(b) - 15);
    }
    const double v = (double)Hist<FP16>::get(hist, o, sc);
    acc += 0.5 * v * v;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, sh[0]);
}

template <int MODE>
void launch_p(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, int blocks,
              cudaStream_t st) {
  if (L.hist_fp16)
    k_fused_p<MODE, true><<<blocks, kThreads, 0, st>>>(g, m, L, it);
  else
    k_fused_p<MODE, false><<<blocks, kThreads, 0, st>>>(g, m, L, it);
}

template <int MODE>
void launch_v(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, int blocks,
              int ngbps, cudaStream_t st) {
  if (L.hist_fp16)
    k_fused_v<MODE, true><<<blocks, kThreads, 0, st>>>(g, m, L, it, ngbps);
  else
    k_fused_v<MODE, false><<<blocks, kThreads, 0, st>>>(g, m, L, it, ngbps);
}

int host_bps(const Grid& g, int chunk) {
  const int nrw = (g.n1e + 31) / 32, ncc = (g.n2e + chunk - 1) / chunk;
  return (nrw * ncc + kWarps - 1) / kWarps;
}

}  // namespace

int fused_warps(const Grid& g, int chunk) { return host_bps(g, chunk) * kWarps; }

void fused_p_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st) {
  const int blocks = host_bps(g, L.chunk) * L.nshots;
  switch (mode) {
    case FM_FWD: launch_p<FM_FWD>(g, m, L, it, blocks, st); break;
    case FM_STAGE_A: launch_p<FM_STAGE_A>(g, m, L, it, blocks, st); break;
    case FM_STAGE_B: launch_p<FM_STAGE_B>(g, m, L, it, blocks, st); break;
    default: launch_p<FM_STAGE_B_ES>(g, m, L, it, blocks, st); break;
  }
}

void fused_v_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st) {
  const int stations = (mode == FM_STAGE_A) ? 0 : L.max_rec + L.max_datum;
  const int ngbps = (stations + kWarps - 1) / kWarps;
  const int blocks = (host_bps(g, L.chunk) + ngbps) * L.nshots;
  switch (mode) {
    case FM_FWD: launch_v<FM_FWD>(g, m, L, it, blocks, ngbps, st); break;
    case FM_STAGE_A: launch_v<FM_STAGE_A>(g, m, L, it, blocks, ngbps, st); break;
    case FM_STAGE_B: launch_v<FM_STAGE_B>(g, m, L, it, blocks, ngbps, st); break;
    default: launch_v<FM_STAGE_B_ES>(g, m, L, it, blocks, ngbps, st); break;
  }
}

void history_cost(const void* hist, int fp16, const unsigned* amax, int nt, int n1, int n2,
                  int inner_ld, size_t field_stride, double* out, cudaStream_t st) {
  const int blocks = 148 * 4;
  if (fp16)
    k_hist_cost<true><<<blocks, 256, 0, st>>>(hist, amax, nt, n1, n2, inner_ld, field_stride, out);
  else
    k_hist_cost<false><<<blocks, 256, 0, st>>>(hist, amax, nt, n1, n2, inner_ld, field_stride, out);
}

}  // namespace daw
