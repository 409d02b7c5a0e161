// Fused time-step kernels for a batch of shots sharing one model.
//
// Mapping: a CTA of 8 warps covers 32 consecutive depth rows (i1, the
// contiguous axis: every warp access is one 128-byte line) and 8*NP columns;
// each thread owns one row and NP consecutive columns.  Every load of a
// thread -- its own values, the i2 neighbours of the staggered stencil
// (columns c-2..c+NP) and the i1 neighbours (rows i1-2..i1+2, L1 hits) -- is
// independent and issued before any arithmetic, so each warp keeps many
// lines in flight: the 2-D state of a 751x2301 shot (~48 MB) lives in L2
// and the kernels are bound by L2/L1 latency hiding, not by a serial loop.
//
// Arithmetic of every update is the reference's, operation by operation
// (separately rounded FP32), so with FP32 histories the fused path reproduces
// the plain port and the FP32 oracle bit for bit.  FP16 histories carry one
// power-of-two scale per (shot, step, field): the kernel that produces a
// field reduces max|x| over the interior; the next kernel, which reads the
// field anyway for its stencil, encodes and stores it -- no extra pass.
#include "fused.cuh"

namespace daw {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;

// Power-of-two scale exponent E of a step/field with max|x| < 2^E; values are
// stored as x * 2^(15-E), so |stored| < 2^15 < 65504.
__device__ __forceinline__ int amax_exponent(unsigned bits) {
  const int ef = (int)(bits >> 23);
  const int e = (ef == 0) ? -126 : ef - 126;
  return max(min(e, 120), -100);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

__device__ __forceinline__ unsigned warp_amax_slots(const unsigned* slots) {
  return __reduce_max_sync(0xffffffffu, slots[threadIdx.x & 31]);
}

template <bool FP16>
struct Hist;
template <>
struct Hist<true> {
  static __device__ __forceinline__ void put(void* base, size_t off, float v, float inv) {
    static_cast<__half*>(base)[off] = __float2half_rn(v * inv);
  }
  static __device__ __forceinline__ float get(const void* base, size_t off, float scale) {
    return __half2float(static_cast<const __half*>(base)[off]) * scale;
  }
};
template <>
struct Hist<false> {
  static __device__ __forceinline__ void put(void* base, size_t off, float v, float) {
    static_cast<float*>(base)[off] = v;
  }
  static __device__ __forceinline__ float get(const void* base, size_t off, float) {
    return static_cast<const float*>(base)[off];
  }
};

struct Tile {
  int shot, i1, c0;
};

template <int NP>
__device__ __forceinline__ int blocks_per_shot(const Grid& g) {
  return ((g.n1e + 31) >> 5) * ((g.n2e + kWarps * NP - 1) / (kWarps * NP));
}

template <int NP>
__device__ __forceinline__ Tile tile_of(const Grid& g, int block) {
  const int nrb = (g.n1e + 31) >> 5;
  const int bps = blocks_per_shot<NP>(g);
  Tile t;
  t.shot = block / bps;
  const int lb = block % bps;
  t.i1 = (lb % nrb) * 32 + (threadIdx.x & 31);
  t.c0 = ((lb / nrb) * kWarps + (threadIdx.x >> 5)) * NP;
  return t;
}

// Hicks injection in gather form at one point: the contributions of the
// stations covering it, in station order (the reference's order).
__device__ __forceinline__ float inject_point(const InjMapDev& m, float v, int i1, int i2,
                                              float dt, float w, const float* amp,
                                              int amp_stride, int sign) {
  const int clo = __ldg(m.col_lo + i2);
  if (i1 < clo || i1 > __ldg(m.col_hi + i2)) return v;
  const int r = __ldg(m.col_base + i2) + (i1 - clo);
  const int e0 = __ldg(m.rowptr + 2 * r), e1 = __ldg(m.rowptr + 2 * r + 1);
  for (int e = e0; e < e1; ++e) {
    const float a = __ldg(amp + (size_t)__ldg(m.sta + e) * amp_stride);
    const float term = fmul(fmul(fmul(__ldg(m.coef + e), dt), a), w);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  return v;
}

__device__ __forceinline__ void cta_amax(unsigned* red, unsigned v, unsigned* slot) {
  const unsigned b = __reduce_max_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned r = 0;
    for (int w = 0; w < kWarps; ++w) r = max(r, red[w]);
    if (r) atomicMax(slot, r);
  }
}

// ---------------------------------------------------------------------------
// Pressure kernel
// ---------------------------------------------------------------------------
template <int MODE, bool FP16, int NP>
__global__ void __launch_bounds__(kThreads)
    k_fused_p(Grid g, ModelDev m, FusedLaunch L, int it) {
  using H = Hist<FP16>;
  __shared__ unsigned red[kWarps];
  const Tile t = tile_of<NP>(g, blockIdx.x);
  if (t.shot >= L.nshots) return;  // CTA-uniform
  const ShotDevice& sd = L.shots[t.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (MODE == FM_STAGE_A ? it > nt + 1 : it > nt) return;
  const bool flush = (MODE == FM_STAGE_A) && it == nt + 1;  // store v history of step nt only
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int fsrows = g.ofs == 1 ? npml + 1 : 0;
  const size_t nih = (size_t)L.n1h * g.n2;
  const int i1 = t.i1;
  const bool row_ok = i1 < n1e;
  const int i1p = i1 - npml;
  const bool row_int = row_ok && i1p >= 0 && i1p < g.n1;
  const bool row_upd = row_ok && i1 >= 2 && i1 < hi1;
  const int ic = nt - it + 1;

  float inv_vx = 1.f, inv_vz = 1.f, sc_p = 1.f;
  if (FP16) {
    if (MODE == FM_STAGE_A && it >= 2) {
      const unsigned* a = sd.amax + (size_t)(it - 2) * 3 * kAmaxSlots;
      inv_vx = pow2f(15 - amax_exponent(warp_amax_slots(a + kAmaxSlots)));
      inv_vz = pow2f(15 - amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + (size_t)(ic - 1) * 3 * kAmaxSlots;
      sc_p = pow2f(amax_exponent(warp_amax_slots(a)) - 15);
    }
  }
  const float* __restrict__ vx = sd.vx;
  const float* __restrict__ vz = sd.vz;

  // ---- loads (all independent)
  float qx[NP + 3];  // vx at columns c0-2 .. c0+NP
#pragma unroll
  for (int j = 0; j < NP + 3; ++j) {
    const int c = t.c0 - 2 + j;
    qx[j] = (row_ok && c >= 0 && c < n2e) ? vx[i1 + (size_t)ld * c] : 0.f;
  }
  float z0[NP], zm1[NP], zm2[NP], zp1[NP], pxv[NP], pzv[NP], kv[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    const bool ok = row_ok && c < n2e;
    const size_t k = i1 + (size_t)ld * c;
    z0[j] = ok ? vz[k] : 0.f;
    const bool upd = ok && row_upd && c >= 2 && c < hi2 && !flush;
    zm2[j] = upd ? vz[k - 2] : 0.f;
    zm1[j] = upd ? vz[k - 1] : 0.f;
    zp1[j] = upd ? vz[k + 1] : 0.f;
    pxv[j] = (ok && !flush) ? sd.px[k] : 0.f;
    pzv[j] = (ok && !flush) ? sd.pz[k] : 0.f;
    kv[j] = (ok && !flush) ? __ldg(m.kap + k) : 0.f;
  }
  const float dtdx = g.dtdx, dt = g.dt, mdt = fmul(-1.0f, dt);
  const float d1a = row_ok ? __ldg(m.d1a + i1) : 0.f;
  const float d1a1 = row_ok ? __ldg(m.d1a1 + i1) : 0.f;
  const bool do_inj = (MODE == FM_STAGE_A) || (MODE == FM_FWD && sd.type_src == 0);
  const int src_lo = (MODE == FM_STAGE_B_ES) ? 1 : 0;
  const int src_hi1 = (MODE == FM_STAGE_B_ES) ? g.n1 - 1 : g.n1;
  const int src_hi2 = (MODE == FM_STAGE_B_ES) ? g.n2 - 1 : g.n2;
  float lmax = 0.f;

#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    if (!row_ok || c >= n2e) continue;
    const size_t k = i1 + (size_t)ld * c;
    const int i2p = c - npml;
    const bool interior = row_int && i2p >= 0 && i2p < g.n2;
    if (MODE == FM_STAGE_A && it >= 2 && interior) {
      // deferred velocity history of step it-1 (the current vx, vz)
      const size_t o = (size_t)(it - 2) * 3 * nih + i1p + (size_t)L.n1h * i2p;
      H::put(sd.hist, o + nih, qx[j + 2], inv_vx);
      H::put(sd.hist, o + 2 * nih, z0[j], inv_vz);
    }
    if (flush) continue;
    float px_ = pxv[j], pz_ = pzv[j];
    if (row_upd && c >= 2 && c < hi2) {
      const float der2 = dminus(qx[j], qx[j + 1], qx[j + 2], qx[j + 3]);
      const float der1 = dminus(zm2[j], zm1[j], z0[j], zp1[j]);
      const float kd = fmul(dtdx, kv[j]);
      const float kw2 = fmul(kd, __ldg(m.d2a1 + c));
      const float kw1 = fmul(kd, d1a1);
      const float ax = fmul(__ldg(m.d2a + c), px_), bx = fmul(kw2, der2);
      const float az = fmul(d1a, pz_), bz = fmul(kw1, der1);
      const bool fwd = (MODE != FM_STAGE_A);
      px_ = fwd ? fadd(ax, bx) : fsub(ax, bx);
      pz_ = fwd ? fadd(az, bz) : fsub(az, bz);
    }
    if (do_inj)
      px_ = inject_point(sd.inj, px_, i1, c, dt, kv[j], sd.amp + (it - 1), sd.amp_stride,
                         MODE == FM_FWD ? +1 : -1);
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      if (interior && i1p >= src_lo && i1p < src_hi1 && i2p >= src_lo && i2p < src_hi2) {
        const size_t o = (size_t)(ic - 1) * 3 * nih + i1p + (size_t)L.n1h * i2p;
        px_ = fadd(px_, fmul(fmul(mdt, H::get(sd.hist, o, sc_p)), kv[j]));
      }
    }
    const float pv = i1 < fsrows ? 0.f : fadd(px_, pz_);
    sd.px[k] = px_;
    sd.pz[k] = pz_;
    sd.p[k] = pv;
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
  if (MODE == FM_STAGE_A && !flush)
    cta_amax(red, __float_as_uint(lmax),
             sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + (blockIdx.x % kAmaxSlots));
}

// ---------------------------------------------------------------------------
// Velocity kernel (+ receiver/datum gathers in the first `ngb` CTAs)
// ---------------------------------------------------------------------------
template <int MODE, bool FP16, int NP>
__global__ void __launch_bounds__(kThreads)
    k_fused_v(Grid g, ModelDev m, FusedLaunch L, int it, int ngb_per_shot) {
  using H = Hist<FP16>;
  __shared__ unsigned red[2][kWarps];
  __shared__ __align__(16) float prod[kWarps][444];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int ngb = ngb_per_shot * L.nshots;
  if ((int)blockIdx.x < ngb) {
    if (MODE == FM_STAGE_A) return;
    const int shot = blockIdx.x / ngb_per_shot;
    const ShotDevice& sd = L.shots[shot];
    if (!sd.active || it > sd.nt || sd.type_rec != 0) return;
    const int s = (blockIdx.x % ngb_per_shot) * kWarps + wib;
    if (s < sd.rec.n) {
      if (sd.out) {
        const float v = warp_gather_ordered(prod[wib], sd.rec.ix1, sd.rec.ix2, sd.rec.tile, s,
                                            sd.p, g.ld, 0, g.n1e, g.n2e);
        const int row = sd.out_reverse ? sd.nt - it : it - 1;
        if (lane == 0) sd.out[row + (size_t)sd.nt * s] = v;
      }
    } else if (s - sd.rec.n < sd.datum.n && sd.red &&
               (MODE == FM_FWD || MODE == FM_STAGE_B_ES)) {
      const int d = s - sd.rec.n;
      const float v = warp_gather_ordered(prod[wib], sd.datum.ix1, sd.datum.ix2, sd.datum.tile,
                                          d, sd.p + g.npml + (size_t)g.ld * g.npml, g.ld,
                                          g.npml, g.n1, g.n2);
      if (lane == 0) sd.red[(it - 1) + (size_t)sd.nt * d] = v;
    }
    return;
  }
  const Tile t = tile_of<NP>(g, blockIdx.x - ngb);
  if (t.shot >= L.nshots) return;
  const ShotDevice& sd = L.shots[t.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (it > nt) return;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const size_t nih = (size_t)L.n1h * g.n2;
  const int i1 = t.i1;
  const bool row_ok = i1 < n1e;
  const int i1p = i1 - npml;
  const bool row_int = row_ok && i1p >= 0 && i1p < g.n1;
  const bool row_upd = row_ok && i1 >= 2 && i1 < hi1;
  const int ic = nt - it + 1;
  float inv_p = 1.f, sc_vx = 1.f, sc_vz = 1.f;
  if (FP16) {
    if (MODE == FM_STAGE_A) {
      const unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots;
      inv_p = pow2f(15 - amax_exponent(warp_amax_slots(a)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + (size_t)(ic - 1) * 3 * kAmaxSlots;
      sc_vx = pow2f(amax_exponent(warp_amax_slots(a + kAmaxSlots)) - 15);
      sc_vz = pow2f(amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)) - 15);
    }
  }
  const float* __restrict__ pp = sd.p;
  // ---- loads
  float qp[NP + 3];  // p at columns c0-1 .. c0+NP+1
#pragma unroll
  for (int j = 0; j < NP + 3; ++j) {
    const int c = t.c0 - 1 + j;
    qp[j] = (row_ok && c >= 0 && c < n2e) ? pp[i1 + (size_t)ld * c] : 0.f;
  }
  float pm1[NP], pp1[NP], pp2[NP], vxv[NP], vzv[NP];
  float hx[NP], hz[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    const bool ok = row_ok && c < n2e;
    const size_t k = i1 + (size_t)ld * c;
    const bool upd = ok && row_upd && c >= 2 && c < hi2;
    pm1[j] = upd ? pp[k - 1] : 0.f;
    pp1[j] = upd ? pp[k + 1] : 0.f;
    pp2[j] = upd ? pp[k + 2] : 0.f;
    vxv[j] = ok ? sd.vx[k] : 0.f;
    vzv[j] = ok ? sd.vz[k] : 0.f;
    hx[j] = 0.f;
    hz[j] = 0.f;
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const int i2p = c - npml;
      if (ok && row_int && i2p >= 0 && i2p < g.n2) {
        const size_t o = (size_t)(ic - 1) * 3 * nih + i1p + (size_t)L.n1h * i2p;
        hx[j] = H::get(sd.hist, o + nih, sc_vx);
        hz[j] = H::get(sd.hist, o + 2 * nih, sc_vz);
      }
    }
  }
  const float dt = g.dt, mdt = fmul(-1.0f, dt);
  const float d1b = row_ok ? __ldg(m.d1b + i1) : 0.f;
  const float bw1 = row_ok ? __ldg(m.bw1 + i1) : 0.f;
  const bool fs_src_row = g.ofs == 1 && i1 == npml;      // also writes vz(npml)
  const bool fs_dst_row = g.ofs == 1 && i1 == npml - 1;  // vz overwritten
  const bool do_inj = (MODE == FM_FWD) && sd.type_src == 1;
  float lmx = 0.f, lmz = 0.f;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    if (!row_ok || c >= n2e) continue;
    const size_t k = i1 + (size_t)ld * c;
    const int i2p = c - npml;
    const bool interior = row_int && i2p >= 0 && i2p < g.n2;
    float vx_ = vxv[j], vz_ = vzv[j];
    if (row_upd && c >= 2 && c < hi2) {
      const float der2 = dplus(qp[j], qp[j + 1], qp[j + 2], qp[j + 3]);
      const float der1 = dplus(pm1[j], qp[j + 1], pp1[j], pp2[j]);
      const float ax = fmul(__ldg(m.d2b + c), vx_), bx = fmul(__ldg(m.bw2 + c), der2);
      const float az = fmul(d1b, vz_), bz = fmul(bw1, der1);
      const bool fwd = (MODE != FM_STAGE_A);
      vx_ = fwd ? fadd(ax, bx) : fsub(ax, bx);
      vz_ = fwd ? fadd(az, bz) : fsub(az, bz);
    }
    if ((MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) && interior) {
      vx_ = fadd(vx_, fmul(fmul(mdt, hx[j]), 1.0f));
      vz_ = fadd(vz_, fmul(fmul(mdt, hz[j]), 1.0f));
    }
    if (do_inj)
      vz_ = inject_point(sd.inj, vz_, i1, c, dt, 1.0f, sd.amp + (it - 1), sd.amp_stride, +1);
    sd.vx[k] = vx_;
    if (!fs_dst_row) sd.vz[k] = vz_;
    if (fs_src_row) sd.vz[k - 1] = vz_;
    if (MODE == FM_STAGE_A && interior) {
      const size_t o = (size_t)(it - 1) * 3 * nih + i1p + (size_t)L.n1h * i2p;
      H::put(sd.hist, o, qp[j + 1], inv_p);  // deferred pressure history of step it
      lmx = fmaxf(lmx, fabsf(vx_));
      lmz = fmaxf(lmz, fabsf(vz_));
    }
  }
  if (MODE == FM_STAGE_A) {
    unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + (blockIdx.x % kAmaxSlots);
    cta_amax(red[0], __float_as_uint(lmx), a + kAmaxSlots);
    cta_amax(red[1], __float_as_uint(lmz), a + 2 * kAmaxSlots);
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

int host_bps(const Grid& g, int np) {
  return ((g.n1e + 31) / 32) * ((g.n2e + kWarps * np - 1) / (kWarps * np));
}

template <int MODE, int NP>
void launch_p_np(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it,
                 cudaStream_t st) {
  const int blocks = host_bps(g, NP) * L.nshots;
  if (L.hist_fp16)
    k_fused_p<MODE, true, NP><<<blocks, kThreads, 0, st>>>(g, m, L, it);
  else
    k_fused_p<MODE, false, NP><<<blocks, kThreads, 0, st>>>(g, m, L, it);
}

template <int MODE, int NP>
void launch_v_np(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it,
                 cudaStream_t st) {
  const int stations = (MODE == FM_STAGE_A) ? 0 : L.max_rec + L.max_datum;
  const int ngbps = (stations + kWarps - 1) / kWarps;
  const int blocks = (host_bps(g, NP) + ngbps) * L.nshots;
  if (L.hist_fp16)
    k_fused_v<MODE, true, NP><<<blocks, kThreads, 0, st>>>(g, m, L, it, ngbps);
  else
    k_fused_v<MODE, false, NP><<<blocks, kThreads, 0, st>>>(g, m, L, it, ngbps);
}

template <int MODE>
void launch_p(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, cudaStream_t st) {
  switch (L.chunk) {
    case 1: launch_p_np<MODE, 1>(g, m, L, it, st); break;
    case 4: launch_p_np<MODE, 4>(g, m, L, it, st); break;
    default: launch_p_np<MODE, 2>(g, m, L, it, st); break;
  }
}

template <int MODE>
void launch_v(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, cudaStream_t st) {
  switch (L.chunk) {
    case 1: launch_v_np<MODE, 1>(g, m, L, it, st); break;
    case 4: launch_v_np<MODE, 4>(g, m, L, it, st); break;
    default: launch_v_np<MODE, 2>(g, m, L, it, st); break;
  }
}

}  // namespace

int fused_warps(const Grid& g, int chunk) { return host_bps(g, chunk) * kWarps; }

void fused_p_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st) {
  switch (mode) {
    case FM_FWD: launch_p<FM_FWD>(g, m, L, it, st); break;
    case FM_STAGE_A: launch_p<FM_STAGE_A>(g, m, L, it, st); break;
    case FM_STAGE_B: launch_p<FM_STAGE_B>(g, m, L, it, st); break;
    default: launch_p<FM_STAGE_B_ES>(g, m, L, it, st); break;
  }
}

void fused_v_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st) {
  switch (mode) {
    case FM_FWD: launch_v<FM_FWD>(g, m, L, it, st); break;
    case FM_STAGE_A: launch_v<FM_STAGE_A>(g, m, L, it, st); break;
    case FM_STAGE_B: launch_v<FM_STAGE_B>(g, m, L, it, st); break;
    default: launch_v<FM_STAGE_B_ES>(g, m, L, it, st); break;
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
