// Fused time-step kernels for a batch of shots sharing one model.
//
// Mapping: a CTA of 8 warps covers 64 consecutive depth rows (i1, the
// contiguous axis) and 8*NP columns.  Each lane owns two adjacent rows
// (float2: every warp access is one 256-byte segment) and NP consecutive
// columns.  All loads of a thread -- its own values and the i2 neighbours of
// the staggered stencil (columns c-2..c+NP) -- are independent and issued
// before any arithmetic; the i1 neighbours come from warp shuffles, with the
// two warp-edge lanes reading their halo rows directly.  The 2-D state of a
// 751x2301 shot (~48 MB) stays in L2, so the kernels are bound by L2 and
// instruction issue; the layout keeps both low (one load instruction per two
// points per field, 32-bit indexing, per-shot descriptor held in registers).
//
// Arithmetic of every update is the reference's, operation by operation
// (separately rounded FP32), so with FP32 histories the fused path reproduces
// the plain port and the FP32 oracle bit for bit.  FP16 histories carry one
// power-of-two scale per (shot, step, field): the kernel that produces a
// field reduces max|x| over the interior; the next kernel, which reads the
// field anyway for its stencil, encodes and stores it -- no extra pass.
//
// History layout: [step][field][i2p][n1h] with extended row i1 stored at row
// i1 - Grid::hist_base(), so the two rows of a lane (even i1) land on an
// aligned pair.
#include "fused.cuh"

namespace daw {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr unsigned kAll = 0xffffffffu;

// Power-of-two scale exponent E of a step/field with max|x| < 2^E; values are
// stored as x * 2^(15-E), so |stored| < 2^15 < 65504.
__device__ __forceinline__ int amax_exponent(unsigned bits) {
  const int ef = (int)(bits >> 23);
  const int e = (ef == 0) ? -126 : ef - 126;
  return max(min(e, 120), -100);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }
__device__ __forceinline__ unsigned warp_amax_slots(const unsigned* slots) {
  return __reduce_max_sync(kAll, slots[threadIdx.x & 31]);
}

__device__ __forceinline__ float2 ld2(const float* p, int k) {
  return *reinterpret_cast<const float2*>(p + k);
}
__device__ __forceinline__ void st2(float* p, int k, float2 v) {
  *reinterpret_cast<float2*>(p + k) = v;
}

// History store/load of the two rows of a lane (rows valid flags v0, v1).
template <bool FP16>
struct Hist;
template <>
struct Hist<true> {
  static __device__ __forceinline__ void put2(void* base, int o, float a, float b, float inv,
                                              bool v0, bool v1) {
    __half* h = static_cast<__half*>(base);
    if (v0 && v1)
      *reinterpret_cast<__half2*>(h + o) = __floats2half2_rn(a * inv, b * inv);
    else if (v0)
      h[o] = __float2half_rn(a * inv);
    else if (v1)
      h[o + 1] = __float2half_rn(b * inv);
  }
  static __device__ __forceinline__ float2 get2(const void* base, int o, float sc, bool v0,
                                                bool v1) {
    const __half* h = static_cast<const __half*>(base);
    if (v0 && v1) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(h + o));
      return make_float2(f.x * sc, f.y * sc);
    }
    return make_float2(v0 ? __half2float(h[o]) * sc : 0.f, v1 ? __half2float(h[o + 1]) * sc : 0.f);
  }
};
template <>
struct Hist<false> {
  static __device__ __forceinline__ void put2(void* base, int o, float a, float b, float,
                                              bool v0, bool v1) {
    float* h = static_cast<float*>(base);
    if (v0 && v1)
      *reinterpret_cast<float2*>(h + o) = make_float2(a, b);
    else if (v0)
      h[o] = a;
    else if (v1)
      h[o + 1] = b;
  }
  static __device__ __forceinline__ float2 get2(const void* base, int o, float, bool v0,
                                                bool v1) {
    const float* h = static_cast<const float*>(base);
    if (v0 && v1) return *reinterpret_cast<const float2*>(h + o);
    return make_float2(v0 ? h[o] : 0.f, v1 ? h[o + 1] : 0.f);
  }
};

template <bool FP16>
__device__ __forceinline__ void* step_base(void* hist, int step0, size_t nih) {
  return static_cast<char*>(hist) + (size_t)step0 * 3 * nih * (FP16 ? 2 : 4);
}

struct Tile {
  int shot, i1, c0;
};

template <int NP>
__device__ __forceinline__ Tile tile_of(const Grid& g, int block) {
  const int nrb = g.ld >> 6;
  const int bps = nrb * ((g.n2e + kWarps * NP - 1) / (kWarps * NP));
  Tile t;
  t.shot = block / bps;
  const int lb = block - t.shot * bps;
  t.i1 = (lb % nrb) * 64 + 2 * (threadIdx.x & 31);
  t.c0 = ((lb / nrb) * kWarps + (threadIdx.x >> 5)) * NP;
  return t;
}

// Injection contributions at (i1, c) in station order, given the column band.
__device__ __forceinline__ float inject_at(const InjMapDev& m, float v, int i1, int clo, int base,
                                           float dt, float w, const float* amp, int amp_stride,
                                           int sign) {
  const int r = base + (i1 - clo);
  const int e0 = __ldg(m.rowptr + 2 * r), e1 = __ldg(m.rowptr + 2 * r + 1);
  for (int e = e0; e < e1; ++e) {
    const float a = __ldg(amp + (size_t)__ldg(m.sta + e) * amp_stride);
    const float term = fmul(fmul(fmul(__ldg(m.coef + e), dt), a), w);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  return v;
}

// max |x| as bit patterns of |x| (NaN/Inf rank above every finite value and
// raise kErrNonFinite)
__device__ __forceinline__ unsigned abs_bits(float x) { return __float_as_uint(x) & 0x7fffffffu; }
__device__ __forceinline__ void cta_amax(unsigned* red, unsigned v, unsigned* slot,
                                         unsigned* err) {
  const unsigned b = __reduce_max_sync(kAll, v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned r = 0;
    for (int w = 0; w < kWarps; ++w) r = max(r, red[w]);
    if (r) atomicMax(slot, r);
    if (r >= 0x7f800000u) atomicOr(err, kErrNonFinite);
  }
}

// ---------------------------------------------------------------------------
// Pressure kernel
// ---------------------------------------------------------------------------
template <int MODE, bool FP16, int NP>
__global__ void __launch_bounds__(kThreads)
    k_fused_p(const Grid g, const ModelDev m, const FusedLaunch L, const int it) {
  using H = Hist<FP16>;
  __shared__ unsigned red[kWarps];
  const int lane = threadIdx.x & 31;
  const Tile t = tile_of<NP>(g, blockIdx.x);
  if (t.shot >= L.nshots) return;  // CTA-uniform
  const ShotDevice sd = L.shots[t.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (MODE == FM_STAGE_A ? it > nt + 1 : it > nt) return;
  const bool flush = (MODE == FM_STAGE_A) && it == nt + 1;  // v history of step nt only
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int fsrows = g.ofs == 1 ? npml + 1 : 0;
  const int n1h = L.n1h;
  const size_t nih = (size_t)n1h * g.n2;
  const int i1 = t.i1;  // rows i1, i1+1
  const bool ok0 = i1 < n1e, ok1 = i1 + 1 < n1e;
  // update range [2, hi1) of each row (row 1 of the first lane is outside it)
  const bool u0 = ok0 && i1 >= 2 && i1 < hi1, u1 = ok1 && i1 + 1 >= 2 && i1 + 1 < hi1;
  const bool r0 = ok0 && i1 >= npml && i1 < npml + g.n1;
  const bool r1 = ok1 && i1 + 1 >= npml && i1 + 1 < npml + g.n1;
  const int h1 = i1 - g.hist_base();  // history row of i1 (even)
  const int ic = nt - it + 1;
  const int hs = ic - 1 - L.hist_step0;  // stage B: history slot of step ic

  float inv_vx = 1.f, inv_vz = 1.f, sc_p = 1.f;
  if (FP16) {
    if (MODE == FM_STAGE_A && it >= 2) {
      const unsigned* a = sd.amax + (size_t)(it - 2) * 3 * kAmaxSlots;
      inv_vx = pow2f(15 - amax_exponent(warp_amax_slots(a + kAmaxSlots)));
      inv_vz = pow2f(15 - amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + (size_t)hs * 3 * kAmaxSlots;
      sc_p = pow2f(amax_exponent(warp_amax_slots(a)) - 15);
    }
  }
  const float* __restrict__ vx = sd.vx;
  const float* __restrict__ vz = sd.vz;
  float* __restrict__ pxa = sd.px;
  float* __restrict__ pza = sd.pz;
  float* __restrict__ pa = sd.p;

  // ---- loads (independent)
  float2 qx[NP + 3];  // vx at columns c0-2 .. c0+NP
#pragma unroll
  for (int j = 0; j < NP + 3; ++j) {
    const int c = t.c0 - 2 + j;
    qx[j] = (c >= 0 && c < n2e) ? ld2(vx, i1 + ld * c) : make_float2(0.f, 0.f);
  }
  float2 z[NP], px2[NP], pz2[NP], k2[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    const int k = i1 + ld * c;
    const bool cok = c < n2e;
    z[j] = cok ? ld2(vz, k) : make_float2(0.f, 0.f);
    px2[j] = (cok && !flush) ? ld2(pxa, k) : make_float2(0.f, 0.f);
    pz2[j] = (cok && !flush) ? ld2(pza, k) : make_float2(0.f, 0.f);
    k2[j] = (cok && !flush) ? __ldg(reinterpret_cast<const float2*>(m.kap + k)) : make_float2(0.f, 0.f);
  }
  const float dtdx = g.dtdx, dt = g.dt, mdt = fmul(-1.0f, dt);
  const float2 d1a = ok1 ? __ldg(reinterpret_cast<const float2*>(m.d1a + i1))
                         : make_float2(ok0 ? __ldg(m.d1a + i1) : 0.f, 0.f);
  const float2 d1a1 = ok1 ? __ldg(reinterpret_cast<const float2*>(m.d1a1 + i1))
                          : make_float2(ok0 ? __ldg(m.d1a1 + i1) : 0.f, 0.f);
  const bool do_inj = (MODE == FM_STAGE_A) || (MODE == FM_FWD && sd.type_src == 0);
  const int slo = (MODE == FM_STAGE_B_ES) ? 1 : 0;
  const int shi1 = (MODE == FM_STAGE_B_ES) ? g.n1 - 1 : g.n1;
  const int shi2 = (MODE == FM_STAGE_B_ES) ? g.n2 - 1 : g.n2;
  const bool s0 = r0 && i1 - npml >= slo && i1 - npml < shi1;
  const bool s1 = r1 && i1 + 1 - npml >= slo && i1 + 1 - npml < shi1;
  void* hv_store = (MODE == FM_STAGE_A && it >= 2) ? step_base<FP16>(sd.hist, it - 2, nih) : nullptr;
  const void* hp_read = (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES)
                            ? step_base<FP16>(sd.hist, hs, nih) : nullptr;
  unsigned lmax = 0;

#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    if (c >= n2e) continue;  // warp-uniform
    // vz at rows i1-2, i1-1 (lane-1) and i1+2 (lane+1)
    float zm2 = __shfl_up_sync(kAll, z[j].x, 1);
    float zm1 = __shfl_up_sync(kAll, z[j].y, 1);
    float zp2 = __shfl_down_sync(kAll, z[j].x, 1);
    const int k = i1 + ld * c;
    if (lane == 0 && i1 >= 2) {
      const float2 e = ld2(vz, k - 2);
      zm2 = e.x;
      zm1 = e.y;
    }
    if (lane == 31 && i1 + 2 < ld) zp2 = vz[k + 2];
    const int i2p = c - npml;
    const bool cint = i2p >= 0 && i2p < g.n2;
    const int ho = h1 + n1h * i2p;
    if (MODE == FM_STAGE_A && it >= 2 && cint)  // deferred v history of step it-1
      if (r0 || r1) {
        H::put2(hv_store, (int)nih + ho, qx[j + 2].x, qx[j + 2].y, inv_vx, r0, r1);
        H::put2(hv_store, 2 * (int)nih + ho, z[j].x, z[j].y, inv_vz, r0, r1);
      }
    if (flush || !ok0) continue;
    float2 px_ = px2[j], pz_ = pz2[j];
    const bool cupd = c >= 2 && c < hi2;
    if (cupd) {
      const float kw2f = __ldg(m.d2a1 + c), d2a = __ldg(m.d2a + c);
      const bool fwd = (MODE != FM_STAGE_A);
      if (u0) {
        const float der2 = dminus(qx[j].x, qx[j + 1].x, qx[j + 2].x, qx[j + 3].x);
        const float der1 = dminus(zm2, zm1, z[j].x, z[j].y);
        const float kd = fmul(dtdx, k2[j].x);
        const float ax = fmul(d2a, px_.x), bx = fmul(fmul(kd, kw2f), der2);
        const float az = fmul(d1a.x, pz_.x), bz = fmul(fmul(kd, d1a1.x), der1);
        px_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
        pz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
      }
      if (u1) {
        const float der2 = dminus(qx[j].y, qx[j + 1].y, qx[j + 2].y, qx[j + 3].y);
        const float der1 = dminus(zm1, z[j].x, z[j].y, zp2);
        const float kd = fmul(dtdx, k2[j].y);
        const float ax = fmul(d2a, px_.y), bx = fmul(fmul(kd, kw2f), der2);
        const float az = fmul(d1a.y, pz_.y), bz = fmul(fmul(kd, d1a1.y), der1);
        px_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
        pz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
      }
    }
    if (do_inj) {
      const int clo = __ldg(sd.inj.col_lo + c);
      const int chi = __ldg(sd.inj.col_hi + c);
      if (i1 + 1 >= clo && i1 <= chi) {
        const int base = __ldg(sd.inj.col_base + c);
        const int sg = MODE == FM_FWD ? +1 : -1;
        if (i1 >= clo && i1 <= chi)
          px_.x = inject_at(sd.inj, px_.x, i1, clo, base, dt, k2[j].x, sd.amp + (it - 1),
                            sd.amp_stride, sg);
        if (ok1 && i1 + 1 >= clo && i1 + 1 <= chi)
          px_.y = inject_at(sd.inj, px_.y, i1 + 1, clo, base, dt, k2[j].y, sd.amp + (it - 1),
                            sd.amp_stride, sg);
      }
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const bool c_src = i2p >= slo && i2p < shi2;
      if (c_src && (s0 || s1)) {
        const float2 hv = H::get2(hp_read, ho, sc_p, s0, s1);
        if (s0) px_.x = fadd(px_.x, fmul(fmul(mdt, hv.x), k2[j].x));
        if (s1) px_.y = fadd(px_.y, fmul(fmul(mdt, hv.y), k2[j].y));
      }
    }
    float2 pv;
    pv.x = i1 < fsrows ? 0.f : fadd(px_.x, pz_.x);
    pv.y = i1 + 1 < fsrows ? 0.f : fadd(px_.y, pz_.y);
    st2(pxa, k, px_);
    st2(pza, k, pz_);
    st2(pa, k, pv);
    if (cint) {
      if (MODE == FM_STAGE_A) {
        if (r0) lmax = max(lmax, abs_bits(pv.x));
        if (r1) lmax = max(lmax, abs_bits(pv.y));
      }
      if ((MODE == FM_FWD || MODE == FM_STAGE_B_ES) && sd.wf && sd.type_rec == 0) {
        float* w = sd.wf + (size_t)(it - 1) * g.int_elems() + (size_t)g.n1 * i2p;
        const int i1p = i1 - npml;
        if (MODE == FM_FWD) {
          if (r0) w[i1p] = pv.x;
          if (r1) w[i1p + 1] = pv.y;
        } else {
          if (r0) w[i1p] = fadd(w[i1p], pv.x);
          if (r1) w[i1p + 1] = fadd(w[i1p + 1], pv.y);
        }
      }
    }
  }
  if (MODE == FM_STAGE_A && !flush)
    cta_amax(red, lmax, sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + (blockIdx.x % kAmaxSlots),
             L.err);
}

// ---------------------------------------------------------------------------
// Velocity kernel (+ receiver/datum gathers in the first `ngb` CTAs)
// ---------------------------------------------------------------------------
template <int MODE, bool FP16, int NP>
__global__ void __launch_bounds__(kThreads)
    k_fused_v(const Grid g, const ModelDev m, const FusedLaunch L, const int it,
              const int ngb_per_shot) {
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
  const ShotDevice sd = L.shots[t.shot];
  if (!sd.active) return;
  const int nt = sd.nt;
  if (it > nt) return;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int n1h = L.n1h;
  const size_t nih = (size_t)n1h * g.n2;
  const int i1 = t.i1;
  const bool ok0 = i1 < n1e, ok1 = i1 + 1 < n1e;
  const bool u0 = ok0 && i1 >= 2 && i1 < hi1, u1 = ok1 && i1 + 1 >= 2 && i1 + 1 < hi1;
  const bool r0 = ok0 && i1 >= npml && i1 < npml + g.n1;
  const bool r1 = ok1 && i1 + 1 >= npml && i1 + 1 < npml + g.n1;
  const int h1 = i1 - g.hist_base();
  const int ic = nt - it + 1;
  const int hs = ic - 1 - L.hist_step0;  // stage B: history slot of step ic
  float inv_p = 1.f, sc_vx = 1.f, sc_vz = 1.f;
  if (FP16) {
    if (MODE == FM_STAGE_A) {
      const unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots;
      inv_p = pow2f(15 - amax_exponent(warp_amax_slots(a)));
    }
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const unsigned* a = sd.amax + (size_t)hs * 3 * kAmaxSlots;
      sc_vx = pow2f(amax_exponent(warp_amax_slots(a + kAmaxSlots)) - 15);
      sc_vz = pow2f(amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)) - 15);
    }
  }
  const float* __restrict__ pp = sd.p;
  float* __restrict__ vxa = sd.vx;
  float* __restrict__ vza = sd.vz;
  void* hp_store = (MODE == FM_STAGE_A) ? step_base<FP16>(sd.hist, it - 1, nih) : nullptr;
  const void* hv_read = (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES)
                            ? step_base<FP16>(sd.hist, hs, nih) : nullptr;
  // ---- loads
  float2 qp[NP + 3];  // p at columns c0-1 .. c0+NP+1
#pragma unroll
  for (int j = 0; j < NP + 3; ++j) {
    const int c = t.c0 - 1 + j;
    qp[j] = (c >= 0 && c < n2e) ? ld2(pp, i1 + ld * c) : make_float2(0.f, 0.f);
  }
  float2 vx2[NP], vz2[NP], hx[NP], hz[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    const int k = i1 + ld * c;
    const bool cok = c < n2e;
    vx2[j] = cok ? ld2(vxa, k) : make_float2(0.f, 0.f);
    vz2[j] = cok ? ld2(vza, k) : make_float2(0.f, 0.f);
    hx[j] = make_float2(0.f, 0.f);
    hz[j] = make_float2(0.f, 0.f);
    if (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) {
      const int i2p = c - npml;
      if (cok && i2p >= 0 && i2p < g.n2 && (r0 || r1)) {
        const int ho = h1 + n1h * i2p;
        hx[j] = H::get2(hv_read, (int)nih + ho, sc_vx, r0, r1);
        hz[j] = H::get2(hv_read, 2 * (int)nih + ho, sc_vz, r0, r1);
      }
    }
  }
  const float dt = g.dt, mdt = fmul(-1.0f, dt);
  const float2 d1b = ok1 ? __ldg(reinterpret_cast<const float2*>(m.d1b + i1))
                         : make_float2(ok0 ? __ldg(m.d1b + i1) : 0.f, 0.f);
  const float2 bw1 = ok1 ? __ldg(reinterpret_cast<const float2*>(m.bw1 + i1))
                         : make_float2(ok0 ? __ldg(m.bw1 + i1) : 0.f, 0.f);
  // free surface vz(npml) = vz(npml+1) (1-based): 0-based row npml-1 takes
  // the value of row npml
  const bool fs = g.ofs == 1;
  const bool dst_x = fs && i1 == npml - 1;      // own pair (npml-1, npml)
  const bool skip_y = fs && i1 + 1 == npml - 1; // row npml-1 written by the next lane
  const bool src_x = fs && i1 == npml;          // also write row npml-1 (previous lane's)
  const bool do_inj = (MODE == FM_FWD) && sd.type_src == 1;
  unsigned lmx = 0, lmz = 0;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int c = t.c0 + j;
    if (c >= n2e) continue;  // warp-uniform
    // p at rows i1-1 (lane-1 .y), i1+2, i1+3 (lane+1)
    float pm1 = __shfl_up_sync(kAll, qp[j + 1].y, 1);
    float pp2 = __shfl_down_sync(kAll, qp[j + 1].x, 1);
    float pp3 = __shfl_down_sync(kAll, qp[j + 1].y, 1);
    const int k = i1 + ld * c;
    if (lane == 0 && i1 >= 1) pm1 = pp[k - 1];
    if (lane == 31 && i1 + 3 < ld) {
      const float2 e = ld2(pp, k + 2);
      pp2 = e.x;
      pp3 = e.y;
    }
    if (!ok0) continue;
    const int i2p = c - npml;
    const bool cint = i2p >= 0 && i2p < g.n2;
    float2 vx_ = vx2[j], vz_ = vz2[j];
    if (c >= 2 && c < hi2) {
      const float d2b = __ldg(m.d2b + c), bw2 = __ldg(m.bw2 + c);
      const bool fwd = (MODE != FM_STAGE_A);
      if (u0) {
        const float der2 = dplus(qp[j].x, qp[j + 1].x, qp[j + 2].x, qp[j + 3].x);
        const float der1 = dplus(pm1, qp[j + 1].x, qp[j + 1].y, pp2);
        const float ax = fmul(d2b, vx_.x), bx = fmul(bw2, der2);
        const float az = fmul(d1b.x, vz_.x), bz = fmul(bw1.x, der1);
        vx_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
        vz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
      }
      if (u1) {
        const float der2 = dplus(qp[j].y, qp[j + 1].y, qp[j + 2].y, qp[j + 3].y);
        const float der1 = dplus(qp[j + 1].x, qp[j + 1].y, pp2, pp3);
        const float ax = fmul(d2b, vx_.y), bx = fmul(bw2, der2);
        const float az = fmul(d1b.y, vz_.y), bz = fmul(bw1.y, der1);
        vx_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
        vz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
      }
    }
    if ((MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) && cint) {
      if (r0) {
        vx_.x = fadd(vx_.x, fmul(fmul(mdt, hx[j].x), 1.0f));
        vz_.x = fadd(vz_.x, fmul(fmul(mdt, hz[j].x), 1.0f));
      }
      if (r1) {
        vx_.y = fadd(vx_.y, fmul(fmul(mdt, hx[j].y), 1.0f));
        vz_.y = fadd(vz_.y, fmul(fmul(mdt, hz[j].y), 1.0f));
      }
    }
    if (do_inj) {
      const int clo = __ldg(sd.inj.col_lo + c);
      const int chi = __ldg(sd.inj.col_hi + c);
      if (i1 + 1 >= clo && i1 <= chi) {
        const int base = __ldg(sd.inj.col_base + c);
        if (i1 >= clo && i1 <= chi)
          vz_.x = inject_at(sd.inj, vz_.x, i1, clo, base, dt, 1.0f, sd.amp + (it - 1),
                            sd.amp_stride, +1);
        if (ok1 && i1 + 1 >= clo && i1 + 1 <= chi)
          vz_.y = inject_at(sd.inj, vz_.y, i1 + 1, clo, base, dt, 1.0f, sd.amp + (it - 1),
                            sd.amp_stride, +1);
      }
    }
    if (dst_x) vz_.x = vz_.y;
    st2(vxa, k, vx_);
    if (skip_y)
      vza[k] = vz_.x;
    else
      st2(vza, k, vz_);
    if (src_x) vza[k - 1] = vz_.x;
    if (MODE == FM_STAGE_A && cint && (r0 || r1)) {
      // deferred pressure history of step it (the current p)
      H::put2(hp_store, h1 + n1h * i2p, qp[j + 1].x, qp[j + 1].y, inv_p, r0, r1);
      if (r0) {
        lmx = max(lmx, abs_bits(vx_.x));
        lmz = max(lmz, abs_bits(vz_.x));
      }
      if (r1) {
        lmx = max(lmx, abs_bits(vx_.y));
        lmz = max(lmz, abs_bits(vz_.y));
      }
    }
  }
  if (MODE == FM_STAGE_A) {
    unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + (blockIdx.x % kAmaxSlots);
    cta_amax(red[0], lmx, a + kAmaxSlots, L.err);
    cta_amax(red[1], lmz, a + 2 * kAmaxSlots, L.err);
  }
}

// Sum of 0.5*sp^2 over a stage-A history (the esource `cost`).
template <bool FP16>
__global__ void k_hist_cost(const void* hist, const unsigned* amax, int nt, int n1, int n2,
                            int inner_ld, int inner_off, size_t field_stride, double* out) {
  __shared__ double sh[256];
  double acc = 0;
  const size_t per = (size_t)n1 * n2;
  const size_t total = per * nt;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(q / per);
    const size_t r = q % per;
    const int i1 = (int)(r % n1), i2 = (int)(r / n1);
    const size_t o = (size_t)it * 3 * field_stride + inner_off + i1 + (size_t)inner_ld * i2;
    float v;
    if (FP16) {
      unsigned b = 0;
      for (int s = 0; s < kAmaxSlots; ++s) b = max(b, amax[(size_t)it * 3 * kAmaxSlots + s]);
      v = __half2float(static_cast<const __half*>(hist)[o]) * pow2f(amax_exponent(b) - 15);
    } else {
      v = static_cast<const float*>(hist)[o];
    }
    acc += 0.5 * (double)v * (double)v;
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
  return (g.ld / 64) * ((g.n2e + kWarps * np - 1) / (kWarps * np));
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
                  int inner_ld, int inner_off, size_t field_stride, double* out,
                  cudaStream_t st) {
  const int blocks = 148 * 4;
  if (fp16)
    k_hist_cost<true><<<blocks, 256, 0, st>>>(hist, amax, nt, n1, n2, inner_ld, inner_off,
                                              field_stride, out);
  else
    k_hist_cost<false><<<blocks, 256, 0, st>>>(hist, amax, nt, n1, n2, inner_ld, inner_off,
                                               field_stride, out);
}

}  // namespace daw
