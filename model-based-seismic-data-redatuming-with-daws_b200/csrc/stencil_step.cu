// One kernel per time step: the pressure update and the velocity update of
// step `it` in a single pass over the grid (the default fused path).
//
// The reference's time step (src/submodeling2.f90:148-236 forward,
// :1013-1087 stage A, :1104-1192 stage B) is a pressure update from the
// velocities, an injection into px, p = px + pz, then a velocity update from
// p.  A tile of 64 depth rows x TC columns needs p on its own points and on a
// halo (one row/column before, two after), so the kernel recomputes p there
// from the neighbours' inputs instead of exchanging it: the redundant work is
// (3*64 + 3*TC) points per tile.  The pass therefore cannot update in place --
// a neighbour may still read a halo value -- and the state alternates between
// two sets of fields: launch `it` reads set (par0 + it - first) & 1 and writes
// the other.  Against the two-kernel split this removes the write and re-read
// of p, the second read of vx/vz and one launch per step: 36 bytes per
// extended point and step, the algorithmic minimum.
//
// Tiles are copied by the tensor-memory accelerator (cp.async.bulk.tensor,
// 2-D boxes of 72 rows with 16-byte aligned starts, no multicast) into a
// double-buffered stage, armed on an mbarrier whose every wait is bounded.
//
// Work queue: tiles (shot-major, row-major within a shot, so the tile row of
// the surface sources and receivers -- the heaviest tiles -- goes first),
// then the gather units of the previous step.  CTAs take items from a global
// counter: launch it owns counter values from (it - first) * (items + grid)
// on, since every CTA takes exactly one item past the end.  The queue order
// only decides which CTA computes a tile, never a result.
//
// Work of step it - 1 done at launch it, because it needs values that are
// complete only when launch it - 1 has finished:
//   - stage A: the pressure and velocity histories, stored with the FP16
//     scale of that step's max |x| (reduced by launch it - 1), from the tile's
//     input boxes (p = px + pz with the free-surface rows zero);
//   - forward / stage B: the receiver and datum gathers, from the input
//     state set (p = px + pz formed on the fly).
// The run's last launch (it = last + 1) does only that.
//
// Arithmetic: the reference's separately rounded FP32 operations in its order
// (stencil, injection in station order, stage-B sources, p = px + pz, the free
// surface), so the FP32-history path reproduces the FP32 oracle bit for bit.
#include <cuda.h>

#include <type_traits>

#include "fused.cuh"
#include "tma.cuh"

namespace daw {
namespace {

constexpr int kT = 256;          // threads per CTA (8 warps)
constexpr int SR = 64;           // rows per tile (32 lanes x 2)
constexpr int SH = 4;            // row halo of the field boxes (aligned start r0 - 4)
constexpr int SB = SR + 2 * SH;  // 72 rows per field box
constexpr int kHPRows = 80;      // rows of the stage-B pressure-history box (start r0 - 8)
constexpr int kAmpMaxS = 2048;   // stations whose amplitudes are staged in shared memory
constexpr int kBatchS = 6;       // injection entries loaded per point at once
constexpr int kMaxBandCols = 40; // >= TC + 3
constexpr int kBandInts = 4 * kMaxBandCols + 8;  // band info of one stage
constexpr int kGatherStride = 444;

__host__ __device__ constexpr int pad128(int x) { return (x + 127) / 128 * 128; }

template <int TC>
struct SG {
  static constexpr int CPT = TC / 8;  // columns per warp
  static constexpr int NX = TC + 6;   // vx box: columns c0-3 .. c0+TC+2
  static constexpr int NP = TC + 3;   // vz, px, pz, kappa boxes: c0-1 .. c0+TC+1
  static constexpr int kVX = pad128(SB * NX * 4);
  static constexpr int kF = pad128(SB * NP * 4);
  static constexpr int kBase = kVX + 4 * kF;
  static constexpr int kHalo = 3 * SR + 3 * TC;
  __host__ __device__ static constexpr bool stage_b(int mode) {
    return mode == FM_STAGE_B || mode == FM_STAGE_B_ES;
  }
  __host__ __device__ static constexpr int hp_bytes(bool fp16) { return kHPRows * NP * (fp16 ? 2 : 4); }
  __host__ __device__ static constexpr int hv_bytes(bool fp16) { return SR * TC * (fp16 ? 2 : 4); }
  __host__ __device__ static constexpr int stage(int mode, bool fp16) {
    return kBase + (stage_b(mode) ? pad128(hp_bytes(fp16)) + 2 * hv_bytes(fp16) : 0);
  }
  // bytes delivered by the copies of one tile (the mbarrier transaction count)
  __host__ __device__ static constexpr int tx(bool hist, bool fp16) {
    return SB * NX * 4 + 4 * SB * NP * 4 + (hist ? hp_bytes(fp16) + 2 * hv_bytes(fp16) : 0);
  }
  __host__ __device__ static constexpr int amp_bytes(int mode) {
    return (mode == FM_FWD || mode == FM_STAGE_A) ? kAmpMaxS * 4 : 0;
  }
  static constexpr size_t smem(int mode, bool fp16) {
    return 2 * (size_t)stage(mode, fp16) + amp_bytes(mode) + 2 * kBandInts * 4 + 64;
  }
  static_assert(2 * kBase >= 8 * kGatherStride * 4, "gather products fit in the stage buffers");
};

struct SItem {
  int kind;  // 0 tile, 1 gather unit, 2 past the end
  int shot, r0, c0, unit;
};

template <int TC>
__device__ __forceinline__ SItem item_of(const Grid& g, int idx, int nshots, int ntile,
                                         int ngath) {
  SItem r{2, 0, 0, 0, 0};
  const int ntall = ntile * nshots;
  if (idx < ntall) {
    r.kind = 0;
    r.shot = idx / ntile;
    const int l = idx - r.shot * ntile;
    const int ncb = (g.n2e + TC - 1) / TC;
    r.r0 = (l / ncb) * SR;
    r.c0 = (l % ncb) * TC;
  } else if (idx < ntall + ngath * nshots) {
    const int u = idx - ntall;
    r.kind = 1;
    r.shot = u / ngath;
    r.unit = u - r.shot * ngath;
  }
  return r;
}

__device__ __forceinline__ int shot_nt(const FusedLaunch& L, int s) {
  return s < L.nparam ? L.shot_nt[s] : L.shots[s].nt;
}
__device__ __forceinline__ bool shot_active(const FusedLaunch& L, int s) {
  return s < 64 ? ((L.active_mask >> s) & 1ull) != 0 : L.shots[s].active != 0;
}

// What launch `it` does for a shot of record length nt (all threads agree).
struct ShotStep {
  bool step;   // a stencil step of this shot
  bool defer;  // the deferred work of step it - 1
  __device__ __forceinline__ bool tile() const { return step; }
};
template <int MODE>
__device__ __forceinline__ ShotStep shot_step(const FusedLaunch& L, int nt, bool active, int it) {
  ShotStep s;
  s.step = active && it <= nt && it <= L.step_last;
  s.defer = active && it > L.first && it - 1 <= nt;
  return s;
}

// The tile is loaded when it has a stencil step or, in stage A, the deferred
// history store of the previous step.
template <int MODE>
__device__ __forceinline__ bool needs_tile(const ShotStep& s) {
  return s.step || (MODE == FM_STAGE_A && s.defer);
}

// True when every pressure point of the tile and its halo and every velocity
// point of the tile is updated, physical (sponge factors exactly 1), below the
// free-surface rows and, for the final esource, inside the source range.
template <int TC>
__device__ __forceinline__ bool step_interior(const Grid& g, int r0, int c0, int mode, int slo,
                                              int shi1, int shi2) {
  const int off = (mode == FM_FWD) ? 2 : 3;
  const int fsrows = g.ofs == 1 ? g.npml + 1 : 0;
  const int rlo = max(max(2, g.npml + slo), fsrows);
  const int rhi = min(g.n1e - off, g.npml + shi1);
  const int clo = max(2, g.npml + slo);
  const int chi = min(g.n2e - off, g.npml + shi2);
  return r0 - 1 >= rlo && r0 + SR + 2 <= rhi && c0 - 1 >= clo && c0 + TC + 2 <= chi;
}

__device__ __forceinline__ float* fld(const ShotDevice& sd, int par, int f) {
  if (par == 0) return f == 0 ? sd.px : f == 1 ? sd.pz : f == 2 ? sd.vx : sd.vz;
  return f == 0 ? sd.px2 : f == 1 ? sd.pz2 : f == 2 ? sd.vx2 : sd.vz2;
}

// Hicks gather of station s of p = px + pz (rows < fs_lim in the station's
// index frame are the free-surface rows, p = 0 there), summed in the
// reference's order by lane 0 (as warp_gather_ordered).
__device__ __forceinline__ float warp_gather_pxpz(float* prod, const int* ix1p, const int* ix2p,
                                                  const float* tiles, int s,
                                                  const float* __restrict__ opx,
                                                  const float* __restrict__ opz, int ld,
                                                  int shift, int hi1, int hi2, int fs_lim) {
  const int lane = threadIdx.x & 31;
  const int ix1 = __ldg(ix1p + s) - shift, ix2 = __ldg(ix2p + s) - shift;
  const int r1a = max(1 - ix1, -kRad), r1b = min(hi1 - ix1, kRad);
  const int r2a = max(1 - ix2, -kRad), r2b = min(hi2 - ix2, kRad);
  const float* tile = tiles + (size_t)s * kTile;
  constexpr int kSteps = (kGatherStride + 31) / 32;
  float tv[kSteps], xv[kSteps], zv[kSteps];
  bool fz[kSteps];
  {
    int a = lane / kTap - kRad, b = lane % kTap - kRad;
#pragma unroll
    for (int k = 0; k < kSteps; ++k) {
      const int t = lane + 32 * k;
      const bool in = t < kTile && a >= r1a && a <= r1b && b >= r2a && b <= r2b;
      const size_t o = (size_t)(ix1 + a - 1) + (size_t)ld * (ix2 + b - 1);
      tv[k] = in ? __ldg(tile + (a + kRad) + kTap * (b + kRad)) : 0.f;
      xv[k] = in ? opx[o] : 0.f;
      zv[k] = in ? opz[o] : 0.f;
      fz[k] = ix1 + a - 1 < fs_lim;
      b += 32 - kTap;
      a += 1;
      if (b > kRad) {
        b -= kTap;
        a += 1;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kSteps; ++k)
    if (lane + 32 * k < kGatherStride)
      prod[lane + 32 * k] = fmul(tv[k], fz[k] ? 0.f : fadd(xv[k], zv[k]));
  __syncwarp();
  float acc = 0.f;
  if (lane == 0) {
    const float4* p4 = reinterpret_cast<const float4*>(prod);
#pragma unroll 4
    for (int q = 0; q < kGatherStride / 4 - 0; ++q) {
      if (4 * q >= kTile) break;
      const float4 v = p4[q];
      acc = fadd(acc, v.x);
      acc = fadd(acc, v.y);
      acc = fadd(acc, v.z);
      acc = fadd(acc, v.w);
    }
  }
  __syncwarp();
  return acc;
}

template <int MODE, bool FP16, int TC>
__global__ void __launch_bounds__(kT, TC == 16 ? 3 : 2)
    k_step(const Grid g, const ModelDev m, const FusedLaunch L, const int it) {
  using G = SG<TC>;
  using H = Hist<FP16>;
  constexpr bool kB = G::stage_b(MODE);
  constexpr int kStage = G::stage(MODE, FP16);
  constexpr int CPT = G::CPT, NP = G::NP;
  constexpr bool kInj = (MODE == FM_FWD || MODE == FM_STAGE_A);
  extern __shared__ __align__(128) unsigned char smem[];
  float* amp_s = reinterpret_cast<float*>(smem + 2 * kStage);
  // injection band of the tile in each stage (written one item ahead):
  // per box column the first band row (clipped), the map's col_lo and
  // col_base, the prefix of band points, then the count of band points
  int* binfo0 = reinterpret_cast<int*>(smem + 2 * kStage + G::amp_bytes(MODE));
  uint64_t* bar = reinterpret_cast<uint64_t*>(binfo0 + 2 * kBandInts);
  int* item_s = reinterpret_cast<int*>(bar + 2);            // item of each stage
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    bar_init(&bar[0]);
    bar_init(&bar[1]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  pdl_trigger();
  // the previous launch's fields, scales, outputs and queue counts are complete
  pdl_wait();
  const int hbase = g.hist_base();
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int fsrows = g.ofs == 1 ? npml + 1 : 0;
  const int n1h = L.n1h;
  const size_t nih = (size_t)n1h * g.n2;
  const float dtdx = g.dtdx, dt = g.dt, mdt = fmul(-1.0f, dt);
  const float dtdx_v = fmul(g.dtdx, 1.0f);
  const int slo = (MODE == FM_STAGE_B_ES) ? 1 : 0;
  const int shi1 = (MODE == FM_STAGE_B_ES) ? g.n1 - 1 : g.n1;
  const int shi2 = (MODE == FM_STAGE_B_ES) ? g.n2 - 1 : g.n2;
  const int pin = (L.par0 + it - L.first) & 1;  // input state set
  const int ntile = ((n1e + SR - 1) / SR) * ((n2e + TC - 1) / TC);
  const int ngath = (MODE == FM_STAGE_A) ? 0 : L.ngath;
  const int nitems = (ntile + ngath) * L.nshots;
  const unsigned qbase = (unsigned)(it - L.first) * (unsigned)(nitems + gridDim.x);

  auto issue = [&](const SItem& id, int s) {
    const StepMaps* mp = L.smaps + id.shot;
    unsigned char* st = smem + s * kStage;
    const int nt = shot_nt(L, id.shot);
    const bool hist = kB && it <= nt && it <= L.step_last;
    bar_expect(&bar[s], G::tx(hist, FP16));
    tma_2d(st, &mp->vx[pin], id.r0 - SH, id.c0 - 3, &bar[s]);
    tma_2d(st + G::kVX, &mp->vz[pin], id.r0 - SH, id.c0 - 1, &bar[s]);
    tma_2d(st + G::kVX + G::kF, &mp->px[pin], id.r0 - SH, id.c0 - 1, &bar[s]);
    tma_2d(st + G::kVX + 2 * G::kF, &mp->pz[pin], id.r0 - SH, id.c0 - 1, &bar[s]);
    tma_2d(st + G::kVX + 3 * G::kF, &mp->kap, id.r0 - SH, id.c0 - 1, &bar[s]);
    if (hist) {
      const int hs = (nt - it + 1) - 1 - L.hist_step0;  // history slot of step nt - it + 1
      const uint64_t pol = l2_evict_first();
      tma_3d(st + G::kBase, &mp->histp, id.r0 - hbase - 8, id.c0 - 1 - npml, hs * 3, &bar[s], pol);
      unsigned char* hv = st + G::kBase + pad128(G::hp_bytes(FP16));
      tma_3d(hv, &mp->histv, id.r0 - hbase, id.c0 - npml, hs * 3 + 1, &bar[s], pol);
      tma_3d(hv + G::hv_bytes(FP16), &mp->histv, id.r0 - hbase, id.c0 - npml, hs * 3 + 2, &bar[s],
             pol);
    }
  };
  // Thread 0 takes items from the queue two ahead of the one the CTA works
  // on, so the atomic's latency hides behind a tile; it stops after the first
  // index past the end (one such index per CTA and launch).
  auto take = [&]() { return (int)(atomicAdd(L.qctr, 1u) - qbase); };
  auto issue_if_tile = [&](int idx, int s) {
    const SItem id = item_of<TC>(g, idx, L.nshots, ntile, ngath);
    if (id.kind != 0 || !shot_active(L, id.shot)) return;
    const ShotStep ss = shot_step<MODE>(L, shot_nt(L, id.shot), true, it);
    if (needs_tile<MODE>(ss)) issue(id, s);
  };
  // Band of the injection map at the tile's pressure points (warp 0): the
  // loads are issued when the tile is next in line, the counts and prefix
  // are stored into its stage's band info at the end of the current item.
  struct BandLoads {
    int olo[2], ohi[2], base[2];
  };
  auto band_load = [&](const SItem& id, const InjMapDev& mp) {
    BandLoads r;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int cc = lane + 32 * h;  // box column: global column c0 - 1 + cc
      const int c = id.c0 - 1 + cc;
      const bool ok = cc < NP && c >= 0 && c < n2e;
      r.olo[h] = ok ? __ldg(mp.col_lo + c) : 0x7fffffff;
      r.ohi[h] = ok ? __ldg(mp.col_hi + c) : -1;
      r.base[h] = ok ? __ldg(mp.col_base + c) : 0;
    }
    return r;
  };
  auto band_store = [&](const SItem& id, const BandLoads& r, int slot) {
    int* bi = binfo0 + slot * kBandInts;
    int cnt[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int cc = lane + 32 * h;
      const bool tcol = cc >= 1 && cc <= TC;
      const int dlo = tcol ? id.r0 - 1 : id.r0;
      const int dhi = min(tcol ? id.r0 + SR + 1 : id.r0 + SR - 1, n1e - 1);
      const int lo = max(r.olo[h], max(dlo, 0));
      const int hi = min(r.ohi[h], dhi);
      cnt[h] = hi >= lo ? hi - lo + 1 : 0;
      if (cc < kMaxBandCols) {
        bi[cc] = lo;
        bi[kMaxBandCols + cc] = r.olo[h];
        bi[2 * kMaxBandCols + cc] = r.base[h];
      }
    }
    int incl0 = cnt[0], incl1 = cnt[1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y0 = __shfl_up_sync(kAll, incl0, o);
      const int y1 = __shfl_up_sync(kAll, incl1, o);
      if (lane >= o) {
        incl0 += y0;
        incl1 += y1;
      }
    }
    const int tot0 = __shfl_sync(kAll, incl0, 31);
    const int tot1 = __shfl_sync(kAll, incl1, 31);
    bi[3 * kMaxBandCols + lane] = incl0 - cnt[0];
    if (lane + 32 < kMaxBandCols) bi[3 * kMaxBandCols + lane + 32] = tot0 + incl1 - cnt[1];
    if (lane == 0) bi[4 * kMaxBandCols] = tot0 + tot1;
  };
  if (tid == 0) {
    const int i0 = take();
    item_s[0] = i0;
    item_s[1] = i0 < nitems ? take() : nitems;
    issue_if_tile(i0, 0);
  }
  __syncthreads();
  if (kInj && warp == 0) {
    const SItem i0 = item_of<TC>(g, item_s[0], L.nshots, ntile, ngath);
    if (i0.kind == 0) band_store(i0, band_load(i0, L.shots[i0.shot].inj), 0);
  }
  __syncthreads();

  uint32_t phase[2] = {0, 0};
  int cur = -1;
  __shared__ __align__(16) ShotDevice sd_s;  // descriptor of the current shot
  const ShotDevice& sd = sd_s;
  ShotStep ss{false, false};
  bool active = false;
  float inv_p = 1.f, inv_vx = 1.f, inv_vz = 1.f, sc_p = 1.f, sc_vx = 1.f, sc_vz = 1.f;
  void* hdef = nullptr;  // stage A: history slot of step it - 1
  bool amp_smem = true;
  unsigned lmp = 0, lmx = 0, lmz = 0;
  const uint64_t pol_first = l2_evict_first();

  auto flush_amax = [&]() {
    if (MODE == FM_STAGE_A && cur >= 0 && ss.step) {
      unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + ((blockIdx.x * 8 + warp) % kAmaxSlots);
      warp_amax_flush(lmp, a, L.err);
      warp_amax_flush(lmx, a + kAmaxSlots, L.err);
      warp_amax_flush(lmz, a + 2 * kAmaxSlots, L.err);
    }
    lmp = lmx = lmz = 0;
  };

  for (int k = 0;; ++k) {
    const int s = k & 1;
    const SItem id = item_of<TC>(g, item_s[s], L.nshots, ntile, ngath);
    if (id.kind == 2) break;
    const int nidx = item_s[s ^ 1];
    const SItem nxt = item_of<TC>(g, nidx, L.nshots, ntile, ngath);
    int pend = nitems;  // item k + 2 (thread 0)
    if (tid == 0) {
      issue_if_tile(nidx, s ^ 1);
      if (nidx < nitems) pend = take();
    }
    if (id.shot != cur) {  // CTA-uniform: shot set-up
      flush_amax();
      __syncthreads();  // every thread is done with the previous descriptor
      cur = id.shot;
      {
        static_assert(sizeof(ShotDevice) % 4 == 0, "descriptor words");
        const unsigned* src = reinterpret_cast<const unsigned*>(L.shots + cur);
        unsigned* dst = reinterpret_cast<unsigned*>(&sd_s);
        for (int q = tid; q < (int)(sizeof(ShotDevice) / 4); q += kT) dst[q] = __ldg(src + q);
      }
      __syncthreads();
      active = sd.active != 0;
      const int nt = sd.nt;
      ss = shot_step<MODE>(L, nt, active, it);
      if (FP16 && MODE == FM_STAGE_A && ss.defer) {
        const unsigned* a = sd.amax + (size_t)(it - 2) * 3 * kAmaxSlots;
        inv_p = pow2f(15 - amax_exponent(warp_amax_slots(a)));
        inv_vx = pow2f(15 - amax_exponent(warp_amax_slots(a + kAmaxSlots)));
        inv_vz = pow2f(15 - amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)));
      }
      if (MODE == FM_STAGE_A && ss.defer) hdef = step_ptr<FP16>(sd.hist, it - 2, nih);
      if (FP16 && kB && ss.step) {
        const unsigned* a = sd.amax + (size_t)(nt - it - L.hist_step0) * 3 * kAmaxSlots;
        sc_p = pow2f(amax_exponent(warp_amax_slots(a)) - 15);
        sc_vx = pow2f(amax_exponent(warp_amax_slots(a + kAmaxSlots)) - 15);
        sc_vz = pow2f(amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)) - 15);
      }
      const bool inj = kInj && ss.step && (MODE == FM_STAGE_A || sd.type_src == 0);
      amp_smem = kInj && sd.inj.nsta <= kAmpMaxS;
      if (inj && amp_smem) {
        const float* src = (cur < L.nparam && L.shot_amp[cur]) ? L.shot_amp[cur] : nullptr;
        for (int q = tid; q < sd.inj.nsta; q += kT)
          amp_s[q] = src ? __ldg(src + (size_t)(it - 1) * sd.inj.nsta + q)
                         : __ldg(sd.amp + (it - 1) + (size_t)q * sd.amp_stride);
      }
      __syncthreads();
    }
    // band loads of the next tile, stored at the end of this item
    const bool nb_on = kInj && warp == 0 && nxt.kind == 0;
    BandLoads nb;
    if (nb_on) nb = band_load(nxt, nxt.shot == cur ? sd.inj : L.shots[nxt.shot].inj);
    do {  // the item; `break` ends it
    if (id.kind == 1) {
      // ---- gather unit: receivers / datum of step it - 1 from the input set
      if (ss.defer && MODE != FM_STAGE_A) {
        float* prod = reinterpret_cast<float*>(smem) + warp * kGatherStride;
        const int sta = id.unit * 8 + warp;
        const float* opx = fld(sd, pin, 0);
        const float* opz = fld(sd, pin, 1);
        const int step = it - 1;
        if (sta < sd.rec.n) {
          if (sd.out && sd.type_rec == 0) {
            const float v = warp_gather_pxpz(prod, sd.rec.ix1, sd.rec.ix2, sd.rec.tile, sta, opx,
                                             opz, ld, 0, n1e, n2e, fsrows);
            const int row = sd.out_reverse ? sd.nt - step : step - 1;
            if (lane == 0) sd.out[row + (size_t)sd.nt * sta] = v;
          }
        } else if (sta - sd.rec.n < sd.datum.n && sd.red &&
                   (MODE == FM_FWD || MODE == FM_STAGE_B_ES)) {
          const int d = sta - sd.rec.n;
          const size_t o = (size_t)npml + (size_t)ld * npml;
          const float v = warp_gather_pxpz(prod, sd.datum.ix1, sd.datum.ix2, sd.datum.tile, d,
                                           opx + o, opz + o, ld, npml, g.n1, g.n2,
                                           fsrows - npml);
          if (lane == 0) sd.red[(step - 1) + (size_t)sd.nt * d] = v;
        }
      }
      break;
    }
    // ---- tile
    if (!(needs_tile<MODE>(ss) && active)) break;
    const int r0 = id.r0, c0 = id.c0;
    const bool interior = step_interior<TC>(g, r0, c0, MODE, slo, shi1, shi2);
    // Injection band of the tile's pressure points (forward source / stage-A
    // receivers), stored with the previous item: per box column, the clipped
    // band rows; their total count.
    const bool inj = kInj && ss.step && (MODE == FM_STAGE_A || sd.type_src == 0);
    const int* bi = binfo0 + s * kBandInts;
    const int* b_lo = bi;
    const int* b_olo = bi + kMaxBandCols;
    const int* b_base = bi + 2 * kMaxBandCols;
    const int* b_pre = bi + 3 * kMaxBandCols;
    const int nband = inj ? bi[4 * kMaxBandCols] : 0;
    const int i1 = r0 + 2 * lane;
    const int cb = c0 + CPT * warp;
    bar_wait(&bar[s], phase[s], L.err);
    phase[s] ^= 1;
    unsigned char* st = smem + s * kStage;
    float* VXf = reinterpret_cast<float*>(st);
    float* VZf = reinterpret_cast<float*>(st + G::kVX);
    float* PXf = reinterpret_cast<float*>(st + G::kVX + G::kF);
    float* PZf = reinterpret_cast<float*>(st + G::kVX + 2 * G::kF);
    const float* KAf = reinterpret_cast<const float*>(st + G::kVX + 3 * G::kF);
    const unsigned char* HP = st + G::kBase;
    const unsigned char* HV = st + G::kBase + pad128(G::hp_bytes(FP16));
    const int pout = pin ^ 1;
    float* opx = fld(sd, pout, 0);
    float* opz = fld(sd, pout, 1);
    float* ovx = fld(sd, pout, 2);
    float* ovz = fld(sd, pout, 3);
    const bool ok0 = i1 < n1e, ok1 = i1 + 1 < n1e;
    const bool u0 = ok0 && i1 >= 2 && i1 < hi1, u1 = ok1 && i1 + 1 >= 2 && i1 + 1 < hi1;
    const bool r0p = ok0 && i1 >= npml && i1 < npml + g.n1;
    const bool r1p = ok1 && i1 + 1 >= npml && i1 + 1 < npml + g.n1;
    const bool s0 = r0p && i1 - npml >= slo && i1 - npml < shi1;
    const bool s1 = r1p && i1 + 1 - npml >= slo && i1 + 1 - npml < shi1;
    const int h1 = i1 - hbase;
    const int rr = 2 * lane + SH;  // box row of i1

    // ---- pressure on the tile's own points (+ deferred stage-A history of step it - 1)
    auto p_main = [&](auto interior_tag) {
      constexpr bool IN = decltype(interior_tag)::value;
      const bool ok0_ = IN || ok0, ok1_ = IN || ok1, u0_ = IN || u0, u1_ = IN || u1;
      const bool r0_ = IN || r0p, r1_ = IN || r1p, s0_ = IN || s0, s1_ = IN || s1;
      if (!ok0_) return;
      float2 q[CPT + 3];  // vx rows (i1, i1+1) at columns cb-2 .. cb+CPT
#pragma unroll
      for (int kk = 0; kk < CPT + 3; ++kk)
        q[kk] = *reinterpret_cast<const float2*>(VXf + (CPT * warp + 1 + kk) * SB + rr);
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int c = cb + j;
        if (!IN && c >= n2e) continue;
        const int pc = CPT * warp + j + 1;  // box column of c
        const size_t kg = (size_t)i1 + (size_t)ld * c;
        const float* vzc = VZf + pc * SB + rr;
        const float2 zm = *reinterpret_cast<const float2*>(vzc - 2);
        const float2 z = *reinterpret_cast<const float2*>(vzc);
        const float zp2 = vzc[2];
        float2* pxp = reinterpret_cast<float2*>(PXf + pc * SB + rr);
        float2* pzp = reinterpret_cast<float2*>(PZf + pc * SB + rr);
        float2 px_ = *pxp, pz_ = *pzp;
        const float2 kv = *reinterpret_cast<const float2*>(KAf + pc * SB + rr);
        const int i2p = c - npml;
        const bool cint = IN || (i2p >= 0 && i2p < g.n2);
        if (MODE == FM_STAGE_A && ss.defer && cint && (r0_ || r1_)) {
          // histories of step it - 1: p = px + pz (free-surface rows zero), vx, vz
          const float pa = (!IN && i1 < fsrows) ? 0.f : fadd(px_.x, pz_.x);
          const float pb = (!IN && i1 + 1 < fsrows) ? 0.f : fadd(px_.y, pz_.y);
          const int ho = h1 + n1h * i2p;
          H::put2(hdef, ho, pa, pb, inv_p, r0_, r1_, pol_first);
          H::put2(hdef, (int)nih + ho, q[j + 2].x, q[j + 2].y, inv_vx, r0_, r1_, pol_first);
          H::put2(hdef, 2 * (int)nih + ho, z.x, z.y, inv_vz, r0_, r1_, pol_first);
        }
        if (!ss.step) continue;
        if (IN || (c >= 2 && c < hi2)) {
          const bool fwd = (MODE != FM_STAGE_A);
          // sponge profiles (exactly 1 on interior tiles, which skip them)
          float d2a = 1.f, d2a1 = 1.f;
          float2 d1a = make_float2(1.f, 1.f), d1a1 = make_float2(1.f, 1.f);
          if (!IN) {
            const float4 pc4 = __ldg(m.pcol + c);
            const float4 r04 = __ldg(m.prow + i1);
            const float4 r14 = ok1_ ? __ldg(m.prow + i1 + 1) : r04;
            d2a = pc4.x;
            d2a1 = pc4.y;
            d1a = make_float2(r04.x, r14.x);
            d1a1 = make_float2(r04.y, r14.y);
          }
          if (u0_) {
            const float der2 = dminus(q[j].x, q[j + 1].x, q[j + 2].x, q[j + 3].x);
            const float der1 = dminus(zm.x, zm.y, z.x, z.y);
            const float kd = fmul(dtdx, kv.x);
            const float ax = IN ? px_.x : fmul(d2a, px_.x);
            const float bx = IN ? fmul(kd, der2) : fmul(fmul(kd, d2a1), der2);
            const float az = IN ? pz_.x : fmul(d1a.x, pz_.x);
            const float bz = IN ? fmul(kd, der1) : fmul(fmul(kd, d1a1.x), der1);
            px_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
            pz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
          }
          if (u1_) {
            const float der2 = dminus(q[j].y, q[j + 1].y, q[j + 2].y, q[j + 3].y);
            const float der1 = dminus(zm.y, z.x, z.y, zp2);
            const float kd = fmul(dtdx, kv.y);
            const float ax = IN ? px_.y : fmul(d2a, px_.y);
            const float bx = IN ? fmul(kd, der2) : fmul(fmul(kd, d2a1), der2);
            const float az = IN ? pz_.y : fmul(d1a.y, pz_.y);
            const float bz = IN ? fmul(kd, der1) : fmul(fmul(kd, d1a1.y), der1);
            px_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
            pz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
          }
        }
        if (kB && (IN || (i2p >= slo && i2p < shi2)) && (s0_ || s1_)) {
          const int e = pc * kHPRows + 2 * lane + 8;  // history box row of i1
          const float2 hv = FP16 ? __half22float2(*reinterpret_cast<const __half2*>(
                                       reinterpret_cast<const __half*>(HP) + e))
                                 : *reinterpret_cast<const float2*>(reinterpret_cast<const float*>(HP) + e);
          if (s0_) px_.x = fadd(px_.x, fmul(fmul(mdt, hv.x * sc_p), kv.x));
          if (s1_) px_.y = fadd(px_.y, fmul(fmul(mdt, hv.y * sc_p), kv.y));
        }
        if (nband > 0) {  // injection pass follows: keep px, pz in the stage
          *pxp = px_;
          *pzp = pz_;
          continue;
        }
        float2 pv;
        pv.x = (!IN && i1 < fsrows) ? 0.f : fadd(px_.x, pz_.x);
        pv.y = (!IN && i1 + 1 < fsrows) ? 0.f : fadd(px_.y, pz_.y);
        if (ok1_) {
          *reinterpret_cast<float2*>(opx + kg) = px_;
          *reinterpret_cast<float2*>(opz + kg) = pz_;
        } else {
          opx[kg] = px_.x;
          opz[kg] = pz_.x;
        }
        pxp->x = pv.x;  // the stage now holds p for the velocity update
        pxp->y = pv.y;
        if (cint) {
          if (MODE == FM_STAGE_A) {
            if (r0_) lmp = max(lmp, abs_bits(pv.x));
            if (r1_) lmp = max(lmp, abs_bits(pv.y));
          }
          if ((MODE == FM_FWD || MODE == FM_STAGE_B_ES) && sd.wf && sd.type_rec == 0) {
            float* w = sd.wf + (size_t)(it - 1) * g.int_elems() + (size_t)g.n1 * i2p;
            const int i1p = i1 - npml;
            if (MODE == FM_FWD) {
              if (r0_) w[i1p] = pv.x;
              if (r1_) w[i1p + 1] = pv.y;
            } else {
              if (r0_) w[i1p] = fadd(w[i1p], pv.x);
              if (r1_) w[i1p + 1] = fadd(w[i1p + 1], pv.y);
            }
          }
        }
      }
    };
    // ---- pressure on the halo points (one point per thread per pass)
    auto p_halo = [&](auto interior_tag) {
      constexpr bool IN = decltype(interior_tag)::value;
      for (int hh = tid; hh < G::kHalo; hh += kT) {
        int i, c;
        if (hh < 3 * SR) {
          const int hc = hh / SR;
          c = hc == 0 ? c0 - 1 : c0 + TC + hc - 1;
          i = r0 + (hh - hc * SR);
        } else {
          const int kk = hh - 3 * SR, hr = kk / TC;
          i = hr == 0 ? r0 - 1 : r0 + SR + hr - 1;
          c = c0 + (kk - hr * TC);
        }
        const int pc = c - (c0 - 1), rw = i - (r0 - SH);
        float* pxp = PXf + pc * SB + rw;
        float* pzp = PZf + pc * SB + rw;
        if (!IN && (i < 0 || i >= n1e || c < 0 || c >= n2e)) {  // never read by an update
          *pxp = 0.f;
          *pzp = 0.f;
          continue;
        }
        float px_ = *pxp, pz_ = *pzp;
        const float kv = KAf[pc * SB + rw];
        const bool upd = IN || (i >= 2 && i < hi1 && c >= 2 && c < hi2);
        if (upd) {
          const float* vxc = VXf + (c - (c0 - 3)) * SB + rw;
          const float der2 = dminus(vxc[-2 * SB], vxc[-SB], vxc[0], vxc[SB]);
          const float* vzc = VZf + pc * SB + rw;
          const float der1 = dminus(vzc[-2], vzc[-1], vzc[0], vzc[1]);
          const float kd = fmul(dtdx, kv);
          const bool fwd = (MODE != FM_STAGE_A);
          float ax, bx, az, bz;
          if (IN) {
            ax = px_; bx = fmul(kd, der2); az = pz_; bz = fmul(kd, der1);
          } else {
            const float4 pc4 = __ldg(m.pcol + c), pr4 = __ldg(m.prow + i);
            ax = fmul(pc4.x, px_);
            bx = fmul(fmul(kd, pc4.y), der2);
            az = fmul(pr4.x, pz_);
            bz = fmul(fmul(kd, pr4.y), der1);
          }
          px_ = fwd ? fadd(ax, bx) : fsub(ax, bx);
          pz_ = fwd ? fadd(az, bz) : fsub(az, bz);
        }
        if (kB) {
          const int i1p = i - npml, i2p = c - npml;
          const bool src = IN || (i1p >= slo && i1p < shi1 && i2p >= slo && i2p < shi2);
          if (src) {
            const int e = pc * kHPRows + (i - (r0 - 8));
            const float hv = FP16 ? __half2float(reinterpret_cast<const __half*>(HP)[e])
                                  : reinterpret_cast<const float*>(HP)[e];
            px_ = fadd(px_, fmul(fmul(mdt, hv * sc_p), kv));
          }
        }
        if (nband > 0) {
          *pxp = px_;
          *pzp = pz_;
        } else {
          *pxp = (!IN && i < fsrows) ? 0.f : fadd(px_, pz_);
        }
      }
    };
    if (interior) {
      p_main(std::true_type{});
      if (ss.step) p_halo(std::true_type{});
    } else {
      p_main(std::false_type{});
      if (ss.step) p_halo(std::false_type{});
    }
    if (ss.step && nband > 0) {
      // ---- injection into px at the band points (gather form, station order)
      __syncthreads();
      const int2* rp2 = reinterpret_cast<const int2*>(sd.inj.rowptr);
      const uint64_t pol = l2_evict_last();
      const float* amp_g = sd.amp + (it - 1);
      const int sg = (MODE == FM_FWD) ? 1 : -1;
      for (int f0 = tid; f0 < nband; f0 += 2 * kT) {
        int e0[2], e1[2], rw[2], pcol[2];
        bool on[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int f = f0 + u * kT;
          on[u] = f < nband;
          e0[u] = e1[u] = 0;
          rw[u] = 0;
          pcol[u] = 0;
          if (on[u]) {
            int lo = 0, hi = NP - 1;  // last box column whose prefix <= f
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (b_pre[mid] <= f) lo = mid; else hi = mid - 1;
            }
            const int r = b_lo[lo] + (f - b_pre[lo]);
            pcol[u] = lo;
            rw[u] = r - (r0 - SH);
            const int2 q = ld_hint_i2(rp2 + b_base[lo] + (r - b_olo[lo]), pol);
            e0[u] = q.x;
            e1[u] = q.y;
          }
        }
        float2 qe[2][kBatchS];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int kk = 0; kk < kBatchS; ++kk)
            qe[u][kk] = e0[u] + kk < e1[u] ? ld_hint_f2(sd.inj.ent + e0[u] + kk, pol)
                                           : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int kk = 0; kk < kBatchS; ++kk) {
            const int sta = __float_as_int(qe[u][kk].y);
            qe[u][kk].y = amp_smem ? amp_s[sta] : __ldg(amp_g + (size_t)sta * sd.amp_stride);
          }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (!on[u]) continue;
          float* pxp = PXf + pcol[u] * SB + rw[u];
          const float kv = KAf[pcol[u] * SB + rw[u]];
          float v = *pxp;
#pragma unroll
          for (int kk = 0; kk < kBatchS; ++kk) {
            const float t = fmul(fmul(fmul(qe[u][kk].x, dt), qe[u][kk].y), kv);
            if (e0[u] + kk < e1[u]) v = sg > 0 ? fadd(v, t) : fsub(v, t);
          }
          for (int e = e0[u] + kBatchS; e < e1[u]; ++e) {
            const float2 q1 = ld_hint_f2(sd.inj.ent + e, pol);
            const int sta = __float_as_int(q1.y);
            const float a1 = amp_smem ? amp_s[sta] : __ldg(amp_g + (size_t)sta * sd.amp_stride);
            const float t = fmul(fmul(fmul(q1.x, dt), a1), kv);
            v = sg > 0 ? fadd(v, t) : fsub(v, t);
          }
          *pxp = v;
        }
      }
      __syncthreads();
      // ---- p = px + pz; the tile's px, pz to global
      if (ok0) {
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int c = cb + j;
          if (c >= n2e) continue;
          const int pc = CPT * warp + j + 1;
          const size_t kg = (size_t)i1 + (size_t)ld * c;
          float2* pxp = reinterpret_cast<float2*>(PXf + pc * SB + rr);
          const float2 px_ = *pxp, pz_ = *reinterpret_cast<const float2*>(PZf + pc * SB + rr);
          float2 pv;
          pv.x = i1 < fsrows ? 0.f : fadd(px_.x, pz_.x);
          pv.y = i1 + 1 < fsrows ? 0.f : fadd(px_.y, pz_.y);
          if (ok1) {
            *reinterpret_cast<float2*>(opx + kg) = px_;
            *reinterpret_cast<float2*>(opz + kg) = pz_;
          } else {
            opx[kg] = px_.x;
            opz[kg] = pz_.x;
          }
          *pxp = pv;
          const int i2p = c - npml;
          if (i2p >= 0 && i2p < g.n2) {
            if (MODE == FM_STAGE_A) {
              if (r0p) lmp = max(lmp, abs_bits(pv.x));
              if (r1p) lmp = max(lmp, abs_bits(pv.y));
            }
            if (MODE == FM_FWD && sd.wf && sd.type_rec == 0) {
              float* w = sd.wf + (size_t)(it - 1) * g.int_elems() + (size_t)g.n1 * i2p;
              if (r0p) w[i1 - npml] = pv.x;
              if (r1p) w[i1 - npml + 1] = pv.y;
            }
          }
        }
      }
      for (int hh = tid; hh < G::kHalo; hh += kT) {
        int i, c;
        if (hh < 3 * SR) {
          const int hc = hh / SR;
          c = hc == 0 ? c0 - 1 : c0 + TC + hc - 1;
          i = r0 + (hh - hc * SR);
        } else {
          const int kk = hh - 3 * SR, hr = kk / TC;
          i = hr == 0 ? r0 - 1 : r0 + SR + hr - 1;
          c = c0 + (kk - hr * TC);
        }
        const int pc = c - (c0 - 1), rw = i - (r0 - SH);
        float* pxp = PXf + pc * SB + rw;
        *pxp = (i < fsrows) ? 0.f : fadd(*pxp, PZf[pc * SB + rw]);
      }
    }
    if (ss.step) {
      __syncthreads();  // p of the tile and its halo is in the stage
      // ---- velocity update of the tile
      auto v_pass = [&](auto interior_tag) {
        constexpr bool IN = decltype(interior_tag)::value;
        const bool ok0_ = IN || ok0, ok1_ = IN || ok1, u0_ = IN || u0, u1_ = IN || u1;
        const bool r0_ = IN || r0p, r1_ = IN || r1p;
        if (!ok0_) return;
        const bool fs = g.ofs == 1;
        const bool dst_x = !IN && fs && i1 == npml - 1;
        const bool skip_y = !IN && fs && i1 + 1 == npml - 1;
        const bool src_x = !IN && fs && i1 == npml;
        float2 a[CPT + 3];  // p rows (i1, i1+1) at columns cb-1 .. cb+CPT+1
#pragma unroll
        for (int kk = 0; kk < CPT + 3; ++kk)
          a[kk] = *reinterpret_cast<const float2*>(PXf + (CPT * warp + kk) * SB + rr);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int c = cb + j;
          if (!IN && c >= n2e) continue;
          const int pc = CPT * warp + j + 1;
          const size_t kg = (size_t)i1 + (size_t)ld * c;
          const float* pcol = PXf + pc * SB + rr;
          const float pm1 = pcol[-1];
          const float2 pcv = a[j + 1];
          const float2 pp = *reinterpret_cast<const float2*>(pcol + 2);
          const int i2p = c - npml;
          const bool cint = IN || (i2p >= 0 && i2p < g.n2);
          float2 vx_ = *reinterpret_cast<const float2*>(VXf + (CPT * warp + j + 3) * SB + rr);
          float2 vz_ = *reinterpret_cast<const float2*>(VZf + pc * SB + rr);
          if (IN || (c >= 2 && c < hi2)) {
            const bool fwd = (MODE != FM_STAGE_A);
            float d2b = 1.f, bw2 = dtdx_v;
            float2 d1b = make_float2(1.f, 1.f), bw1 = make_float2(dtdx_v, dtdx_v);
            if (!IN) {
              const float4 pc4 = __ldg(m.pcol + c);
              const float4 r04 = __ldg(m.prow + i1);
              const float4 r14 = ok1_ ? __ldg(m.prow + i1 + 1) : r04;
              d2b = pc4.z;
              bw2 = pc4.w;
              d1b = make_float2(r04.z, r14.z);
              bw1 = make_float2(r04.w, r14.w);
            }
            if (u0_) {
              const float der2 = dplus(a[j].x, pcv.x, a[j + 2].x, a[j + 3].x);
              const float der1 = dplus(pm1, pcv.x, pcv.y, pp.x);
              const float ax = IN ? vx_.x : fmul(d2b, vx_.x);
              const float bx = fmul(IN ? dtdx_v : bw2, der2);
              const float az = IN ? vz_.x : fmul(d1b.x, vz_.x);
              const float bz = fmul(IN ? dtdx_v : bw1.x, der1);
              vx_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
              vz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
            }
            if (u1_) {
              const float der2 = dplus(a[j].y, pcv.y, a[j + 2].y, a[j + 3].y);
              const float der1 = dplus(pcv.x, pcv.y, pp.x, pp.y);
              const float ax = IN ? vx_.y : fmul(d2b, vx_.y);
              const float bx = fmul(IN ? dtdx_v : bw2, der2);
              const float az = IN ? vz_.y : fmul(d1b.y, vz_.y);
              const float bz = fmul(IN ? dtdx_v : bw1.y, der1);
              vx_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
              vz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
            }
          }
          if (kB && cint && (r0_ || r1_)) {
            const int e = (CPT * warp + j) * SR + 2 * lane;
            float2 hx, hz;
            if (FP16) {
              const __half* hb = reinterpret_cast<const __half*>(HV);
              hx = __half22float2(*reinterpret_cast<const __half2*>(hb + e));
              hz = __half22float2(*reinterpret_cast<const __half2*>(hb + SR * TC + e));
            } else {
              const float* hb = reinterpret_cast<const float*>(HV);
              hx = *reinterpret_cast<const float2*>(hb + e);
              hz = *reinterpret_cast<const float2*>(hb + SR * TC + e);
            }
            if (r0_) {
              vx_.x = fadd(vx_.x, fmul(fmul(mdt, hx.x * sc_vx), 1.0f));
              vz_.x = fadd(vz_.x, fmul(fmul(mdt, hz.x * sc_vz), 1.0f));
            }
            if (r1_) {
              vx_.y = fadd(vx_.y, fmul(fmul(mdt, hx.y * sc_vx), 1.0f));
              vz_.y = fadd(vz_.y, fmul(fmul(mdt, hz.y * sc_vz), 1.0f));
            }
          }
          if (MODE == FM_FWD && sd.type_src == 1) {  // vz source (type_src = 1)
            const int clo = __ldg(sd.inj.col_lo + c), chi = __ldg(sd.inj.col_hi + c);
            if (i1 + 1 >= clo && i1 <= chi) {
              const int base = __ldg(sd.inj.col_base + c) - clo;
              if (i1 >= clo) vz_.x = inject_at_global(sd.inj, vz_.x, base + i1, dt, 1.0f, sd.amp + (it - 1), sd.amp_stride, +1);
              if (ok1_ && i1 + 1 <= chi)
                vz_.y = inject_at_global(sd.inj, vz_.y, base + i1 + 1, dt, 1.0f, sd.amp + (it - 1), sd.amp_stride, +1);
            }
          }
          if (dst_x) vz_.x = vz_.y;
          if (ok1_) {
            *reinterpret_cast<float2*>(ovx + kg) = vx_;
            if (skip_y)
              ovz[kg] = vz_.x;
            else
              *reinterpret_cast<float2*>(ovz + kg) = vz_;
          } else {
            ovx[kg] = vx_.x;
            ovz[kg] = vz_.x;
          }
          if (src_x) ovz[kg - 1] = vz_.x;
          if (MODE == FM_STAGE_A && cint) {
            if (r0_) {
              lmx = max(lmx, abs_bits(vx_.x));
              lmz = max(lmz, abs_bits(vz_.x));
            }
            if (r1_) {
              lmx = max(lmx, abs_bits(vx_.y));
              lmz = max(lmz, abs_bits(vz_.y));
            }
          }
        }
      };
      if (interior)
        v_pass(std::true_type{});
      else
        v_pass(std::false_type{});
    }
    } while (false);
    if (nb_on) band_store(nxt, nb, s ^ 1);
    if (tid == 0) item_s[s] = pend;
    __syncthreads();  // stage s free for the copies of item k + 2
  }
  flush_amax();
}

template <int MODE, bool FP16, int TC>
void launch_t(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, int grid,
              cudaStream_t st) {
  launch_pdl(k_step<MODE, FP16, TC>, grid, kT, SG<TC>::smem(MODE, FP16), st, L.pdl != 0, g, m, L,
             it);
}

template <int MODE, bool FP16>
void launch_m(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, int grid,
              cudaStream_t st) {
  if (L.tile_cols == 16)
    launch_t<MODE, FP16, 16>(g, m, L, it, grid, st);
  else
    launch_t<MODE, FP16, 32>(g, m, L, it, grid, st);
}

template <int MODE>
void launch_f(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, int grid,
              cudaStream_t st) {
  if (L.hist_fp16)
    launch_m<MODE, true>(g, m, L, it, grid, st);
  else
    launch_m<MODE, false>(g, m, L, it, grid, st);
}

template <int MODE, bool FP16, int TC>
int occ_t() {
  const size_t sm = SG<TC>::smem(MODE, FP16);
  if (cudaFuncSetAttribute(k_step<MODE, FP16, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm) != cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<MODE, FP16, TC>, kT, sm) !=
      cudaSuccess)
    return 0;
  return n;
}

template <int MODE, bool FP16>
int occ_m(int tc) {
  return tc == 16 ? occ_t<MODE, FP16, 16>() : occ_t<MODE, FP16, 32>();
}

}  // namespace

int step_tiles(const Grid& g, int tile_cols) {
  return ((g.n1e + SR - 1) / SR) * ((g.n2e + tile_cols - 1) / tile_cols);
}

int step_occupancy(int mode, bool fp16, int tile_cols) {
  switch (mode) {
    case FM_FWD: return fp16 ? occ_m<FM_FWD, true>(tile_cols) : occ_m<FM_FWD, false>(tile_cols);
    case FM_STAGE_A:
      return fp16 ? occ_m<FM_STAGE_A, true>(tile_cols) : occ_m<FM_STAGE_A, false>(tile_cols);
    case FM_STAGE_B:
      return fp16 ? occ_m<FM_STAGE_B, true>(tile_cols) : occ_m<FM_STAGE_B, false>(tile_cols);
    default:
      return fp16 ? occ_m<FM_STAGE_B_ES, true>(tile_cols) : occ_m<FM_STAGE_B_ES, false>(tile_cols);
  }
}

void step_prepare() {
  for (int mode = 0; mode < 4; ++mode)
    for (int f = 0; f < 2; ++f)
      for (int tc : {16, 32}) step_occupancy(mode, f != 0, tc);
  cudaGetLastError();
}

void step_launch(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                 int grid, cudaStream_t st) {
  switch (mode) {
    case FM_FWD: launch_f<FM_FWD>(g, m, L, it, grid, st); break;
    case FM_STAGE_A: launch_f<FM_STAGE_A>(g, m, L, it, grid, st); break;
    case FM_STAGE_B: launch_f<FM_STAGE_B>(g, m, L, it, grid, st); break;
    default: launch_f<FM_STAGE_B_ES>(g, m, L, it, grid, st); break;
  }
}

// Host: the tensor maps of one shot for tiles of `tile_cols` columns.
bool step_encode_maps(const Grid& g, float* const st[2][4], const float* kap, const void* hist,
                      int hist_fp16, int n1h, int nsteps, int tile_cols, StepMaps* out) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&encode),
                                cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !encode) {
      encode = nullptr;
      return false;
    }
  }
  auto make = [&](CUtensorMap* map, const float* base, int bc) {
    cuuint64_t dims[2] = {(cuuint64_t)g.n1e, (cuuint64_t)g.n2e};
    cuuint64_t strides[1] = {(cuuint64_t)g.ld * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)SB, (cuuint32_t)bc};
    cuuint32_t es[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides,
                  box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
  };
  const int tc = tile_cols;
  bool ok = true;
  for (int p = 0; p < 2; ++p) {
    ok = ok && make(&out->vx[p], st[p][2], tc + 6) && make(&out->vz[p], st[p][3], tc + 3) &&
         make(&out->px[p], st[p][0], tc + 3) && make(&out->pz[p], st[p][1], tc + 3);
  }
  ok = ok && make(&out->kap, kap, tc + 3);
  const size_t esz = hist_fp16 ? 2 : 4;
  const CUtensorMapDataType ht =
      hist_fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  cuuint64_t hd[3] = {(cuuint64_t)n1h, (cuuint64_t)g.n2, (cuuint64_t)3 * nsteps};
  cuuint64_t hs[2] = {(cuuint64_t)n1h * esz, (cuuint64_t)n1h * g.n2 * esz};
  cuuint32_t he[3] = {1, 1, 1};
  cuuint32_t hbp[3] = {(cuuint32_t)kHPRows, (cuuint32_t)(tc + 3), 1};
  cuuint32_t hbv[3] = {(cuuint32_t)SR, (cuuint32_t)tc, 1};
  ok = ok &&
       encode(&out->histp, ht, 3, const_cast<void*>(hist), hd, hs, hbp, he,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
       encode(&out->histv, ht, 3, const_cast<void*>(hist), hd, hs, hbv, he,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  return ok;
}

}  // namespace daw
