// TMA-pipelined persistent time-step kernels (the default fused path).
//
// A persistent CTA (256 threads) walks tiles of 64 depth rows x 32 columns.
// For every tile one thread issues 2-D tensor copies (cp.async.bulk.tensor)
// of the fields the tile needs -- with their stencil halos -- into a
// double-buffered shared-memory stage and arms an mbarrier with the byte
// count; while the CTA computes tile k from stage k&1, the copies of tile
// k+1 are in flight.  The copies zero-fill outside the grid, which supplies
// the boundary values the stencil reads.  Each thread computes 2 rows x 4
// columns from shared memory (conflict-free float2 reads) with the
// reference's separately rounded FP32 operations, and writes its results
// with coalesced float2 stores.
//
// The 1-D sponge profiles and the injection band bounds of a tile are loaded
// into registers before the CTA waits for the tile, so those latencies overlap
// the copy; the shot descriptor and the step's FP16 scales are fetched once
// per shot, not per tile.
//
// Stage A injects the residual at every receiver (441 taps each, summed per
// grid point in station order).  Tiles crossing that band park their
// post-stencil pressure pairs in the stage buffer; after a warp barrier each
// warp finishes the band rows of its own columns with one lane per row,
// issuing the row pointers and the tap entries of several points as batches
// so that the dependent loads overlap.
//
// L2 policy: the history stream (written once, read once) is stored and
// copied with an evict-first hint so it does not push the wavefield state out
// of L2; the injection tables, re-read every step, are loaded evict-last.
//
// Every mbarrier wait is bounded (clock64 budget, ~1 s); on expiry the
// kernel raises the error flag and continues without hanging.
#include <cuda.h>

#include <type_traits>

#include "fused.cuh"
#include "tma.cuh"

namespace daw {
namespace {

constexpr int TR = 64;        // rows per tile
constexpr int TC = 32;        // columns per tile
constexpr int CPT = 4;        // columns per thread (8 warps x 4 = TC)
constexpr int HR = 4;         // row halo (16-byte aligned TMA start)
constexpr int kThreadsT = 256;

// stage layouts (bytes, 128-aligned sections)
constexpr int kPVX = TR * (TC + 3) * 4;       // 8960  vx, columns c0-2..c0+TC
constexpr int kPVZ = (TR + 2 * HR) * TC * 4;  // 9216  vz, rows r0-4..r0+TR+3
constexpr int kPF = TR * TC * 4;              // 8192  px, pz, kappa
constexpr int kPStage = kPVX + kPVZ + 3 * kPF;  // 42752
constexpr int kVPb = (TR + 2 * HR) * (TC + 3) * 4;  // 10080 p, 72 rows x 35 columns
constexpr int kVP = 10112;                    // (padded to 128)
constexpr int kVStage = kVP + 2 * kPF;        // 26496
constexpr int kGatherBytes = 8 * 444 * 4;     // 14208
constexpr int kAmpMax = 2048;                 // stations whose amplitudes are staged in smem
constexpr int kBatch = 6;                     // band-pass entry loads issued per point at once
constexpr int kAmpBytes = kAmpMax * 4;

// Stage sizes by mode/precision: stage B adds the history box(es) of the
// time-reversed step (64 x 32 elements per field).
__host__ __device__ constexpr int hist_box(bool fp16) { return TR * TC * (fp16 ? 2 : 4); }
__host__ __device__ constexpr int p_stage(int mode, bool fp16) {
  return kPStage + ((mode == FM_STAGE_B || mode == FM_STAGE_B_ES) ? hist_box(fp16) : 0);
}
__host__ __device__ constexpr int v_stage(int mode, bool fp16) {
  return kVStage + ((mode == FM_STAGE_B || mode == FM_STAGE_B_ES) ? 2 * hist_box(fp16) : 0);
}
constexpr size_t p_smem(int mode, bool fp16) { return 2 * p_stage(mode, fp16) + 16 + kAmpBytes; }
// The gathers' products (kGatherBytes) reuse the stage buffers after the tiles.
constexpr size_t v_smem(int mode, bool fp16) { return 2 * v_stage(mode, fp16) + 128; }
static_assert(2 * kVStage >= kGatherBytes, "gather products fit in the stage buffers");

// Injection at row i1 of a column band: the (coefficient, station) entries
// of the point in station order, amplitudes of this step staged in `amp`
// (shared memory).
__device__ __forceinline__ float inject_at(const InjMapDev& m, float v, int r, float dt, float w,
                                           const float* amp, int sign) {
  const int e0 = __ldg(m.rowptr + 2 * r), e1 = __ldg(m.rowptr + 2 * r + 1);
#pragma unroll 4
  for (int e = e0; e < e1; ++e) {
    const float2 q = __ldg(m.ent + e);
    const float term = fmul(fmul(fmul(q.x, dt), amp[__float_as_int(q.y)]), w);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  return v;
}

struct TileId {
  int shot, r0, c0;
};

// True when no boundary of the stencil passes crosses the tile: all its rows
// and columns are updated (away from the grid edge), physical (inside the
// PML frame), below the free surface rows and, for the final esource, inside
// the source range [slo, shi).
__device__ __forceinline__ bool tile_interior(const Grid& g, const TileId& id, int mode, int slo,
                                              int shi1, int shi2) {
  const int off = (mode == FM_FWD) ? 2 : 3;
  const int fsrows = g.ofs == 1 ? g.npml + 1 : 0;
  const int rlo = max(max(2, g.npml + slo), fsrows);
  const int rhi = min(min(g.n1e - off, g.npml + shi1), g.n1e);
  const int clo = max(2, g.npml + slo);
  const int chi = min(min(g.n2e - off, g.npml + shi2), g.n2e);
  return id.r0 >= rlo && id.r0 + TR <= rhi && id.c0 >= clo && id.c0 + TC <= chi;
}

// The tiles a persistent CTA walks: first, stride, end (exclusive).  With at
// least one CTA per shot the grid is split into equal groups, one per shot,
// each walking its shot's tiles round robin, so a CTA sets up one shot only
// (CTAs left over from the split walk none); otherwise all tiles round robin.
struct Walk {
  int t0, stride, end;
};
__device__ __forceinline__ Walk tile_walk(int ntiles, int nshots) {
  const int cps = gridDim.x / nshots;
  if (cps == 0) return Walk{(int)blockIdx.x, (int)gridDim.x, ntiles};
  const int sh = blockIdx.x / cps, tps = ntiles / nshots;
  if (sh >= nshots) return Walk{0, 1, 0};
  return Walk{sh * tps + (int)blockIdx.x % cps, cps, (sh + 1) * tps};
}

// Tile t of the launch: group t / tiles-per-shot is live shot L.live[group].
__device__ __forceinline__ TileId tile_id(const Grid& g, int t, const FusedLaunch& L) {
  const int nrb = (g.n1e + TR - 1) / TR, ncb = (g.n2e + TC - 1) / TC;
  const int tps = nrb * ncb;
  TileId id;
  const int grp = t / tps;
  id.shot = L.live[grp];
  const int l = t - grp * tps;
  id.r0 = (l % nrb) * TR;
  id.c0 = (l / nrb) * TC;
  return id;
}

// Two rows (2*lane, 2*lane+1) of column cc of a history box in shared memory.
template <bool FP16>
__device__ __forceinline__ float2 hist_box_read(const unsigned char* box, int cc, int lane) {
  if (FP16)
    return __half22float2(reinterpret_cast<const __half2*>(box)[cc * (TR / 2) + lane]);
  return reinterpret_cast<const float2*>(box)[cc * (TR / 2) + lane];
}

// Stage the step's station amplitudes amp[(it-1) + s*stride] in shared memory
// (CTA-wide; called at a shot change, which is CTA-uniform).
__device__ __forceinline__ void stage_amp(float* amp_s, const float* amp, int stride, int nsta) {
  const int n = min(nsta, kAmpMax);
  for (int s = threadIdx.x; s < n; s += blockDim.x) amp_s[s] = __ldg(amp + (size_t)s * stride);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Pressure kernel
// ---------------------------------------------------------------------------
template <int MODE, bool FP16>
__global__ void __launch_bounds__(kThreadsT, 2)
    k_tma_p(const Grid g, const ModelDev m, const FusedLaunch L, const int it, const int ntiles) {
  using H = Hist<FP16>;
  constexpr bool kB = (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES);
  constexpr int kStage = p_stage(MODE, FP16);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * kStage);
  float* amp_s = reinterpret_cast<float*>(smem + 2 * kStage + 16);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    bar_init(&bar[0]);
    bar_init(&bar[1]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  pdl_trigger();
  __syncthreads();
  pdl_wait();  // the previous step's fields, scales and outputs are complete
  const int hbase = g.hist_base();
  auto issue = [&](int t, int s) {
    const TileId id = tile_id(g, t, L);
    const TmaMaps* mp = L.maps + id.shot;
    unsigned char* st = smem + s * kStage;
    bar_expect(&bar[s], kStage);  // kPStage (+ history box) = bytes copied
    tma_2d(st, &mp->vx19, id.r0, id.c0 - 2, &bar[s]);
    tma_2d(st + kPVX, &mp->vz72, id.r0 - HR, id.c0, &bar[s]);
    tma_2d(st + kPVX + kPVZ, &mp->px, id.r0, id.c0, &bar[s]);
    tma_2d(st + kPVX + kPVZ + kPF, &mp->pz, id.r0, id.c0, &bar[s]);
    tma_2d(st + kPVX + kPVZ + 2 * kPF, &mp->kap, id.r0, id.c0, &bar[s]);
    if (kB) {  // pressure history of the time-reversed step
      // record length from the kernel parameters (no load on the issuing thread's path)
      const int ic = (id.shot < L.nparam ? L.shot_nt[id.shot] : L.shots[id.shot].nt) - it + 1;
      const int hs = ic - 1 - L.hist_step0;  // history slot of step ic
      tma_3d(st + kPStage, &mp->hist, id.r0 - hbase, id.c0 - g.npml, hs * 3, &bar[s],
             l2_evict_first());
    }
  };
  const Walk wk = tile_walk(ntiles, L.nlive);
  int t = wk.t0;
  if (tid == 0 && t < wk.end) issue(t, 0);
  uint32_t phase0 = 0, phase1 = 0;
  int stage = 0;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int fsrows = g.ofs == 1 ? npml + 1 : 0;
  const int n1h = L.n1h;
  const size_t nih = (size_t)n1h * g.n2;
  const float dtdx = g.dtdx, dt = g.dt, mdt = fmul(-1.0f, dt);
  const int slo = (MODE == FM_STAGE_B_ES) ? 1 : 0;
  const int shi1 = (MODE == FM_STAGE_B_ES) ? g.n1 - 1 : g.n1;
  const int shi2 = (MODE == FM_STAGE_B_ES) ? g.n2 - 1 : g.n2;
  int cur = -1;
  ShotDevice sd;
  bool live = false, flush = false, do_inj = false, amp_smem = false;
  float inv_vx = 1.f, inv_vz = 1.f, sc_p = 1.f;
  void* hvs = nullptr;
  unsigned lmax = 0;
  for (; t < wk.end; t += wk.stride) {
    const int tn = t + wk.stride;
    if (tid == 0 && tn < wk.end) issue(tn, stage ^ 1);
    const TileId id = tile_id(g, t, L);
    if (id.shot != cur) {  // CTA-uniform
      if (MODE == FM_STAGE_A && cur >= 0 && live && !flush)
        warp_amax_flush(lmax, sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots +
                                  ((blockIdx.x * 8 + warp) % kAmaxSlots), L.err);
      cur = id.shot;
      if (cur < L.nparam) {
        // one round of independent loads: scale slots, amplitudes, descriptor
        const int ntc = L.shot_nt[cur], nsta = L.shot_nsta[cur];
        const unsigned* am = L.shot_amax[cur];
        unsigned s0v = 0, s1v = 0;
        if (MODE == FM_STAGE_A && FP16 && it >= 2 && it <= ntc + 1) {
          s0v = am[(size_t)(it - 2) * 3 * kAmaxSlots + kAmaxSlots + lane];
          s1v = am[(size_t)(it - 2) * 3 * kAmaxSlots + 2 * kAmaxSlots + lane];
        }
        if (kB && FP16 && it <= ntc)
          s0v = am[(size_t)(ntc - it - L.hist_step0) * 3 * kAmaxSlots + lane];
        constexpr int kPer = kAmpMax / kThreadsT;
        float av[kPer];
        const bool want_amps = (MODE == FM_STAGE_A || MODE == FM_FWD) && it <= ntc &&
                               nsta <= kAmpMax && L.shot_amp[cur] != nullptr;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          const int s = tid + k * kThreadsT;
          av[k] = (want_amps && s < nsta) ? __ldg(L.shot_amp[cur] + (size_t)(it - 1) * nsta + s) : 0.f;
        }
        sd = L.shots[cur];
        live = sd.active && (MODE == FM_STAGE_A ? it <= ntc + 1 : it <= ntc);
        flush = (MODE == FM_STAGE_A) && it == ntc + 1;
        do_inj = live && !flush && ((MODE == FM_STAGE_A) || (MODE == FM_FWD && sd.type_src == 0));
        lmax = 0;
        if (live && MODE == FM_STAGE_A && it >= 2) {
          hvs = step_ptr<FP16>(sd.hist, it - 2, nih);
          if (FP16) {
            inv_vx = pow2f(15 - amax_exponent(__reduce_max_sync(kAll, s0v)));
            inv_vz = pow2f(15 - amax_exponent(__reduce_max_sync(kAll, s1v)));
          }
        }
        if (live && kB && FP16) sc_p = pow2f(amax_exponent(__reduce_max_sync(kAll, s0v)) - 15);
        amp_smem = nsta <= kAmpMax;
        if (do_inj && amp_smem) {  // CTA-uniform
#pragma unroll
          for (int k = 0; k < kPer; ++k)
            if (tid + k * kThreadsT < nsta) amp_s[tid + k * kThreadsT] = av[k];
          __syncthreads();
        }
      } else {
        sd = L.shots[cur];
        const int nt = sd.nt;
        live = sd.active && (MODE == FM_STAGE_A ? it <= nt + 1 : it <= nt);
        flush = (MODE == FM_STAGE_A) && it == nt + 1;
        do_inj = live && !flush && ((MODE == FM_STAGE_A) || (MODE == FM_FWD && sd.type_src == 0));
        lmax = 0;
        if (live && MODE == FM_STAGE_A && it >= 2) {
          hvs = step_ptr<FP16>(sd.hist, it - 2, nih);
          if (FP16) {
            const unsigned* a = sd.amax + (size_t)(it - 2) * 3 * kAmaxSlots;
            inv_vx = pow2f(15 - amax_exponent(warp_amax_slots(a + kAmaxSlots)));
            inv_vz = pow2f(15 - amax_exponent(warp_amax_slots(a + 2 * kAmaxSlots)));
          }
        }
        if (live && kB && FP16)
          sc_p = pow2f(amax_exponent(warp_amax_slots(
                           sd.amax + (size_t)(nt - it - L.hist_step0) * 3 * kAmaxSlots)) - 15);
        amp_smem = sd.inj.nsta <= kAmpMax;
        if (do_inj && amp_smem) stage_amp(amp_s, sd.amp + (it - 1), sd.amp_stride, sd.inj.nsta);
      }
    }
    const int i1 = id.r0 + 2 * lane;
    const bool ok0 = i1 < n1e, ok1 = i1 + 1 < n1e;
    const bool u0 = ok0 && i1 >= 2 && i1 < hi1, u1 = ok1 && i1 + 1 >= 2 && i1 + 1 < hi1;
    const bool r0 = ok0 && i1 >= npml && i1 < npml + g.n1;
    const bool r1 = ok1 && i1 + 1 >= npml && i1 + 1 < npml + g.n1;
    const int h1 = i1 - hbase;
    const bool s0 = r0 && i1 - npml >= slo && i1 - npml < shi1;
    const bool s1 = r1 && i1 + 1 - npml >= slo && i1 + 1 - npml < shi1;
    const int cb = id.c0 + CPT * warp;
    // Interior tiles lie inside the physical region, where every sponge factor
    // is exactly 1 (x * 1 == x), so they load no profiles.
    const bool interior = tile_interior(g, id, MODE, slo, shi1, shi2);
    // ---- global prefetch before waiting for the tile
    float2 d1a = make_float2(0.f, 0.f), d1a1 = make_float2(0.f, 0.f);
    float d2a[CPT], d2a1[CPT];
    int clo[CPT], chi[CPT];  // forward-source band rows of the thread's columns
    // Stage A: the receiver band of column cb + lane is held by lane < CPT
    // (first row, last row, dense-row base) and shuffled out when needed.
    int bl = 0x7fffffff, bh = -1, bb = 0;
    if (live && !flush && !interior) {
      if (ok1) {
        d1a = ldg2(m.d1a + i1);
        d1a1 = ldg2(m.d1a1 + i1);
      } else if (ok0) {
        d1a.x = __ldg(m.d1a + i1);
        d1a1.x = __ldg(m.d1a1 + i1);
      }
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = cb + j;
      const bool cok = live && !flush && c < n2e;
      d2a[j] = cok && !interior ? __ldg(m.d2a + c) : 0.f;
      d2a1[j] = cok && !interior ? __ldg(m.d2a1 + c) : 0.f;
      clo[j] = (MODE != FM_STAGE_A && cok && do_inj) ? __ldg(sd.inj.col_lo + c) : 0x7fffffff;
      chi[j] = (MODE != FM_STAGE_A && cok && do_inj) ? __ldg(sd.inj.col_hi + c) : -1;
    }
    if (MODE == FM_STAGE_A && do_inj && lane < CPT && cb + lane < n2e) {
      bl = __ldg(sd.inj.col_lo + cb + lane);
      bh = __ldg(sd.inj.col_hi + cb + lane);
      bb = __ldg(sd.inj.col_base + cb + lane);
    }
    bar_wait(&bar[stage], stage ? phase1 : phase0, L.err);
    if (stage) phase1 ^= 1; else phase0 ^= 1;
    unsigned park = 0;  // stage A: bit j set when the row pair (i1, i1+1) of column j is in the band
    if (MODE == FM_STAGE_A) {
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const int lo = __shfl_sync(kAll, bl, j), hi = __shfl_sync(kAll, bh, j);
        if (i1 + 1 >= lo && i1 <= hi) park |= 1u << j;
      }
    }
    unsigned char* st = smem + stage * kStage;
    const float2* VX = reinterpret_cast<const float2*>(st);         // [TC+3][32]
    const float* VZ = reinterpret_cast<const float*>(st + kPVX);    // [TC][72]
    const float2* PX = reinterpret_cast<const float2*>(st + kPVX + kPVZ);
    const float2* PZ = PX + TR * TC / 2;
    const float2* KA = PZ + TR * TC / 2;
    // The stencil pass, compiled twice: for interior tiles (no grid edge, PML
    // row/column edge, free surface or physical-interior boundary inside the
    // tile) every boundary predicate is the constant true/false.
    auto stencil_pass = [&](auto interior_tag) {
      constexpr bool IN = decltype(interior_tag)::value;
      const bool ok0_ = IN || ok0, ok1_ = IN || ok1, u0_ = IN || u0, u1_ = IN || u1;
      const bool r0_ = IN || r0, r1_ = IN || r1, s0_ = IN || s0, s1_ = IN || s1;
      if (live && ok0_) {
        float2 q[CPT + 3];  // vx at columns cb-2 .. cb+CPT
  #pragma unroll
        for (int k = 0; k < CPT + 3; ++k) q[k] = VX[(CPT * warp + k) * 32 + lane];
  #pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int cc = CPT * warp + j;
          const int c = id.c0 + cc;
          if (!IN && c >= n2e) continue;
          const int k = i1 + ld * c;
          const float* vzc = VZ + cc * (TR + 2 * HR) + 2 * lane;  // row i1-4
          const float2 zm = *reinterpret_cast<const float2*>(vzc + 2);
          const float2 z = *reinterpret_cast<const float2*>(vzc + 4);
          const float zp2 = vzc[6];
          const int i2p = c - npml;
          const bool cint = IN || (i2p >= 0 && i2p < g.n2);
          if (MODE == FM_STAGE_A && it >= 2 && cint && (r0_ || r1_)) {
            const int ho = h1 + n1h * i2p;
            const uint64_t pol = l2_evict_first();
            H::put2(hvs, (int)nih + ho, q[j + 2].x, q[j + 2].y, inv_vx, r0_, r1_, pol);
            H::put2(hvs, 2 * (int)nih + ho, z.x, z.y, inv_vz, r0_, r1_, pol);
          }
          if (flush) continue;
          float2 px_ = PX[cc * 32 + lane], pz_ = PZ[cc * 32 + lane];
          const float2 kv = KA[cc * 32 + lane];
          if (IN || (c >= 2 && c < hi2)) {
            const bool fwd = (MODE != FM_STAGE_A);
            if (u0_) {
              const float der2 = dminus(q[j].x, q[j + 1].x, q[j + 2].x, q[j + 3].x);
              const float der1 = dminus(zm.x, zm.y, z.x, z.y);
              const float kd = fmul(dtdx, kv.x);
              const float ax = IN ? px_.x : fmul(d2a[j], px_.x);
              const float bx = IN ? fmul(kd, der2) : fmul(fmul(kd, d2a1[j]), der2);
              const float az = IN ? pz_.x : fmul(d1a.x, pz_.x);
              const float bz = IN ? fmul(kd, der1) : fmul(fmul(kd, d1a1.x), der1);
              px_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
              pz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
            }
            if (u1_) {
              const float der2 = dminus(q[j].y, q[j + 1].y, q[j + 2].y, q[j + 3].y);
              const float der1 = dminus(zm.y, z.x, z.y, zp2);
              const float kd = fmul(dtdx, kv.y);
              const float ax = IN ? px_.y : fmul(d2a[j], px_.y);
              const float bx = IN ? fmul(kd, der2) : fmul(fmul(kd, d2a1[j]), der2);
              const float az = IN ? pz_.y : fmul(d1a.y, pz_.y);
              const float bz = IN ? fmul(kd, der1) : fmul(fmul(kd, d1a1.y), der1);
              px_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
              pz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
            }
          }
          if (MODE == FM_STAGE_A && ((park >> j) & 1u)) {
            // receiver band: park the post-stencil pair in the stage buffer for
            // the band pass after this loop
            *reinterpret_cast<float2*>(sd.pz + k) = pz_;
            reinterpret_cast<float2*>(st + kPVX + kPVZ)[cc * 32 + lane] = px_;
            reinterpret_cast<float2*>(st + kPVX + kPVZ + kPF)[cc * 32 + lane] = pz_;
            continue;
          }
          if (i1 + 1 >= clo[j] && i1 <= chi[j]) {  // forward source
            const int base = __ldg(sd.inj.col_base + c) - clo[j];
            const int sg = MODE == FM_FWD ? +1 : -1;
            if (amp_smem) {
              if (i1 >= clo[j]) px_.x = inject_at(sd.inj, px_.x, base + i1, dt, kv.x, amp_s, sg);
              if (ok1_ && i1 + 1 <= chi[j])
                px_.y = inject_at(sd.inj, px_.y, base + i1 + 1, dt, kv.y, amp_s, sg);
            } else {
              if (i1 >= clo[j])
                px_.x = inject_at_global(sd.inj, px_.x, base + i1, dt, kv.x, sd.amp + (it - 1),
                                         sd.amp_stride, sg);
              if (ok1_ && i1 + 1 <= chi[j])
                px_.y = inject_at_global(sd.inj, px_.y, base + i1 + 1, dt, kv.y, sd.amp + (it - 1),
                                         sd.amp_stride, sg);
            }
          }
          if (kB && (IN || (i2p >= slo && i2p < shi2)) && (s0_ || s1_)) {
            const float2 hv = hist_box_read<FP16>(st + kPStage, cc, lane);
            if (s0_) px_.x = fadd(px_.x, fmul(fmul(mdt, hv.x * sc_p), kv.x));
            if (s1_) px_.y = fadd(px_.y, fmul(fmul(mdt, hv.y * sc_p), kv.y));
          }
          float2 pv;
          pv.x = (!IN && i1 < fsrows) ? 0.f : fadd(px_.x, pz_.x);
          pv.y = (!IN && i1 + 1 < fsrows) ? 0.f : fadd(px_.y, pz_.y);
          *reinterpret_cast<float2*>(sd.px + k) = px_;
          *reinterpret_cast<float2*>(sd.pz + k) = pz_;
          *reinterpret_cast<float2*>(sd.p + k) = pv;
          if (cint) {
            if (MODE == FM_STAGE_A) {
              if (r0_) lmax = max(lmax, abs_bits(pv.x));
              if (r1_) lmax = max(lmax, abs_bits(pv.y));
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
      }
    };
    if (interior)
      stencil_pass(std::true_type{});
    else
      stencil_pass(std::false_type{});
    if (MODE == FM_STAGE_A) {
      // Receiver band of this tile: each warp finishes the parked rows of its
      // own columns, one lane per row.  The row pointers of all its columns
      // are loaded first, then each point's entries as one batch; the sum
      // keeps the station order.
      const int rlast = min(id.r0 + TR, n1e) - 1;
      // A warp only reads row pairs parked by its own lanes (its own
      // columns), so a warp vote and a warp barrier order the pass.
      const bool wb = lane < CPT && bl <= rlast && bh >= id.r0;
      if (__any_sync(kAll, wb)) {  // warp-uniform
        __syncwarp();
        const float* PXf = reinterpret_cast<const float*>(st + kPVX + kPVZ);
        const float* PZf = PXf + TR * TC;
        const float* KAf = PZf + TR * TC;
        const int2* rp2 = reinterpret_cast<const int2*>(sd.inj.rowptr);
        // rows to finish per column: the band's row pairs inside the tile
        int rows = 0;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int blo = __shfl_sync(kAll, bl, j), bhi = __shfl_sync(kAll, bh, j);
          const int lo = max(blo & ~1, id.r0), hi = min(bhi | 1, rlast);
          if (blo <= rlast && bhi >= id.r0) rows = max(rows, hi - lo + 1);
        }
        for (int pass = 0; pass < rows; pass += 32) {
          int rr[CPT], e0[CPT], e1[CPT];
          bool on[CPT];
#pragma unroll
          for (int j = 0; j < CPT; ++j) {
            const int blo = __shfl_sync(kAll, bl, j), bhi = __shfl_sync(kAll, bh, j);
            const int bbase = __shfl_sync(kAll, bb, j);
            const int lo = max(blo & ~1, id.r0), hi = min(bhi | 1, rlast);
            rr[j] = lo + pass + lane;
            on[j] = blo <= rlast && bhi >= id.r0 && rr[j] <= hi;
            e0[j] = e1[j] = 0;
            if (on[j] && rr[j] >= blo && rr[j] <= bhi) {
              const int2 q = ld_hint_i2(rp2 + bbase + (rr[j] - blo), l2_evict_last());
              e0[j] = q.x;
              e1[j] = q.y;
            }
          }
          // Column pairs: the first kBatch entries of the pair's points are
          // loaded as one batch, their amplitudes looked up once (the source
          // is CTA-uniform; unused slots hold station 0, a valid index), then
          // the two chains run interleaved, each in station order.
          const uint64_t pol = l2_evict_last();
          const float* amp_g = sd.amp + (it - 1);
#pragma unroll
          for (int h = 0; h < CPT; h += 2) {
            float2 q[2][kBatch];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
              for (int k = 0; k < kBatch; ++k)
                q[u][k] = e0[h + u] + k < e1[h + u] ? ld_hint_f2(sd.inj.ent + e0[h + u] + k, pol)
                                                    : make_float2(0.f, 0.f);
            if (amp_smem) {
#pragma unroll
              for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int k = 0; k < kBatch; ++k) q[u][k].y = amp_s[__float_as_int(q[u][k].y)];
            } else {
#pragma unroll
              for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int k = 0; k < kBatch; ++k)
                  q[u][k].y = __ldg(amp_g + (size_t)__float_as_int(q[u][k].y) * sd.amp_stride);
            }
            float v[2], kv[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int o = (CPT * warp + h + u) * TR + (rr[h + u] - id.r0);
              v[u] = on[h + u] ? PXf[o] : 0.f;
              kv[u] = on[h + u] ? KAf[o] : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k)
#pragma unroll
              for (int u = 0; u < 2; ++u) {
                const float t = fmul(fmul(fmul(q[u][k].x, dt), q[u][k].y), kv[u]);
                v[u] = e0[h + u] + k < e1[h + u] ? fsub(v[u], t) : v[u];
              }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int j = h + u;
              for (int e = e0[j] + kBatch; e < e1[j]; ++e) {  // more stations than kBatch
                const float2 q1 = ld_hint_f2(sd.inj.ent + e, pol);
                const int st1 = __float_as_int(q1.y);
                const float a1 = amp_smem ? amp_s[st1] : __ldg(amp_g + (size_t)st1 * sd.amp_stride);
                v[u] = fsub(v[u], fmul(fmul(fmul(q1.x, dt), a1), kv[u]));
              }
              if (!on[j]) continue;
              const int c = cb + j, r = rr[j];
              const int o = (CPT * warp + j) * TR + (r - id.r0);
              const float pvv = r < fsrows ? 0.f : fadd(v[u], PZf[o]);
              const size_t k = (size_t)r + (size_t)ld * c;
              sd.px[k] = v[u];
              sd.p[k] = pvv;
              if (r >= npml && r < npml + g.n1 && c >= npml && c < npml + g.n2)
                lmax = max(lmax, abs_bits(pvv));
            }
          }
        }
      }
    }
    __syncthreads();  // stage buffer (and staged amplitudes) free for reuse
    stage ^= 1;
  }
  if (MODE == FM_STAGE_A && cur >= 0 && live && !flush)
    warp_amax_flush(lmax, sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots +
                              ((blockIdx.x * 8 + warp) % kAmaxSlots), L.err);
}

// ---------------------------------------------------------------------------
// Velocity kernel.  The receiver / datum gathers (8 stations per unit) run
// after the stencil tiles, on the CTAs that drew one tile fewer.
// ---------------------------------------------------------------------------
// 3 CTAs per SM in the forward and stage-A modes (80 registers); the stage-B
// modes keep 2 (their heavier body and tile count balance better at 2).
// RHO: a density other than 1 -- the update coefficients and the buoyancy
// weight of the velocity sources come from the 2-D fields m.rbw1, m.rbw2 and
// m.rbue (one float2 load per column and point pair) instead of the 1-D
// sponge profiles and the constant 1.
template <int MODE, bool FP16, bool RHO>
__global__ void __launch_bounds__(kThreadsT,
                                  (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES) ? 2 : 3)
    k_tma_v(const Grid g, const ModelDev m, const FusedLaunch L, const int it, const int ntiles,
            const int ngb_per_shot) {
  constexpr bool kB = (MODE == FM_STAGE_B || MODE == FM_STAGE_B_ES);
  constexpr int kStage = v_stage(MODE, FP16);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * kStage);
  float* prod = reinterpret_cast<float*>(smem);  // gathers run after the tiles
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    bar_init(&bar[0]);
    bar_init(&bar[1]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  pdl_trigger();
  __syncthreads();
  pdl_wait();  // the previous step's fields, scales and outputs are complete
  const int hbase = g.hist_base();
  auto issue = [&](int t, int s) {
    const TileId id = tile_id(g, t, L);
    const TmaMaps* mp = L.maps + id.shot;
    unsigned char* st = smem + s * kStage;
    bar_expect(&bar[s], kVPb + 2 * kPF + (kB ? 2 * hist_box(FP16) : 0));  // bytes copied
    tma_2d(st, &mp->p72, id.r0 - HR, id.c0 - 1, &bar[s]);
    tma_2d(st + kVP, &mp->vx16, id.r0, id.c0, &bar[s]);
    tma_2d(st + kVP + kPF, &mp->vz16, id.r0, id.c0, &bar[s]);
    if (kB) {  // velocity histories of the time-reversed step
      // record length from the kernel parameters (no load on the issuing thread's path)
      const int ic = (id.shot < L.nparam ? L.shot_nt[id.shot] : L.shots[id.shot].nt) - it + 1;
      const uint64_t pol = l2_evict_first();
      const int hs = ic - 1 - L.hist_step0;  // history slot of step ic
      tma_3d(st + kVStage, &mp->hist, id.r0 - hbase, id.c0 - g.npml, hs * 3 + 1, &bar[s], pol);
      tma_3d(st + kVStage + hist_box(FP16), &mp->hist, id.r0 - hbase, id.c0 - g.npml, hs * 3 + 2,
             &bar[s], pol);
    }
  };
  const Walk wk = tile_walk(ntiles, L.nlive);
  int t = wk.t0;
  if (tid == 0 && t < wk.end) issue(t, 0);
  uint32_t phase0 = 0, phase1 = 0;
  int stage = 0;
  const int ld = g.ld, n1e = g.n1e, n2e = g.n2e, npml = g.npml;
  const int off = (MODE == FM_FWD) ? 2 : 3;
  const int hi1 = n1e - off, hi2 = n2e - off;
  const int n1h = L.n1h;
  const size_t nih = (size_t)n1h * g.n2;
  const float dt = g.dt, mdt = fmul(-1.0f, dt);
  const float dtdx_v = fmul(g.dtdx, 1.0f);  // bw1 = bw2 in the physical interior
  const bool fs = g.ofs == 1;
  int cur = -1;
  ShotDevice sd;
  bool live = false, do_inj = false;
  float inv_p = 1.f, sc_vx = 1.f, sc_vz = 1.f;
  void* hps = nullptr;
  unsigned lmx = 0, lmz = 0;
  for (; t < wk.end; t += wk.stride) {
    const int tn = t + wk.stride;
    if (tid == 0 && tn < wk.end) issue(tn, stage ^ 1);
    const TileId id = tile_id(g, t, L);
    if (id.shot != cur) {
      if (MODE == FM_STAGE_A && cur >= 0 && live) {
        unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + ((blockIdx.x * 8 + warp) % kAmaxSlots);
        warp_amax_flush(lmx, a + kAmaxSlots, L.err);
        warp_amax_flush(lmz, a + 2 * kAmaxSlots, L.err);
      }
      cur = id.shot;
      // scale slots loaded together with the descriptor when the shot's
      // pointers are kernel parameters
      unsigned s0v = 0, s1v = 0;
      const bool fast = cur < L.nparam;
      if (fast && FP16) {
        const int ntc = L.shot_nt[cur];
        const unsigned* am = L.shot_amax[cur];
        if (MODE == FM_STAGE_A && it <= ntc) s0v = am[(size_t)(it - 1) * 3 * kAmaxSlots + lane];
        if (kB && it <= ntc) {
          s0v = am[(size_t)(ntc - it - L.hist_step0) * 3 * kAmaxSlots + kAmaxSlots + lane];
          s1v = am[(size_t)(ntc - it - L.hist_step0) * 3 * kAmaxSlots + 2 * kAmaxSlots + lane];
        }
      }
      sd = L.shots[cur];
      live = sd.active && it <= sd.nt;
      do_inj = live && (MODE == FM_FWD) && sd.type_src == 1;
      lmx = lmz = 0;
      if (live && MODE == FM_STAGE_A) {
        hps = step_ptr<FP16>(sd.hist, it - 1, nih);
        if (FP16)
          inv_p = pow2f(15 - amax_exponent(
                                 fast ? __reduce_max_sync(kAll, s0v)
                                      : warp_amax_slots(sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots)));
      }
      if (live && kB && FP16) {
        const unsigned* a = sd.amax + (size_t)(sd.nt - it - L.hist_step0) * 3 * kAmaxSlots;
        sc_vx = pow2f(amax_exponent(fast ? __reduce_max_sync(kAll, s0v)
                                         : warp_amax_slots(a + kAmaxSlots)) - 15);
        sc_vz = pow2f(amax_exponent(fast ? __reduce_max_sync(kAll, s1v)
                                         : warp_amax_slots(a + 2 * kAmaxSlots)) - 15);
      }
    }
    const int i1 = id.r0 + 2 * lane;
    const bool ok0 = i1 < n1e, ok1 = i1 + 1 < n1e;
    const bool u0 = ok0 && i1 >= 2 && i1 < hi1, u1 = ok1 && i1 + 1 >= 2 && i1 + 1 < hi1;
    const bool r0 = ok0 && i1 >= npml && i1 < npml + g.n1;
    const bool r1 = ok1 && i1 + 1 >= npml && i1 + 1 < npml + g.n1;
    const int h1 = i1 - hbase;
    const int cb = id.c0 + CPT * warp;
    // interior tiles: sponge factors exactly 1, bw1 = bw2 = dtdx
    const bool interior = tile_interior(g, id, MODE, 0, g.n1, g.n2);
    float2 d1b = make_float2(0.f, 0.f), bw1 = make_float2(0.f, 0.f);
    if (live && !interior) {
      if (ok1) {
        d1b = ldg2(m.d1b + i1);
        if (!RHO) bw1 = ldg2(m.bw1 + i1);
      } else if (ok0) {
        d1b.x = __ldg(m.d1b + i1);
        if (!RHO) bw1.x = __ldg(m.bw1 + i1);
      }
    }
    float d2b[CPT], bw2[CPT];
    int clo[CPT], chi[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
      const int c = cb + j;
      const bool cok = live && c < n2e;
      d2b[j] = cok && !interior ? __ldg(m.d2b + c) : 0.f;
      bw2[j] = cok && !interior && !RHO ? __ldg(m.bw2 + c) : 0.f;
      clo[j] = (cok && do_inj) ? __ldg(sd.inj.col_lo + c) : 0x7fffffff;
      chi[j] = (cok && do_inj) ? __ldg(sd.inj.col_hi + c) : -1;
    }
    bar_wait(&bar[stage], stage ? phase1 : phase0, L.err);
    if (stage) phase1 ^= 1; else phase0 ^= 1;
    const unsigned char* st = smem + stage * kStage;
    const float* P = reinterpret_cast<const float*>(st);  // [TC+3][72]: row 0 = r0-4, col 0 = c0-1
    const float2* P2 = reinterpret_cast<const float2*>(st);
    const float2* VX = reinterpret_cast<const float2*>(st + kVP);
    const float2* VZ = VX + TR * TC / 2;
    // The stencil pass, compiled twice (interior tiles: every boundary
    // predicate constant, as in the pressure kernel).
    auto stencil_pass = [&](auto interior_tag) {
      constexpr bool IN = decltype(interior_tag)::value;
      const bool ok0_ = IN || ok0, ok1_ = IN || ok1, u0_ = IN || u0, u1_ = IN || u1;
      const bool r0_ = IN || r0, r1_ = IN || r1;
      if (live && ok0_) {
        float2 a[CPT + 3];  // p rows (i1, i1+1) at columns cb-1 .. cb+CPT+1
  #pragma unroll
        for (int k = 0; k < CPT + 3; ++k) a[k] = P2[(CPT * warp + k) * ((TR + 2 * HR) / 2) + 2 + lane];
        const bool dst_x = !IN && fs && i1 == npml - 1;
        const bool skip_y = !IN && fs && i1 + 1 == npml - 1;
        const bool src_x = !IN && fs && i1 == npml;
  #pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const int cc = CPT * warp + j;
          const int c = id.c0 + cc;
          if (!IN && c >= n2e) continue;
          const int k = i1 + ld * c;
          const float* pcol = P + (cc + 1) * (TR + 2 * HR) + 2 * lane;  // own column, row i1-4
          const float pm1 = pcol[3];
          const float2 pc = a[j + 1];
          const float2 pp = *reinterpret_cast<const float2*>(pcol + 6);
          const int i2p = c - npml;
          const bool cint = IN || (i2p >= 0 && i2p < g.n2);
          float2 vx_ = VX[cc * 32 + lane], vz_ = VZ[cc * 32 + lane];
          if (IN || (c >= 2 && c < hi2)) {
            const bool fwd = (MODE != FM_STAGE_A);
            // k + 1 stays inside the padded column (i1 even, ld a multiple of 64)
            const float2 rb2 = RHO ? ldg2(m.rbw2 + k) : make_float2(0.f, 0.f);
            const float2 rb1 = RHO ? ldg2(m.rbw1 + k) : make_float2(0.f, 0.f);
            if (u0_) {
              const float der2 = dplus(a[j].x, pc.x, a[j + 2].x, a[j + 3].x);
              const float der1 = dplus(pm1, pc.x, pc.y, pp.x);
              const float ax = IN ? vx_.x : fmul(d2b[j], vx_.x);
              const float bx = fmul(RHO ? rb2.x : IN ? dtdx_v : bw2[j], der2);
              const float az = IN ? vz_.x : fmul(d1b.x, vz_.x);
              const float bz = fmul(RHO ? rb1.x : IN ? dtdx_v : bw1.x, der1);
              vx_.x = fwd ? fadd(ax, bx) : fsub(ax, bx);
              vz_.x = fwd ? fadd(az, bz) : fsub(az, bz);
            }
            if (u1_) {
              const float der2 = dplus(a[j].y, pc.y, a[j + 2].y, a[j + 3].y);
              const float der1 = dplus(pc.x, pc.y, pp.x, pp.y);
              const float ax = IN ? vx_.y : fmul(d2b[j], vx_.y);
              const float bx = fmul(RHO ? rb2.y : IN ? dtdx_v : bw2[j], der2);
              const float az = IN ? vz_.y : fmul(d1b.y, vz_.y);
              const float bz = fmul(RHO ? rb1.y : IN ? dtdx_v : bw1.y, der1);
              vx_.y = fwd ? fadd(ax, bx) : fsub(ax, bx);
              vz_.y = fwd ? fadd(az, bz) : fsub(az, bz);
            }
          }
          if (kB && cint && (r0_ || r1_)) {
            const float2 hx = hist_box_read<FP16>(st + kVStage, cc, lane);
            const float2 hz = hist_box_read<FP16>(st + kVStage + hist_box(FP16), cc, lane);
            const float2 bu = RHO ? ldg2(m.rbue + k) : make_float2(1.0f, 1.0f);
            if (r0_) {
              vx_.x = fadd(vx_.x, fmul(fmul(mdt, hx.x * sc_vx), bu.x));
              vz_.x = fadd(vz_.x, fmul(fmul(mdt, hz.x * sc_vz), bu.x));
            }
            if (r1_) {
              vx_.y = fadd(vx_.y, fmul(fmul(mdt, hx.y * sc_vx), bu.y));
              vz_.y = fadd(vz_.y, fmul(fmul(mdt, hz.y * sc_vz), bu.y));
            }
          }
          if (i1 + 1 >= clo[j] && i1 <= chi[j]) {  // vz source (type_src = 1)
            const int base = __ldg(sd.inj.col_base + c) - clo[j];
            const float2 bu = RHO ? ldg2(m.rbue + k) : make_float2(1.0f, 1.0f);
            if (i1 >= clo[j])
              vz_.x = inject_at_global(sd.inj, vz_.x, base + i1, dt, bu.x, sd.amp + (it - 1),
                                       sd.amp_stride, +1);
            if (ok1_ && i1 + 1 <= chi[j])
              vz_.y = inject_at_global(sd.inj, vz_.y, base + i1 + 1, dt, bu.y, sd.amp + (it - 1),
                                       sd.amp_stride, +1);
          }
          if (dst_x) vz_.x = vz_.y;
          *reinterpret_cast<float2*>(sd.vx + k) = vx_;
          if (skip_y)
            sd.vz[k] = vz_.x;
          else
            *reinterpret_cast<float2*>(sd.vz + k) = vz_;
          if (src_x) sd.vz[k - 1] = vz_.x;
          if (MODE == FM_STAGE_A && cint && (r0_ || r1_)) {
            Hist<FP16>::put2(hps, h1 + n1h * i2p, pc.x, pc.y, inv_p, r0_, r1_, l2_evict_first());
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
      }
    };
    if (interior)
      stencil_pass(std::true_type{});
    else
      stencil_pass(std::false_type{});
    __syncthreads();
    stage ^= 1;
  }
  if (MODE == FM_STAGE_A && cur >= 0 && live) {
    unsigned* a = sd.amax + (size_t)(it - 1) * 3 * kAmaxSlots + ((blockIdx.x * 8 + warp) % kAmaxSlots);
    warp_amax_flush(lmx, a + kAmaxSlots, L.err);
    warp_amax_flush(lmz, a + 2 * kAmaxSlots, L.err);
  }
  // receiver / datum gathers (the pressure field is not modified here)
  if (MODE != FM_STAGE_A) {
    const int ngb = ngb_per_shot * L.nlive;
    for (int gb = gridDim.x - 1 - blockIdx.x; gb < ngb; gb += gridDim.x) {
      const int shot = L.live[gb / ngb_per_shot];
      const ShotDevice& so = L.shots[shot];
      if (!so.active || it > so.nt || so.type_rec != 0) continue;
      const int s = (gb % ngb_per_shot) * 8 + warp;
      if (s < so.rec.n) {
        if (so.out) {
          const float v = warp_gather_ordered(prod + warp * 444, so.rec.ix1, so.rec.ix2,
                                              so.rec.tile, s, so.p, g.ld, 0, g.n1e, g.n2e);
          const int row = so.out_reverse ? so.nt - it : it - 1;
          if (lane == 0) so.out[row + (size_t)so.nt * s] = v;
        }
      } else if (s - so.rec.n < so.datum.n && so.red &&
                 (MODE == FM_FWD || MODE == FM_STAGE_B_ES)) {
        const int d = s - so.rec.n;
        const float v = warp_gather_ordered(prod + warp * 444, so.datum.ix1, so.datum.ix2,
                                            so.datum.tile, d,
                                            so.p + g.npml + (size_t)g.ld * g.npml, g.ld,
                                            g.npml, g.n1, g.n2);
        if (lane == 0) so.red[(it - 1) + (size_t)so.nt * d] = v;
      }
    }
  }
}

template <int MODE>
void launch_p(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, cudaStream_t st) {
  const int ntiles = tma_tiles(g) * L.nlive;
  const int grid = std::min(ntiles, L.persist_p);
  if (L.hist_fp16)
    launch_pdl(k_tma_p<MODE, true>, grid, kThreadsT, p_smem(MODE, true), st, L.pdl != 0, g, m, L,
               it, ntiles);
  else
    launch_pdl(k_tma_p<MODE, false>, grid, kThreadsT, p_smem(MODE, false), st, L.pdl != 0, g, m,
               L, it, ntiles);
}

template <int MODE>
void launch_v(const Grid& g, const ModelDev& m, const FusedLaunch& L, int it, cudaStream_t st) {
  const int ntiles = tma_tiles(g) * L.nlive;
  const int stations = (MODE == FM_STAGE_A) ? 0 : L.max_rec + L.max_datum;
  const int ngbps = (stations + 7) / 8;
  const int grid = std::max(1, std::min(std::max(ntiles, ngbps * L.nlive), L.persist_v));
  const bool fp16 = L.hist_fp16 != 0, rho = m.rbw1 != nullptr;
  const size_t smem = v_smem(MODE, fp16);
  const bool pdl = L.pdl != 0;
  if (fp16 && !rho)
    launch_pdl(k_tma_v<MODE, true, false>, grid, kThreadsT, smem, st, pdl, g, m, L, it, ntiles,
               ngbps);
  else if (!rho)
    launch_pdl(k_tma_v<MODE, false, false>, grid, kThreadsT, smem, st, pdl, g, m, L, it, ntiles,
               ngbps);
  else if (fp16)
    launch_pdl(k_tma_v<MODE, true, true>, grid, kThreadsT, smem, st, pdl, g, m, L, it, ntiles,
               ngbps);
  else
    launch_pdl(k_tma_v<MODE, false, true>, grid, kThreadsT, smem, st, pdl, g, m, L, it, ntiles,
               ngbps);
}

template <typename K>
int occupancy(K kernel, size_t smem) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreadsT, smem);
  return n;
}

template <int MODE, bool FP16>
void prep_mode(int* pp, int* pv, int* pv_mode) {
  *pp = std::min(*pp, occupancy(k_tma_p<MODE, FP16>, p_smem(MODE, FP16)));
  const int ov = std::min(occupancy(k_tma_v<MODE, FP16, false>, v_smem(MODE, FP16)),
                          occupancy(k_tma_v<MODE, FP16, true>, v_smem(MODE, FP16)));
  *pv = std::min(*pv, ov);
  pv_mode[MODE * 2 + (FP16 ? 1 : 0)] = ov;
}

// Self-test of the failure path of the bounded waits: thread 0 waits on an
// mbarrier that no copy and no thread will complete, with a short budget; the
// wait gives up, raises kErrTimeout and returns (no copy is in flight).
__global__ void k_wait_selftest(unsigned* err, long long budget) {
  __shared__ __align__(8) uint64_t b;
  if (threadIdx.x == 0) {
    bar_init(&b);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) bar_wait(&b, 0, err, budget);
}

}  // namespace

void tma_wait_selftest(unsigned* err, long long budget, cudaStream_t st) {
  k_wait_selftest<<<1, 32, 0, st>>>(err, budget);
}

int tma_tiles(const Grid& g) { return ((g.n1e + TR - 1) / TR) * ((g.n2e + TC - 1) / TC); }

// Persistent grid sizes (CTAs resident on all SMs) and the dynamic shared
// memory opt-in of every instantiation; call once per device, outside graph
// capture.
void tma_prepare(int* persist_p, int* persist_v, int* persist_v_mode) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int op = 64, ov = 64;
  int pvm[8] = {};
  prep_mode<FM_FWD, true>(&op, &ov, pvm);
  prep_mode<FM_FWD, false>(&op, &ov, pvm);
  prep_mode<FM_STAGE_A, true>(&op, &ov, pvm);
  prep_mode<FM_STAGE_A, false>(&op, &ov, pvm);
  prep_mode<FM_STAGE_B, true>(&op, &ov, pvm);
  prep_mode<FM_STAGE_B, false>(&op, &ov, pvm);
  prep_mode<FM_STAGE_B_ES, true>(&op, &ov, pvm);
  prep_mode<FM_STAGE_B_ES, false>(&op, &ov, pvm);
  *persist_p = std::max(1, op) * sms;
  *persist_v = std::max(1, ov) * sms;
  for (int i = 0; i < 8; ++i) persist_v_mode[i] = std::max(1, pvm[i]) * sms;
}

void tma_p_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                cudaStream_t st) {
  switch (mode) {
    case FM_FWD: launch_p<FM_FWD>(g, m, L, it, st); break;
    case FM_STAGE_A: launch_p<FM_STAGE_A>(g, m, L, it, st); break;
    case FM_STAGE_B: launch_p<FM_STAGE_B>(g, m, L, it, st); break;
    default: launch_p<FM_STAGE_B_ES>(g, m, L, it, st); break;
  }
}

void tma_v_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                cudaStream_t st) {
  switch (mode) {
    case FM_FWD: launch_v<FM_FWD>(g, m, L, it, st); break;
    case FM_STAGE_A: launch_v<FM_STAGE_A>(g, m, L, it, st); break;
    case FM_STAGE_B: launch_v<FM_STAGE_B>(g, m, L, it, st); break;
    default: launch_v<FM_STAGE_B_ES>(g, m, L, it, st); break;
  }
}

// Host: the tensor maps of one shot -- 2-D maps of the extended-grid fields
// (innermost dimension n1e rows with stride ld, n2e columns) and the 3-D map
// of its history [3*nsteps][n2][n1h] (FP16 or FP32).
bool tma_encode_maps(const Grid& g, const float* vx, const float* vz, const float* px,
                     const float* pz, const float* p, const float* kap, const void* hist,
                     int hist_fp16, int n1h, int nsteps, TmaMaps* out) {
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
  auto make = [&](CUtensorMap* map, const float* base, int br, int bc) {
    cuuint64_t dims[2] = {(cuuint64_t)g.n1e, (cuuint64_t)g.n2e};
    cuuint64_t strides[1] = {(cuuint64_t)g.ld * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)br, (cuuint32_t)bc};
    cuuint32_t es[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims,
                  strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
  };
  const size_t esz = hist_fp16 ? 2 : 4;
  cuuint64_t hd[3] = {(cuuint64_t)n1h, (cuuint64_t)g.n2, (cuuint64_t)3 * nsteps};
  cuuint64_t hs[2] = {(cuuint64_t)n1h * esz, (cuuint64_t)n1h * g.n2 * esz};
  cuuint32_t hb[3] = {(cuuint32_t)TR, (cuuint32_t)TC, 1};
  cuuint32_t he[3] = {1, 1, 1};
  const bool ok_hist =
      encode(&out->hist, hist_fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
             3, const_cast<void*>(hist), hd, hs, hb, he, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  return ok_hist && make(&out->vx19, vx, TR, TC + 3) && make(&out->vz72, vz, TR + 2 * HR, TC) &&
         make(&out->px, px, TR, TC) && make(&out->pz, pz, TR, TC) &&
         make(&out->p72, p, TR + 2 * HR, TC + 3) && make(&out->vx16, vx, TR, TC) &&
         make(&out->vz16, vz, TR, TC) && make(&out->kap, kap, TR, TC);
}

}  // namespace daw
