// The plain FP32 GPU port: one kernel per loop nest of the reference's time
// step (src/submodeling2.f90), FP32 throughout.  It is the baseline the
// fused path (stencil_fused.cu) is measured against, and the path whose
// results are compared bit for bit with the FP32 oracle.
#include "kernels.cuh"

namespace daw {
namespace {

constexpr int kBX = 32, kBY = 8;

// Pressure update over reference indices [3, n-off] (:148-155 forward,
// :1014-1021 stage A with SIGN = -1, :1108-1115 stage B).
template <int SIGN>
__global__ void __launch_bounds__(256) k_p_update(float* __restrict__ px, float* __restrict__ pz,
                                                  const float* __restrict__ vx,
                                                  const float* __restrict__ vz,
                                                  const float* __restrict__ kap, ModelDev m,
                                                  float dtdx, int ld, int hi1, int hi2) {
  const int i1 = 2 + blockIdx.x * kBX + threadIdx.x;
  const int i2 = 2 + blockIdx.y * kBY + threadIdx.y;
  if (i1 >= hi1 || i2 >= hi2) return;
  const size_t k = i1 + (size_t)ld * i2;
  const float der2 = dminus(vx[k - 2 * ld], vx[k - ld], vx[k], vx[k + ld]);
  const float der1 = dminus(vz[k - 2], vz[k - 1], vz[k], vz[k + 1]);
  const float kd = fmul(dtdx, kap[k]);
  const float kw2 = fmul(kd, m.d2a1[i2]);
  const float kw1 = fmul(kd, m.d1a1[i1]);
  const float ax = fmul(m.d2a[i2], px[k]), bx = fmul(kw2, der2);
  const float az = fmul(m.d1a[i1], pz[k]), bz = fmul(kw1, der1);
  px[k] = SIGN > 0 ? fadd(ax, bx) : fsub(ax, bx);
  pz[k] = SIGN > 0 ? fadd(az, bz) : fsub(az, bz);
}

// Particle-velocity update (:229-236, :1067-1074, :1165-1172).
template <int SIGN>
__global__ void __launch_bounds__(256) k_v_update(float* __restrict__ vx, float* __restrict__ vz,
                                                  const float* __restrict__ p, ModelDev m,
                                                  int ld, int hi1, int hi2) {
  const int i1 = 2 + blockIdx.x * kBX + threadIdx.x;
  const int i2 = 2 + blockIdx.y * kBY + threadIdx.y;
  if (i1 >= hi1 || i2 >= hi2) return;
  const size_t k = i1 + (size_t)ld * i2;
  const float der2 = dplus(p[k - ld], p[k], p[k + ld], p[k + 2 * ld]);
  const float der1 = dplus(p[k - 1], p[k], p[k + 1], p[k + 2]);
  // coefficients: 1-D profiles for rho = 1, the 2-D buoyancy fields otherwise
  const float bw2 = m.rbw2 ? m.rbw2[k] : m.bw2[i2], bw1 = m.rbw1 ? m.rbw1[k] : m.bw1[i1];
  const float ax = fmul(m.d2b[i2], vx[k]), bx = fmul(bw2, der2);
  const float az = fmul(m.d1b[i1], vz[k]), bz = fmul(bw1, der1);
  vx[k] = SIGN > 0 ? fadd(ax, bx) : fsub(ax, bx);
  vz[k] = SIGN > 0 ? fadd(az, bz) : fsub(az, bz);
}

// Hicks scatter in gather form (:172-177, :1039-1044): each touched point
// adds its contributions in station order, the reference's per-point order.
__global__ void k_inject(InjMapDev map, float* __restrict__ fld, const float* __restrict__ w,
                         float dt, const float* __restrict__ amp, int amp_stride, int sign) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= map.npts) return;
  const int k = map.pt[t];
  float v = fld[k];
  const float wk = w ? w[k] : 1.0f;
  for (int e = map.ptr[t]; e < map.ptr[t + 1]; ++e) {
    const float term = fmul(fmul(fmul(map.coef[e], dt), amp[(size_t)map.sta[e] * amp_stride]), wk);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  fld[k] = v;
}

// p = px + pz everywhere; the free surface zeroes rows 1..npml+1 (:183-189).
__global__ void k_psum(float* __restrict__ p, const float* __restrict__ px,
                       const float* __restrict__ pz, int n1e, int n2e, int ld, int fsrows) {
  const int i1 = blockIdx.x * kBX + threadIdx.x;
  const int i2 = blockIdx.y * kBY + threadIdx.y;
  if (i1 >= n1e || i2 >= n2e) return;
  const size_t k = i1 + (size_t)ld * i2;
  p[k] = i1 < fsrows ? 0.0f : fadd(px[k], pz[k]);
}

__global__ void k_store(float* __restrict__ dst, const float* __restrict__ src, int n1, int n2,
                        int npml, int ld, int acc) {
  const int i1 = blockIdx.x * kBX + threadIdx.x;
  const int i2 = blockIdx.y * kBY + threadIdx.y;
  if (i1 >= n1 || i2 >= n2) return;
  const float v = src[(i1 + npml) + (size_t)ld * (i2 + npml)];
  const size_t j = i1 + (size_t)n1 * i2;
  dst[j] = acc ? fadd(dst[j], v) : v;
}

// Stage-B pressure extended source px += ((-1*dt)*sp)*kappa over the interior
// (:1121-1125), or interior indices 2..n-1 for the final esource (:777-781).
__global__ void k_psrc(float* __restrict__ px, const float* __restrict__ sp,
                       const float* __restrict__ kap, float dt, int n1, int n2, int npml, int ld,
                       int lo, int hi1, int hi2) {
  const int i1 = lo + blockIdx.x * kBX + threadIdx.x;
  const int i2 = lo + blockIdx.y * kBY + threadIdx.y;
  if (i1 >= hi1 || i2 >= hi2) return;
  const size_t k = (i1 + npml) + (size_t)ld * (i2 + npml);
  px[k] = fadd(px[k], fmul(fmul(fmul(-1.0f, dt), sp[i1 + (size_t)n1 * i2]), kap[k]));
}

// Stage-B velocity extended sources (:1175-1186), buoyancy 1.
__global__ void k_vsrc(float* __restrict__ vx, float* __restrict__ vz,
                       const float* __restrict__ svx, const float* __restrict__ svz,
                       const float* __restrict__ bue, float dt, int n1, int n2, int npml,
                       int ld) {
  const int i1 = blockIdx.x * kBX + threadIdx.x;
  const int i2 = blockIdx.y * kBY + threadIdx.y;
  if (i1 >= n1 || i2 >= n2) return;
  const size_t k = (i1 + npml) + (size_t)ld * (i2 + npml);
  const size_t j = i1 + (size_t)n1 * i2;
  const float mdt = fmul(-1.0f, dt);
  const float b = bue ? bue[k] : 1.0f;
  vx[k] = fadd(vx[k], fmul(fmul(mdt, svx[j]), b));
  vz[k] = fadd(vz[k], fmul(fmul(mdt, svz[j]), b));
}

// vz(npml,:) = vz(npml+1,:) (:260-264).
__global__ void k_vz_fs(float* __restrict__ vz, int npml, int n2e, int ld) {
  const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i2 >= n2e) return;
  vz[(npml - 1) + (size_t)ld * i2] = vz[npml + (size_t)ld * i2];
}

// One warp per station: lanes form the 441 products c*f in parallel, lane 0
// adds them in the reference's order (i1 outer, i2 inner), so the sum rounds
// exactly as src/submodeling2.f90:214-219 does.
constexpr int kGatherWarps = 8;
__global__ void __launch_bounds__(kGatherWarps * 32)
    k_gather(StationsDev st, const float* __restrict__ origin, int ld, int shift, int hi1,
             int hi2, float* __restrict__ out, int out_stride, int row, size_t field_stride) {
  __shared__ __align__(16) float prod[kGatherWarps][444];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int s = blockIdx.x * kGatherWarps + wib;
  const int t_row = blockIdx.y;  // history index when batching rows
  if (s >= st.n) return;
  const float* f = origin + field_stride * t_row;
  const float acc = warp_gather_ordered(prod[wib], st.ix1, st.ix2, st.tile, s, f, ld, shift,
                                        hi1, hi2);
  if (lane == 0) out[(row + t_row) + (size_t)out_stride * s] = acc;
}

dim3 grid2(int n1, int n2) { return dim3((n1 + kBX - 1) / kBX, (n2 + kBY - 1) / kBY); }

}  // namespace

void plain_p_update(const Grid& g, const ModelDev& m, PlainFields f, int off, int sign,
                    cudaStream_t st) {
  const int hi1 = g.n1e - off, hi2 = g.n2e - off;
  if (hi1 <= 2 || hi2 <= 2) return;
  dim3 grid = grid2(hi1 - 2, hi2 - 2), block(kBX, kBY);
  if (sign > 0)
    k_p_update<1><<<grid, block, 0, st>>>(f.px, f.pz, f.vx, f.vz, m.kap, m, g.dtdx, g.ld, hi1, hi2);
  else
    k_p_update<-1><<<grid, block, 0, st>>>(f.px, f.pz, f.vx, f.vz, m.kap, m, g.dtdx, g.ld, hi1, hi2);
}

void plain_v_update(const Grid& g, const ModelDev& m, PlainFields f, int off, int sign,
                    cudaStream_t st) {
  const int hi1 = g.n1e - off, hi2 = g.n2e - off;
  if (hi1 <= 2 || hi2 <= 2) return;
  dim3 grid = grid2(hi1 - 2, hi2 - 2), block(kBX, kBY);
  if (sign > 0)
    k_v_update<1><<<grid, block, 0, st>>>(f.vx, f.vz, f.p, m, g.ld, hi1, hi2);
  else
    k_v_update<-1><<<grid, block, 0, st>>>(f.vx, f.vz, f.p, m, g.ld, hi1, hi2);
}

void plain_inject(const InjMapDev& map, float* fld, const float* w, float dt, const float* amp,
                  int amp_stride, int sign, cudaStream_t st) {
  if (map.npts == 0) return;
  k_inject<<<(map.npts + 255) / 256, 256, 0, st>>>(map, fld, w, dt, amp, amp_stride, sign);
}

void plain_psum(const Grid& g, PlainFields f, cudaStream_t st) {
  const int fsrows = g.ofs == 1 ? g.npml + 1 : 0;
  k_psum<<<grid2(g.n1e, g.n2e), dim3(kBX, kBY), 0, st>>>(f.p, f.px, f.pz, g.n1e, g.n2e, g.ld,
                                                         fsrows);
}

void plain_store_interior(const Grid& g, float* dst, const float* src, bool accumulate,
                          cudaStream_t st) {
  k_store<<<grid2(g.n1, g.n2), dim3(kBX, kBY), 0, st>>>(dst, src, g.n1, g.n2, g.npml, g.ld,
                                                        accumulate ? 1 : 0);
}

void plain_psrc(const Grid& g, const ModelDev& m, float* px, const float* sp, bool esource,
                cudaStream_t st) {
  const int lo = esource ? 1 : 0;
  const int hi1 = esource ? g.n1 - 1 : g.n1, hi2 = esource ? g.n2 - 1 : g.n2;
  if (hi1 <= lo || hi2 <= lo) return;
  k_psrc<<<grid2(hi1 - lo, hi2 - lo), dim3(kBX, kBY), 0, st>>>(px, sp, m.kap, g.dt, g.n1, g.n2,
                                                               g.npml, g.ld, lo, hi1, hi2);
}

void plain_vsrc(const Grid& g, const ModelDev& m, float* vx, float* vz, const float* svx,
                const float* svz, cudaStream_t st) {
  k_vsrc<<<grid2(g.n1, g.n2), dim3(kBX, kBY), 0, st>>>(vx, vz, svx, svz, m.rbue, g.dt, g.n1,
                                                       g.n2, g.npml, g.ld);
}

void plain_vz_free_surface(const Grid& g, float* vz, cudaStream_t st) {
  if (g.ofs != 1 || g.npml < 1) return;
  k_vz_fs<<<(g.n2e + 255) / 256, 256, 0, st>>>(vz, g.npml, g.n2e, g.ld);
}

void hicks_gather(const StationsDev& st, const float* origin, int ld, int shift, int hi1,
                  int hi2, float* out, int out_stride, int row, int nrows, size_t field_stride,
                  cudaStream_t s) {
  if (st.n == 0 || nrows <= 0) return;
  dim3 grid((st.n + kGatherWarps - 1) / kGatherWarps, nrows);
  k_gather<<<grid, kGatherWarps * 32, 0, s>>>(st, origin, ld, shift, hi1, hi2, out, out_stride,
                                              row, field_stride);
}

}  // namespace daw
