// Device helpers and kernel declarations shared by the CUDA sources.
#pragma once

#include "daw_internal.h"

namespace daw {

// Separately rounded single-precision operations: the reference's REAL
// arithmetic with no fused multiply-add, so the stencil and Hicks sums round
// exactly as the Fortran code's statements do.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

// Fourth-order staggered weights (src/submodeling2.f90:48-49).
constexpr float kA0 = 1.125f;
constexpr float kA1 = -1.0f / 24.0f;

// D-(f)_i = a0 (f_i - f_{i-1}) + a1 (f_{i+1} - f_{i-2})
__device__ __forceinline__ float dminus(float fm2, float fm1, float f0, float fp1) {
  return fadd(fmul(kA0, fsub(f0, fm1)), fmul(kA1, fsub(fp1, fm2)));
}
// D+(f)_i = a0 (f_{i+1} - f_i) + a1 (f_{i+2} - f_{i-1})
__device__ __forceinline__ float dplus(float fm1, float f0, float fp1, float fp2) {
  return fadd(fmul(kA0, fsub(fp1, f0)), fmul(kA1, fsub(fp2, fm1)));
}

// Hicks gather of station s by one warp, summed in the reference's order
// (i1 outer, i2 inner; src/submodeling2.f90:214-219).  The lanes form the 441
// products c*f in parallel into `prod` (shared, 444 floats, 16-byte aligned);
// lane 0 then adds them in order.  Taps outside the support clipped to
// [1,hi1]x[1,hi2] contribute +0, which leaves every partial sum's value
// unchanged.  Returns the sum on lane 0.
__device__ __forceinline__ float warp_gather_ordered(float* prod, const int* ix1p,
                                                     const int* ix2p, const float* tiles, int s,
                                                     const float* __restrict__ origin, int ld,
                                                     int shift, int hi1, int hi2) {
  const int lane = threadIdx.x & 31;
  const int ix1 = __ldg(ix1p + s) - shift, ix2 = __ldg(ix2p + s) - shift;
  const int r1a = max(1 - ix1, -kRad), r1b = min(hi1 - ix1, kRad);
  const int r2a = max(1 - ix2, -kRad), r2b = min(hi2 - ix2, kRad);
  const float* tile = tiles + (size_t)s * kTile;
  // Lane l owns taps t = l + 32 k (k < 14); all 28 loads are issued before
  // the products, so their latencies overlap.  Tap t = (a+10)*21 + (b+10):
  // stepping t by 32 = 21 + 11 steps b by 11 and a by 1 (or 2 on wrap).
  constexpr int kSteps = (444 + 31) / 32;
  float tv[kSteps], pv[kSteps];
  {
    int a = lane / kTap - kRad, b = lane % kTap - kRad;
#pragma unroll
    for (int k = 0; k < kSteps; ++k) {
      const int t = lane + 32 * k;
      const bool in = t < kTile && a >= r1a && a <= r1b && b >= r2a && b <= r2b;
      tv[k] = in ? __ldg(tile + (a + kRad) + kTap * (b + kRad)) : 0.f;
      pv[k] = in ? origin[(ix1 + a - 1) + (size_t)ld * (ix2 + b - 1)] : 0.f;
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
    if (lane + 32 * k < 444) prod[lane + 32 * k] = fmul(tv[k], pv[k]);  // +0 outside the support
  __syncwarp();
  float acc = 0.f;
  if (lane == 0) {
    const float4* p4 = reinterpret_cast<const float4*>(prod);
#pragma unroll 4
    for (int q = 0; q < 111; ++q) {
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

// ---------------------------------------------------------------------------
// Launch wrappers (stencil_plain.cu): the literal port, one kernel per
// reference loop nest.  Indices are 0-based; reference index I = i + 1.
// ---------------------------------------------------------------------------
struct PlainFields {
  float *p, *px, *pz, *vx, *vz;
};

void plain_p_update(const Grid& g, const ModelDev& m, PlainFields f, int off, int sign,
                    cudaStream_t st);
void plain_v_update(const Grid& g, const ModelDev& m, PlainFields f, int off, int sign,
                    cudaStream_t st);
// fld[k] +/-= ((c*dt)*amp[sta*amp_stride])*w[k] for every touched point.
void plain_inject(const InjMapDev& map, float* fld, const float* w, float dt,
                  const float* amp, int amp_stride, int sign, cudaStream_t st);
void plain_psum(const Grid& g, PlainFields f, cudaStream_t st);
// dst(n1,n2) = (or +=) interior of the extended field src.
void plain_store_interior(const Grid& g, float* dst, const float* src, bool accumulate,
                          cudaStream_t st);
void plain_psrc(const Grid& g, const ModelDev& m, float* px, const float* sp, bool esource,
                cudaStream_t st);
// v += -dt * s * bu (bu = 1 when the model has no density).
void plain_vsrc(const Grid& g, const ModelDev& m, float* vx, float* vz, const float* svx,
                const float* svz, cudaStream_t st);
void plain_vz_free_surface(const Grid& g, float* vz, cudaStream_t st);

// Hicks gather of `field` (leading dimension ld; `origin` is the address of
// 1-based index (1,1) of the station indices after subtracting `shift`) at
// every station, support clipped to [1,hi1]x[1,hi2]; one sequential sum per
// station in the reference's order (i1 outer, i2 inner).
// out[row + out_stride*station] = sum.  nrows > 1 batches consecutive
// histories (field advanced by field_stride, row by 1).
void hicks_gather(const StationsDev& st, const float* origin, int ld, int shift, int hi1,
                  int hi2, float* out, int out_stride, int row, int nrows,
                  size_t field_stride, cudaStream_t s);

// ---------------------------------------------------------------------------
// MINRES vector kernels (minres.cu)
// ---------------------------------------------------------------------------
template <typename S>
struct MinresDev {
  S beta1, beta, oldb, alfa, dbar, epsln, qrnorm, phibar, rhs1, rhs2, tnorm2, ynorm2;
  S cs, sn, gmax, gmin, shift, anorm, acond, rnorm, ynorm, arnorml;
  S s_inv, q1, q2, oldeps, delta, denom, phi, eps, rtol, fac;
  int itn, istop, itnlim, nlog, done, log_capacity;
};

template <typename S>
struct MinresOps {
  static void dot(const float* a, const float* b, size_t n, S* partials, int nblk,
                  cudaStream_t st);
  static void init(MinresDev<S>* d, const S* pb, const S* pgb, const S* pbb, int nblk,
                   float mu, int itnlim, float rtol, cudaStream_t st);
  static void arnorm0(MinresDev<S>* d, const S* pww, int nblk, cudaStream_t st);
  static void v_from_y(MinresDev<S>* d, float* v, const float* y, size_t n, cudaStream_t st);
  static void y1(MinresDev<S>* d, float* y, const float* v, const float* r1, size_t n,
                 S* partials, int nblk, cudaStream_t st);
  static void alfa(MinresDev<S>* d, const S* partials, int nblk, cudaStream_t st);
  static void y2(MinresDev<S>* d, float* y, const float* r2, size_t n, S* partials, int nblk,
                 cudaStream_t st);
  static void scal(MinresDev<S>* d, const S* partials, int nblk, double* log,
                   const float* x0, cudaStream_t st);
  static void xw(MinresDev<S>* d, float* w, const float* w1, const float* w2, const float* v,
                 float* x, size_t n, cudaStream_t st);
};
int minres_blocks(size_t n);

// Residuals and sums (minres.cu)
// deltadr(nt-it+1, r) = dobs(it, r) - datar(it, r)  (src/subresiduals.f90:12-16)
void residuals(const float* dobs, const float* datar, float* deltadr, int nt, int nr,
               cudaStream_t st);
void vec_add(const float* a, const float* b, float* c, size_t n, cudaStream_t st);
// Traces (nt, nr), time fastest, to step-major [nt][nr] (minres.cu).
void transpose_traces(const float* in, float* out, int nt, int nr, cudaStream_t st);

// filmartin2d on the device (filter.cu): weights w[0..nto] as the reference
// builds them; each trace zero padded to nto, FP64 real FFT, bins 0..nto/2-1
// scaled by w[k], the Nyquist bin by w[0], inverse.
void filter_traces(const float* in, float* out, int nt, int nr, int nto, const double* w,
                   double* scratch, cudaStream_t st);
size_t filter_scratch_bytes(int nr, int nto);
// Loads the filter kernel onto the current device (filter.cu).
bool filter_preload();
// Set-up of daw_filmartin2d_noalloc on the current device (filter_noalloc.cu):
// takes the device address of its fixed work-space array (which loads that
// array's module and so reserves the array) and loads the filter kernel.
// Idempotent per device; 0 or a negative daw_status, with the message in err.
int filter_noalloc_prepare(char* err, int err_len);
// Padded length nto of filmartin2d (next power of two >= nt, 8..65536), or 0
// when nt exceeds 65536 (src/minresModule.f90:503-510).
int filter_nto(int nt);
// The band-pass weights w[0..nto] (src/minresModule.f90:505-586) into caller
// storage: fm (work) of nto + 1 floats, w of nto + 1 doubles.  Applies the
// reference's in-place fhig/lhig clamp.  Returns nto, 0 when nt > 65536.
int filter_weights_into(int nt, float dt, float* flow, float* fhig, float* llow, float* lhig,
                        float* fm, double* w);

}  // namespace daw
