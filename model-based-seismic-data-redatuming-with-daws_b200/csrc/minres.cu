// Device-resident MINRES (src/minresModule.f90:10-360 as called by
// src/sublinearminres.f90:30-86): FP32 vectors; inner products, norms and the
// Lanczos/Givens scalars in S (float for the plain port, double for the
// mixed path).  Reductions are deterministic: fixed per-block partial sums,
// then one block adds the partials in a fixed tree order.
#include <cfloat>

#include "kernels.cuh"

namespace daw {
namespace {

constexpr int kThreads = 256;

template <typename S>
__device__ S block_sum(S v, S* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  S r = sh[0];
  __syncthreads();
  return r;
}

// Sum of nblk partials by one block in a fixed order.
template <typename S>
__device__ S reduce_partials(const S* p, int nblk, S* sh) {
  S acc = 0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += p[i];
  return block_sum<S>(acc, sh);
}

template <typename S>
__global__ void __launch_bounds__(kThreads) k_dot(const float* __restrict__ a,
                                                  const float* __restrict__ b, size_t n,
                                                  S* __restrict__ partials) {
  __shared__ S sh[kThreads];
  S acc = 0;
  for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads)
    acc += (S)a[i] * (S)b[i];
  S r = block_sum<S>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// sublinearminres.f90:64-72 and MINRES set-up (minresModule.f90:70-153).
template <typename S>
__global__ void __launch_bounds__(kThreads) k_init(MinresDev<S>* d, const S* pb, const S* pgb,
                                                   const S* pbb, int nblk, float mu,
                                                   int itnlim, float rtol) {
  __shared__ S sh[kThreads];
  const S nb2 = reduce_partials<S>(pb, nblk, sh);
  const S ngb2 = reduce_partials<S>(pgb, nblk, sh);
  const S bb = reduce_partials<S>(pbb, nblk, sh);
  if (threadIdx.x != 0) return;
  // datanorm(deltadr), datanorm(G G^T deltadr); fac = norm ratio * mu.
  const S fac = (S)sqrt(nb2) / (S)sqrt(ngb2) * (S)mu;
  d->fac = fac;
  d->shift = -fac;
  d->eps = (S)FLT_EPSILON;  // epsilon of the reference's REAL
  d->rtol = (S)rtol;
  d->itnlim = itnlim;
  d->itn = 0;
  d->istop = 0;
  d->nlog = 0;
  d->anorm = d->acond = d->rnorm = d->ynorm = 0;
  d->done = 0;
  S beta1 = bb;  // dot_product(b, y) with y = b
  if (beta1 < 0) { d->istop = 8; d->done = 1; return; }
  if (beta1 == 0) { d->istop = 0; d->done = 1; return; }
  beta1 = (S)sqrt(beta1);
  d->beta1 = beta1;
  d->oldb = 0;
  d->beta = beta1;
  d->dbar = 0;
  d->epsln = 0;
  d->qrnorm = beta1;
  d->phibar = beta1;
  d->rhs1 = beta1;
  d->rhs2 = 0;
  d->tnorm2 = 0;
  d->ynorm2 = 0;
  d->cs = -1;
  d->sn = 0;
  d->gmax = d->gmin = 0;
  d->s_inv = (S)1 / beta1;
  d->q1 = 0;
}

template <typename S>
__global__ void __launch_bounds__(kThreads) k_arnorm0(MinresDev<S>* d, const S* pww, int nblk) {
  __shared__ S sh[kThreads];
  const S ww = reduce_partials<S>(pww, nblk, sh);
  if (threadIdx.x == 0) d->arnorml = (S)sqrt(ww);
}

// v = (1/beta) y  (minresModule.f90:181-182)
template <typename S>
__global__ void k_v(const MinresDev<S>* __restrict__ d, float* __restrict__ v,
                    const float* __restrict__ y, size_t n) {
  if (d->done) return;
  const S s = d->s_inv;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    v[i] = (float)(s * (S)y[i]);
}

// y = y - shift v; y = y - (beta/oldb) r1 (itn >= 2); partial v.y
// (minresModule.f90:185-190)
template <typename S>
__global__ void __launch_bounds__(kThreads) k_y1(const MinresDev<S>* __restrict__ d,
                                                 float* __restrict__ y,
                                                 const float* __restrict__ v,
                                                 const float* __restrict__ r1, size_t n,
                                                 S* __restrict__ partials) {
  __shared__ S sh[kThreads];
  if (d->done) return;
  const S shift = d->shift, q = d->q1;
  const bool second = d->itn >= 1;  // itn counts completed iterations here
  S acc = 0;
  for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads) {
    S vi = (S)v[i];
    S yi = (S)y[i];
    if (sizeof(S) == sizeof(float)) {
      yi = (S)(float)(yi - shift * vi);
      if (second) yi = (S)(float)(yi - q * (S)r1[i]);
    } else {
      yi = yi - shift * vi;
      if (second) yi = yi - q * (S)r1[i];
    }
    const float yf = (float)yi;
    y[i] = yf;
    acc += vi * (S)yf;
  }
  S r = block_sum<S>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

template <typename S>
__global__ void __launch_bounds__(kThreads) k_alfa(MinresDev<S>* d, const S* partials, int nblk) {
  __shared__ S sh[kThreads];
  const S a = reduce_partials<S>(partials, nblk, sh);
  if (threadIdx.x == 0 && !d->done) {
    d->alfa = a;
    d->q2 = a / d->beta;
  }
}

// y = y - (alfa/beta) r2; partial y.y  (:191-197, with r2 := y afterwards)
template <typename S>
__global__ void __launch_bounds__(kThreads) k_y2(const MinresDev<S>* __restrict__ d,
                                                 float* __restrict__ y,
                                                 const float* __restrict__ r2, size_t n,
                                                 S* __restrict__ partials) {
  __shared__ S sh[kThreads];
  if (d->done) return;
  const S q = d->q2;
  S acc = 0;
  for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads) {
    const float yf = (float)((S)y[i] - q * (S)r2[i]);
    y[i] = yf;
    acc += (S)yf * (S)yf;
  }
  S r = block_sum<S>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// Lanczos/Givens scalars of one iteration (minresModule.f90:196-303).
template <typename S>
__global__ void __launch_bounds__(kThreads) k_scal(MinresDev<S>* d, const S* partials, int nblk,
                                                   double* log, const float* x) {
  __shared__ S sh[kThreads];
  const S bb = reduce_partials<S>(partials, nblk, sh);
  if (threadIdx.x != 0 || d->done) return;
  const int itn = d->itn + 1;
  d->itn = itn;
  const S alfa = d->alfa;
  const S oldb = d->beta;
  d->oldb = oldb;
  S beta = bb;
  if (beta < 0) {
    d->istop = 6;
    d->done = 1;
    return;
  }
  beta = (S)sqrt(beta);
  d->beta = beta;
  d->tnorm2 = d->tnorm2 + alfa * alfa + oldb * oldb + beta * beta;
  if (itn == 1) {
    if (beta / d->beta1 <= (S)10 * d->eps) d->istop = -1;
    d->gmax = (S)fabs(alfa);
    d->gmin = d->gmax;
  }
  const S oldeps = d->epsln;
  const S delta = d->cs * d->dbar + d->sn * alfa;
  const S gbar = d->sn * d->dbar - d->cs * alfa;
  d->epsln = d->sn * beta;
  d->dbar = -d->cs * beta;
  const S gamma = (S)sqrt(gbar * gbar + beta * beta);
  d->cs = gbar / gamma;
  d->sn = beta / gamma;
  const S phi = d->cs * d->phibar;
  d->phibar = d->sn * d->phibar;
  d->oldeps = oldeps;
  d->delta = delta;
  d->denom = (S)1 / gamma;
  d->phi = phi;
  d->gmax = d->gmax > gamma ? d->gmax : gamma;
  d->gmin = d->gmin < gamma ? d->gmin : gamma;
  const S z = d->rhs1 / gamma;
  d->ynorm2 = z * z + d->ynorm2;
  d->rhs1 = d->rhs2 - delta * z;
  d->rhs2 = -d->epsln * z;
  d->anorm = (S)sqrt(d->tnorm2);
  d->ynorm = (S)sqrt(d->ynorm2);
  d->qrnorm = d->phibar;
  const S rnorml = d->rnorm;
  d->rnorm = d->qrnorm;
  const S rootl = (S)sqrt(gbar * gbar + d->dbar * d->dbar);
  d->arnorml = rnorml * rootl;
  d->acond = d->gmax / d->gmin;
  if (d->istop == 0) {
    if (itn >= d->itnlim) d->istop = 5;
    if (d->qrnorm / d->beta1 <= d->rtol) d->istop = 1;
  }
  // next iteration's v = y/beta and y -= (beta/oldb) r1
  d->s_inv = (S)1 / beta;
  d->q1 = beta / oldb;
}

// w1 = w2; w2 = w; w = (v - oldeps w1 - delta w2)/gamma; x += phi w
// (minresModule.f90:250-257).  The host rotates the w buffers, so `w` is the
// old w1 buffer, w1 the old w2 and w2 the old w.
template <typename S>
__global__ void k_xw(MinresDev<S>* __restrict__ d, float* __restrict__ w,
                     const float* __restrict__ w1, const float* __restrict__ w2,
                     const float* __restrict__ v, float* __restrict__ x, size_t n) {
  if (d->done) return;
  const S oe = d->oldeps, de = d->delta, dn = d->denom, ph = d->phi;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    S wi;
    if (sizeof(S) == sizeof(float)) {
      wi = (S)(float)((S)(float)((S)(float)((S)v[i] - oe * (S)w1[i]) - de * (S)w2[i]) * dn);
      x[i] = (float)((S)x[i] + ph * wi);
    } else {
      wi = ((S)v[i] - oe * (S)w1[i] - de * (S)w2[i]) * dn;
      x[i] = (float)((S)x[i] + ph * wi);
    }
    w[i] = (float)wi;
  }
}

// Log row and stop flag, after the x update (x(1) is reported, :323).
template <typename S>
__global__ void k_log(MinresDev<S>* d, double* log, const float* x) {
  if (d->done) return;
  if (log && d->nlog < d->log_capacity) {
    double* r = log + 5 * (size_t)d->nlog;
    r[0] = d->itn;
    r[1] = (double)x[0];
    r[2] = (double)(d->qrnorm / d->beta1);
    r[3] = (double)d->anorm;
    r[4] = (double)d->acond;
    d->nlog++;
  }
  if (d->istop != 0) d->done = 1;
}

__global__ void k_residuals(const float* __restrict__ dobs, const float* __restrict__ datar,
                            float* __restrict__ res, int nt, int nr) {
  const size_t n = (size_t)nt * nr;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int it = (int)(i % nt);
    const size_t r = i / nt;
    res[(nt - 1 - it) + (size_t)nt * r] = __fsub_rn(dobs[i], datar[i]);
  }
}

__global__ void k_add(const float* a, const float* b, float* c, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    c[i] = __fadd_rn(a[i], b[i]);
}

// out[t * nr + r] = in[t + nt * r]: traces (nt, nr) to step-major order, by
// 32 x 32 tiles through shared memory (both sides coalesced).
__global__ void k_transpose(const float* __restrict__ in, float* __restrict__ out, int nt, int nr) {
  __shared__ float tile[32][33];
  const int t0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int t = t0 + threadIdx.x, r = r0 + k;
    if (t < nt && r < nr) tile[k][threadIdx.x] = in[t + (size_t)nt * r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int t = t0 + k, r = r0 + threadIdx.x;
    if (t < nt && r < nr) out[(size_t)t * nr + r] = tile[threadIdx.x][k];
  }
}

int grid_for(size_t n) {
  size_t b = (n + 1023) / 1024;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

}  // namespace

int minres_blocks(size_t n) {
  size_t b = (n + 4 * kThreads - 1) / (4 * kThreads);
  if (b < 1) b = 1;
  if (b > 148 * 8) b = 148 * 8;
  return (int)b;
}

template <typename S>
void MinresOps<S>::dot(const float* a, const float* b, size_t n, S* partials, int nblk,
                       cudaStream_t st) {
  k_dot<S><<<nblk, kThreads, 0, st>>>(a, b, n, partials);
}
template <typename S>
void MinresOps<S>::init(MinresDev<S>* d, const S* pb, const S* pgb, const S* pbb, int nblk,
                        float mu, int itnlim, float rtol, cudaStream_t st) {
  k_init<S><<<1, kThreads, 0, st>>>(d, pb, pgb, pbb, nblk, mu, itnlim, rtol);
}
template <typename S>
void MinresOps<S>::arnorm0(MinresDev<S>* d, const S* pww, int nblk, cudaStream_t st) {
  k_arnorm0<S><<<1, kThreads, 0, st>>>(d, pww, nblk);
}
template <typename S>
void MinresOps<S>::v_from_y(MinresDev<S>* d, float* v, const float* y, size_t n,
                            cudaStream_t st) {
  k_v<S><<<grid_for(n), 256, 0, st>>>(d, v, y, n);
}
template <typename S>
void MinresOps<S>::y1(MinresDev<S>* d, float* y, const float* v, const float* r1, size_t n,
                      S* partials, int nblk, cudaStream_t st) {
  k_y1<S><<<nblk, kThreads, 0, st>>>(d, y, v, r1, n, partials);
}
template <typename S>
void MinresOps<S>::alfa(MinresDev<S>* d, const S* partials, int nblk, cudaStream_t st) {
  k_alfa<S><<<1, kThreads, 0, st>>>(d, partials, nblk);
}
template <typename S>
void MinresOps<S>::y2(MinresDev<S>* d, float* y, const float* r2, size_t n, S* partials,
                      int nblk, cudaStream_t st) {
  k_y2<S><<<nblk, kThreads, 0, st>>>(d, y, r2, n, partials);
}
template <typename S>
void MinresOps<S>::scal(MinresDev<S>* d, const S* partials, int nblk, double* log,
                        const float* x0, cudaStream_t st) {
  k_scal<S><<<1, kThreads, 0, st>>>(d, partials, nblk, log, x0);
}
template <typename S>
void MinresOps<S>::xw(MinresDev<S>* d, float* w, const float* w1, const float* w2,
                      const float* v, float* x, size_t n, cudaStream_t st) {
  k_xw<S><<<grid_for(n), 256, 0, st>>>(d, w, w1, w2, v, x, n);
}

template struct MinresOps<float>;
template struct MinresOps<double>;

// Exposed to the engine for the log/stop step.
void minres_log_f32(MinresDev<float>* d, double* log, const float* x, cudaStream_t st) {
  k_log<float><<<1, 1, 0, st>>>(d, log, x);
}
void minres_log_f64(MinresDev<double>* d, double* log, const float* x, cudaStream_t st) {
  k_log<double><<<1, 1, 0, st>>>(d, log, x);
}

void residuals(const float* dobs, const float* datar, float* deltadr, int nt, int nr,
               cudaStream_t st) {
  const size_t n = (size_t)nt * nr;
  k_residuals<<<grid_for(n), 256, 0, st>>>(dobs, datar, deltadr, nt, nr);
}

void vec_add(const float* a, const float* b, float* c, size_t n, cudaStream_t st) {
  k_add<<<grid_for(n), 256, 0, st>>>(a, b, c, n);
}

void transpose_traces(const float* in, float* out, int nt, int nr, cudaStream_t st) {
  if (nt <= 0 || nr <= 0) return;
  const dim3 grid((nt + 31) / 32, (nr + 31) / 32);
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(in, out, nt, nr);
}

}  // namespace daw
