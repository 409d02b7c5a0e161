// filmartin2d on the device (src/minresModule.f90:486-614): each trace is
// zero padded to nto (a power of two), transformed with an FP64 real FFT,
// scaled bin by bin by the reference's trapezoid + Hanning^2 weights, and
// transformed back.  The reference's packed REALFT2S layout
// (src/libfourier.f90:199-276) stores the Nyquist coefficient in the
// imaginary slot of bin 0, so the filter multiplies it by the DC weight w[0];
// that is kept here.
//
// The real transform of length nto = 2N is computed through one complex
// radix-2 FFT of length N on z[n] = x[2n] + i x[2n+1] (the standard
// even/odd packing), one CTA per trace, in shared memory when 16N bytes fit
// and in a global scratch slice otherwise.
#include "kernels.cuh"

namespace daw {
namespace {

constexpr int kFftThreads = 512;
constexpr size_t kSmemLimit = 160 * 1024;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place radix-2 complex FFT of length n = 2^logn; sign -1 forward, +1
// inverse (unnormalised).
__device__ void fft_inplace(double2* z, int n, int logn, double sign) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int r = (int)(__brev((unsigned)k) >> (32 - logn));
    if (k < r) {
      const double2 t = z[k];
      z[k] = z[r];
      z[r] = t;
    }
  }
  __syncthreads();
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1;
    for (int j = threadIdx.x; j < n / 2; j += blockDim.x) {
      const int pos = j % half;
      const int i0 = (j / half) * len + pos, i1 = i0 + half;
      double s, c;
      sincospi(sign * 2.0 * (double)pos / (double)len, &s, &c);
      const double2 t = cmul(make_double2(c, s), z[i1]);
      const double2 a = z[i0];
      z[i0] = make_double2(a.x + t.x, a.y + t.y);
      z[i1] = make_double2(a.x - t.x, a.y - t.y);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kFftThreads)
    k_filter(const float* __restrict__ in, float* __restrict__ out, int nt, int nto, int logn,
             const double* __restrict__ w, double2* __restrict__ scratch, int use_smem) {
  extern __shared__ double2 smem[];
  const int n = nto / 2;
  const int tr = blockIdx.x;
  double2* z = use_smem ? smem : scratch + (size_t)tr * n;
  const float* x = in + (size_t)nt * tr;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int a = 2 * k, b = 2 * k + 1;
    z[k] = make_double2(a < nt ? (double)x[a] : 0.0, b < nt ? (double)x[b] : 0.0);
  }
  __syncthreads();
  fft_inplace(z, n, logn, -1.0);
  // Unpack to the real spectrum X[k], k = 0..n, weight it, repack for the
  // inverse.  Thread handles the pair (k, n-k).
  for (int k = threadIdx.x; k <= n / 2; k += blockDim.x) {
    const int m = (n - k) % n;  // partner index (0 pairs with n)
    const double2 zk = z[k], zm = z[m];
    double2 Xk, Xm;  // X[k], X[n-k]
    if (k == 0) {
      Xk = make_double2(zk.x + zk.y, 0.0);   // X[0]
      Xm = make_double2(zk.x - zk.y, 0.0);   // X[n] (Nyquist)
    } else {
      // Fe = (z[k] + conj z[m]) / 2 ; Fo = (z[k] - conj z[m]) / (2i)
      const double2 fe = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
      const double2 fo = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
      double s, c;
      sincospi(-(double)k / (double)n, &s, &c);
      const double2 t = cmul(make_double2(c, s), fo);
      Xk = make_double2(fe.x + t.x, fe.y + t.y);
      // X[n-k] = conj(Fe) - e^{-i pi k/n}... from the same halves:
      // X[m] = conj(fe) + e^{-i pi m/n} conj(fo) = conj(fe) - conj(e^{-i pi k / n} fo)
      Xm = make_double2(fe.x - t.x, -(fe.y - t.y));
    }
    const double wk = w[k];
    const double wm = (k == 0) ? w[0] : w[n - k];
    Xk.x *= wk; Xk.y *= wk;
    Xm.x *= wm; Xm.y *= wm;
    if (k == 0) {
      // Z'[0] = Ye + i Yo with Ye = (X0 + Xn)/2, Yo = (X0 - Xn)/2 (both real)
      z[0] = make_double2(0.5 * (Xk.x + Xm.x), 0.5 * (Xk.x - Xm.x));
    } else {
      // Ye[k] = (X[k] + conj X[n-k]) / 2, Yo[k] = (X[k] - conj X[n-k]) e^{+i pi k/n} / 2
      double s, c;
      sincospi((double)k / (double)n, &s, &c);
      const double2 ye = make_double2(0.5 * (Xk.x + Xm.x), 0.5 * (Xk.y - Xm.y));
      const double2 yo = cmul(make_double2(0.5 * (Xk.x - Xm.x), 0.5 * (Xk.y + Xm.y)),
                              make_double2(c, s));
      z[k] = make_double2(ye.x - yo.y, ye.y + yo.x);
      if (m != k) {
        // Ye[m] = conj(Ye[k]); Yo[m] = (X[m] - conj X[k]) e^{+i pi m/n} / 2 = conj(Yo[k])
        z[m] = make_double2(ye.x + yo.y, -ye.y + yo.x);
      }
    }
  }
  __syncthreads();
  fft_inplace(z, n, logn, +1.0);
  float* y = out + (size_t)nt * tr;
  const double inv = 1.0 / (double)n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int a = 2 * k, b = 2 * k + 1;
    if (a < nt) y[a] = (float)(z[k].x * inv);
    if (b < nt) y[b] = (float)(z[k].y * inv);
  }
}

}  // namespace

// Loads the filter kernel's code onto the current device and sets its
// shared-memory opt-in.  Under lazy module loading (the default since CUDA
// 12.2) that would otherwise happen at its first launch and may need device
// memory then.
bool filter_preload() {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, k_filter) == cudaSuccess &&
         cudaFuncSetAttribute(k_filter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kSmemLimit) == cudaSuccess;
}

size_t filter_scratch_bytes(int nr, int nto) {
  const size_t per = (size_t)(nto / 2) * sizeof(double2);
  return per <= kSmemLimit ? 0 : per * (size_t)nr;
}

void filter_traces(const float* in, float* out, int nt, int nr, int nto, const double* w,
                   double* scratch, cudaStream_t st) {
  if (nr <= 0) return;
  int logn = 0;
  while ((1 << logn) < nto / 2) ++logn;
  const size_t bytes = (size_t)(nto / 2) * sizeof(double2);
  const int use_smem = bytes <= kSmemLimit ? 1 : 0;
  if (use_smem) {
    cudaFuncSetAttribute(k_filter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
  }
  k_filter<<<nr, kFftThreads, use_smem ? bytes : 0, st>>>(in, out, nt, nto, logn, w,
                                                         reinterpret_cast<double2*>(scratch),
                                                         use_smem);
}

}  // namespace daw
