// daw_filmartin2d_noalloc: the filmartin2d band-pass on traces that are
// already in device memory, with no device allocation at all.
//
// Who needs it.  Some callers cannot call cudaMalloc when they want to filter:
//   - a process whose GPU memory is already spoken for -- a shot batch of this
//     library is admitted by HBM footprint and may hold ~92 % of the device
//     for wavefield histories, and a host framework with its own caching
//     allocator may own the rest -- so a new allocation fails;
//   - code that must not stall other streams: cudaMalloc and cudaFree
//     synchronise the whole device.
// The regular entry point (daw_filmartin2d) takes host arrays and draws its
// weights and FFT work space from a handle's device pool.  This one takes the
// caller's device buffers for the input and output traces and keeps its work
// space in one fixed array, g_filter_scratch below.
//
// The fixed array: kScratchBytes (4 MiB) on every GPU where it is set up,
// held until the process exits.  Its first kWeightBytes hold the nto + 1 FP64
// weights (nto <= 65536, the reference's own limit); the rest is FFT work
// space for traces whose transform does not fit in shared memory
// (nt > 16384), filtered a few traces per launch.  Nothing in it has to start
// at zero: each call writes every weight and every FFT element before it
// reads them.
//
// Set-up, once per device, with that device current
// (filter_noalloc_prepare): host code cannot use g_filter_scratch's name as a
// device address, so the set-up takes the address with cudaGetSymbolAddress
// and keeps it.  Under lazy module loading (the CUDA default since 12.2) that
// call is also what loads this file's module onto the device and so reserves
// the 4 MiB; the set-up loads the filter kernel's code as well.  Both can
// need device memory, so they must not wait for a call made when HBM is
// full: daw_create runs the set-up for its device, and a caller that never
// creates a handle on a device makes one call with nr = 0 (buffers may then
// be NULL) before filling the device.  A first call that finds the set-up
// undone runs it itself; make that call before any stream capture.
//
// Every call shares the one array and leaves its contents behind.  Work from
// two calls that overlapped on the GPU would race on it, so calls are
// serialised: a lock is held from the weight upload until the call's GPU work
// has finished, and the call returns only then.
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "daw_internal.h"
#include "kernels.cuh"

namespace {

constexpr int kMaxNto = 65536;
constexpr size_t kWeightBytes = 524544;      // (kMaxNto + 1) doubles, rounded up to 256 B
constexpr size_t kScratchBytes = 4u << 20;   // 4 MiB in all
static_assert(kWeightBytes >= (size_t)(kMaxNto + 1) * sizeof(double) && kWeightBytes % 256 == 0,
              "weight region");
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_filter_scratch[kScratchBytes];

std::mutex g_lock;
unsigned char* g_scratch_ptr[kMaxDevices] = {};  // device address of g_filter_scratch, per device
// Host staging of the weights (static: the call allocates no host memory
// either); used under g_lock only.
float g_fm[kMaxNto + 1];
double g_w[kMaxNto + 1];

int fail(char* err, int err_len, int code, const char* fmt, ...) {
  if (err && err_len > 0) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(err, (size_t)err_len, fmt, ap);
    va_end(ap);
  }
  return code;
}

bool is_device_pointer(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

// The set-up of one device, under g_lock; 0 or a negative daw_status.
int prepare_locked(int dev, char* err, int err_len) {
  using namespace daw;
  if (dev < 0 || dev >= kMaxDevices)
    return fail(err, err_len, DAW_ERR_ARG, "daw_filmartin2d_noalloc: device %d outside 0..%d",
                dev, kMaxDevices - 1);
  if (g_scratch_ptr[dev]) return DAW_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_filter_scratch);
  if (e != cudaSuccess || !p)
    return fail(err, err_len, DAW_ERR_CUDA,
                "daw_filmartin2d_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(e));
  if (!filter_preload()) {
    e = cudaGetLastError();
    return fail(err, err_len, DAW_ERR_CUDA,
                "daw_filmartin2d_noalloc: loading the filter kernel failed on device %d: %s", dev,
                cudaGetErrorString(e));
  }
  g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  return DAW_OK;
}

}  // namespace

namespace daw {
int filter_noalloc_prepare(char* err, int err_len) {
  std::lock_guard<std::mutex> guard(g_lock);
  int dev = -1;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0)
    return fail(err, err_len, DAW_ERR_NODEV, "daw_filmartin2d_noalloc: no current device (%s)",
                cudaGetErrorString(e));
  return prepare_locked(dev, err, err_len);
}
}  // namespace daw

extern "C" int daw_filmartin2d_noalloc(const float* d_in, int32_t nr, int32_t nt, float dt,
                                       float* flow, float* fhig, float* llow, float* lhig,
                                       float* d_out, void* stream, char* err, int32_t err_len) {
  using namespace daw;
  if ((nr > 0 && (!d_in || !d_out)) || !flow || !fhig || !llow || !lhig || nr < 0 || nt <= 0 ||
      !(dt > 0))
    return fail(err, err_len, DAW_ERR_ARG, "daw_filmartin2d_noalloc: bad arguments");
  if (nt > kMaxNto)
    return fail(err, err_len, DAW_ERR_ARG,
                "daw_filmartin2d_noalloc: nt = %d exceeds the maximum of %d samples that its "
                "fixed %zu-byte work space holds",
                nt, kMaxNto, kScratchBytes);
  std::lock_guard<std::mutex> guard(g_lock);
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0)
    return fail(err, err_len, DAW_ERR_NODEV, "daw_filmartin2d_noalloc: no current device (%s)",
                cudaGetErrorString(e));
  const int rc = prepare_locked(dev, err, err_len);  // once per device
  if (rc != DAW_OK) return rc;
  if (nr > 0 && (!is_device_pointer(d_in, dev) || !is_device_pointer(d_out, dev)))
    return fail(err, err_len, DAW_ERR_ARG,
                "daw_filmartin2d_noalloc: input and output must be device memory of the "
                "current device %d",
                dev);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nto = filter_weights_into(nt, dt, flow, fhig, llow, lhig, g_fm, g_w);
  double* w = reinterpret_cast<double*>(g_scratch_ptr[dev]);
  double* fft = reinterpret_cast<double*>(g_scratch_ptr[dev] + kWeightBytes);
  // Pageable source: the copy has taken g_w's contents when it returns.
  e = cudaMemcpyAsync(w, g_w, (size_t)(nto + 1) * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess)
    return fail(err, err_len, DAW_ERR_CUDA, "daw_filmartin2d_noalloc: weight upload: %s",
                cudaGetErrorString(e));
  if (nr > 0) {
    const size_t per_trace = filter_scratch_bytes(1, nto);  // 0: shared-memory transform
    const int group =
        per_trace ? (int)((kScratchBytes - kWeightBytes) / per_trace) : (int)nr;
    for (int r0 = 0; r0 < nr; r0 += group) {
      const int ng = group < nr - r0 ? group : nr - r0;
      filter_traces(d_in + (size_t)nt * r0, d_out + (size_t)nt * r0, nt, ng, nto, w,
                    per_trace ? fft : nullptr, st);
      e = cudaGetLastError();
      if (e != cudaSuccess) break;
    }
  }
  // Return only once this call's work on the array has finished.
  const cudaError_t es = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess)
    return fail(err, err_len, DAW_ERR_CUDA, "daw_filmartin2d_noalloc: %s",
                cudaGetErrorString(e));
  return DAW_OK;
}
