// Device helpers shared by the TMA-pipelined kernels (stencil_tma.cu,
// stencil_step.cu): mbarriers with bounded waits, 2-D/3-D tensor copies,
// L2 eviction policies, the max-|x| bookkeeping of the FP16 histories and the
// history stores/loads of a lane's row pair.
#pragma once

#include <cuda.h>

#include "fused.cuh"

namespace daw {
namespace {

constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(1) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: `budget` cycles (~1 s by default), then the error flag is
// raised and the caller proceeds (results of that launch are then invalid;
// the host reports it).
__device__ __forceinline__ void bar_wait(uint64_t* b, uint32_t parity, unsigned* err,
                                         long long budget = 1LL << 31) {
  if (bar_try(b, parity)) return;
  const long long t0 = clock64();
  while (!bar_try(b, parity)) {
    if (clock64() - t0 > budget) {
      atomicOr(err, kErrTimeout);
      return;
    }
  }
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y,
                                       uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(b))
      : "memory");
}
__device__ __forceinline__ void tma_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                       uint64_t* b, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(b)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ int amax_exponent(unsigned bits) {
  const int ef = (int)(bits >> 23);
  const int e = (ef == 0) ? -126 : ef - 126;
  return max(min(e, 120), -100);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }
__device__ __forceinline__ unsigned warp_amax_slots(const unsigned* slots) {
  return __reduce_max_sync(kAll, slots[threadIdx.x & 31]);
}
// The running max |x| is kept as the bit pattern of |x|: for finite values the
// integer order is the float order, and NaN/Inf patterns rank above every
// finite one, so a non-finite value in a history field raises kErrNonFinite.
__device__ __forceinline__ unsigned abs_bits(float x) { return __float_as_uint(x) & 0x7fffffffu; }
__device__ __forceinline__ void warp_amax_flush(unsigned v, unsigned* slot, unsigned* err) {
  const unsigned b = __reduce_max_sync(kAll, v);
  if ((threadIdx.x & 31) == 0 && b) {
    atomicMax(slot, b);
    if (b >= 0x7f800000u) atomicOr(err, kErrNonFinite);
  }
}

// L2 eviction priorities.  The history stream (written once in stage A, read
// once in stage B) is marked evict-first, so that it does not push the
// wavefield state out of L2; the injection tables, re-read every step, are
// marked evict-last.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_hint(void* p, uint32_t v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(void* p, unsigned short v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.b16 [%0], %1, %2;" ::"l"(p), "h"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(void* p, float2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ float2 ld_hint_f2(const float2* p, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
               : "=f"(v.x), "=f"(v.y)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int2 ld_hint_i2(const int2* p, uint64_t pol) {
  int2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
               : "=r"(v.x), "=r"(v.y)
               : "l"(p), "l"(pol));
  return v;
}

template <bool FP16>
struct Hist;
template <>
struct Hist<true> {
  static __device__ __forceinline__ void put2(void* base, int o, float a, float b, float inv,
                                              bool v0, bool v1, uint64_t pol) {
    __half* h = static_cast<__half*>(base);
    if (v0 && v1) {
      const __half2 q = __floats2half2_rn(a * inv, b * inv);
      st_hint(h + o, *reinterpret_cast<const uint32_t*>(&q), pol);
    } else if (v0) {
      st_hint(h + o, __half_as_ushort(__float2half_rn(a * inv)), pol);
    } else if (v1) {
      st_hint(h + o + 1, __half_as_ushort(__float2half_rn(b * inv)), pol);
    }
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
                                              bool v0, bool v1, uint64_t pol) {
    float* h = static_cast<float*>(base);
    if (v0 && v1)
      st_hint(h + o, make_float2(a, b), pol);
    else if (v0)
      st_hint(h + o, __float_as_uint(a), pol);
    else if (v1)
      st_hint(h + o + 1, __float_as_uint(b), pol);
  }
  static __device__ __forceinline__ float2 get2(const void* base, int o, float, bool v0,
                                                bool v1) {
    const float* h = static_cast<const float*>(base);
    if (v0 && v1) return *reinterpret_cast<const float2*>(h + o);
    return make_float2(v0 ? h[o] : 0.f, v1 ? h[o + 1] : 0.f);
  }
};

template <bool FP16>
__device__ __forceinline__ void* step_ptr(void* hist, int step0, size_t nih) {
  return static_cast<char*>(hist) + (size_t)step0 * 3 * nih * (FP16 ? 2 : 4);
}


// Programmatic dependent launch: a kernel lets the next one in its stream
// start launching (trigger), and waits, before touching anything an earlier
// kernel wrote, until those kernels have completed and their writes are
// visible (wait).  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launch with the programmatic-stream-serialization attribute when `pdl`.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*k)(KArgs...), int grid, int block, size_t smem,
                              cudaStream_t st, bool pdl, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

__device__ __forceinline__ float2 ldg2(const float* p) {
  return __ldg(reinterpret_cast<const float2*>(p));
}

// Same with the amplitudes read from global memory (more than kAmpMax
// stations, or the vz source of type_src = 1).
__device__ __forceinline__ float inject_at_global(const InjMapDev& m, float v, int r, float dt,
                                                  float w, const float* amp, int amp_stride,
                                                  int sign) {
  const int e0 = __ldg(m.rowptr + 2 * r), e1 = __ldg(m.rowptr + 2 * r + 1);
  for (int e = e0; e < e1; ++e) {
    const float2 q = __ldg(m.ent + e);
    const float a = __ldg(amp + (size_t)__float_as_int(q.y) * amp_stride);
    const float term = fmul(fmul(fmul(q.x, dt), a), w);
    v = sign > 0 ? fadd(v, term) : fsub(v, term);
  }
  return v;
}

}  // namespace
}  // namespace daw
