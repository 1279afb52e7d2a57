// fg_common.cuh -- shared types and helpers of the B200 MD-step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Bounds-checked builds (-DFG_BOUNDS_CHECK=1) test every shared-memory and
// global index of the FFT and field kernels; an out-of-range access is
// skipped and recorded in fg_dev_error (first offending index wins).
#ifndef FG_BOUNDS_CHECK
#define FG_BOUNDS_CHECK 0
#endif

namespace fg {

// Complex numbers as float2 / double2 (8- and 16-byte aligned vector types).
template <typename T> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };
template <typename T> using cplx = typename CT<T>::type;
template <typename T> struct RT2;  // two reals packed (x even, y odd)
template <> struct RT2<float> { using type = float2; };
template <> struct RT2<double> { using type = double2; };

template <typename C> __host__ __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <typename C, bool INV> __device__ __forceinline__ C mul_mi(C a) {
  return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}

// Dynamic shared memory of a kernel, 16-byte aligned.  The host emulation
// of the kernels (tests/host_emu) defines it, and the inline-PTX helpers
// below (FG_HOST_EMU), as plain host code.
#ifndef FG_DYN_SMEM
#define FG_DYN_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#endif

#ifndef FG_HOST_EMU
// Asynchronous global -> shared copies (cp.async, sm_80+): many copies in
// flight per thread without register staging; complete with cp_async_wait().
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (BYTES == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else if (BYTES == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
#endif  // FG_HOST_EMU

// L2 eviction priority for data read once and not needed again before it is
// rewritten (a spectrum the next pass consumes, rwork read by the assembly):
// an evict_first cache policy on those loads keeps the fields that later
// kernels re-read (u, p, F) in the 126 MB L2.  The FP32 step uses it (7 us
// of 233 at 128^3); the FP64 step, whose fields are twice as large, measured
// no faster with it (459 against 457 us), so FG_L2_HINT_FP64 is 0.
#ifndef FG_L2_HINT_FP64
#define FG_L2_HINT_FP64 0
#endif
#ifndef FG_HOST_EMU
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// 16-byte cp.async with that policy
__device__ __forceinline__ void cp_async16_first(void* smem, const void* gmem, unsigned long long pol) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "l"(pol) : "memory");
}
// 8- or 16-byte loads of two reals (a complex value) and 16-byte loads of
// four floats or two doubles, with that policy
__device__ __forceinline__ float2 ld_first(const float2* a, unsigned long long pol) {
  float2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;\n" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double2 ld_first(const double2* a, unsigned long long pol) {
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_first(const float4* a, unsigned long long pol) {
  float4 v;
  asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;\n"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Programmatic dependent launch: let the next kernel of the stream be
// scheduled now, then wait until the previous kernel has completed and its
// writes are visible.  Both are no-ops for launches without the
// programmatic-serialization attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}
#endif  // FG_HOST_EMU

// Device error record (bounds checks, non-finite reductions).  The library
// is one translation unit, so this __device__ variable has one definition.
struct DevError {
  int code;  // 0 = none
  int pad;
  long long idx;
};
__device__ DevError g_fg_err;

__device__ __forceinline__ void fg_record_error(int code, long long idx) {
  if (atomicCAS(&g_fg_err.code, 0, code) == 0) g_fg_err.idx = idx;
}

}  // namespace fg
