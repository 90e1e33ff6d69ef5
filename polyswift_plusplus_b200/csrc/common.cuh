// Shared types and helpers for the sm_100a SCFT kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace psb {

template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using c2_t = typename C2<T>::type;

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return {a.x + b.x, a.y + b.y}; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return {a.x - b.x, a.y - b.y}; }

#if !defined(PSB_SCALAR_F32)
#define PSB_PACKED_F32X2 1
#endif
#if defined(PSB_PACKED_F32X2)
// FP32 complex add / subtract as one packed two-lane instruction (sm_100
// f32x2 arithmetic, round to nearest: the same result as two scalar ops).
template <>
__device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <>
__device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
#endif
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename C>
__device__ __forceinline__ C cmulc(C a, C b) {
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename C, typename S>
__device__ __forceinline__ C cscale(C a, S s) { return {a.x * s, a.y * s}; }

// Multiply by -i (forward) or +i (inverse).
template <bool INV, typename C>
__device__ __forceinline__ C mul_mi(C a) {
  if (INV) return {-a.y, a.x};
  return {a.y, -a.x};
}

// Programmatic dependent launch (sm_90+).  A sweep kernel launched with the
// programmatic-serialisation attribute may be launched before the kernel ahead
// of it on the stream has finished: it does its independent prologue (twiddle
// tables, work descriptors), then pdl_wait() blocks until that kernel has
// completed and its writes are visible; without the attribute pdl_wait() is a
// no-op.  No kernel triggers its dependents early: blocks of the next sweep
// kernel parked on pdl_wait() hold shared memory and registers that the
// concurrent sweep's kernels need.  At 128^3 a trigger after the loads was 4%
// slower, and a late one (plane pass after its real-space step, pencil pass
// after its k^2 pass) 2-3% slower, although it cut the time from the last
// block's exit to the next kernel's release from about 2.5 to 1.6 us.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace psb
