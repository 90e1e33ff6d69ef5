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

}  // namespace psb
