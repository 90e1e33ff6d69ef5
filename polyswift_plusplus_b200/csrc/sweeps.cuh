// Launch sequence of a set of propagator sweeps run in lockstep.
//
// A SweepSet is the per-global-step work tables of one grid size and
// precision: all executed sweeps of one instance (engine.cu), or of every
// instance of one size class of a batch (batch.cu).  Step k launches one
// row/plane pass over plane_cnt[k] works and one spectral pass over
// pencil_cnt[k] works; works of different sweeps and instances are
// independent, so merging them only widens the launch.
#pragma once

#include <vector>

#include "field_kernels.cuh"
#include "kernels.h"

namespace psb {

// A junction start of a branched polymer in lockstep launches: the product of
// the arriving sweeps' final slices (PsBlock::combineSetJnt), written into the
// leaving sweep's start buffer between two global steps.
template <typename T> struct JunctionLaunch {
  JunctionIn<T> in;
  T* out;
  long long n;
};

template <typename T> struct SweepSet {
  int n[3] = {0, 0, 0};
  int nzh = 0;
  bool fused_plane = true;
  bool xy_ok = false;
  int kmax = -1;
  const c2_t<T>* tw_x = nullptr;
  const c2_t<T>* tw_y = nullptr;
  const c2_t<T>* tw_z = nullptr;
  const c2_t<T>* tw_zh = nullptr;
  const PlaneWork<T>* d_plane = nullptr;
  const PencilWork<T>* d_pencil = nullptr;
  const int* plane_off = nullptr;   // host arrays of kmax + 1 entries
  const int* plane_cnt = nullptr;
  const int* pencil_off = nullptr;
  const int* pencil_cnt = nullptr;
  // junction starts launched before global step k (branched polymers in lockstep)
  const JunctionLaunch<T>* junc = nullptr;
  const int* junc_off = nullptr;
  const int* junc_cnt = nullptr;
};

// The cluster plane pass exists for 256 x 256 planes (eight CTAs per plane).
template <typename T>
inline bool cluster_path(const SweepSet<T>& s, int variant) {
  return (variant & VARIANT_CLUSTER) && !s.fused_plane &&
         cluster_plane_supported((int)sizeof(T), s.n[1], s.n[2]);
}
template <typename T>
inline cudaError_t launch_plane_cluster_t(const PlaneWork<T>* w, int nw, int nx, const c2_t<T>* ty,
                                          const c2_t<T>* tzh, const c2_t<T>* tz, cudaStream_t st) {
  return launch_plane_cluster<T>(w, nw, nx, ty, tzh, tz, st);
}

template <typename T>
cudaError_t launch_sweep_set(const SweepSet<T>& s, int variant, cudaStream_t st, long long* nlaunch) {
  const int nx = s.n[0], ny = s.n[1], nz = s.n[2];
  cudaError_t e = cudaSuccess;
#define PSB_L(call)            \
  do {                         \
    e = (call);                \
    if (e != cudaSuccess) return e; \
    ++*nlaunch;                \
  } while (0)
  for (int k = 0; k <= s.kmax; ++k) {
    if (s.junc)
      for (int j = s.junc_off[k]; j < s.junc_off[k] + s.junc_cnt[k]; ++j)
        PSB_L(launch_junction<T>(s.junc[j].in, s.junc[j].n, s.junc[j].out, st));
    const PlaneWork<T>* pw = s.d_plane + s.plane_off[k];
    const int np = s.plane_cnt[k];
    const PencilWork<T>* xw = s.d_pencil + s.pencil_off[k];
    const int nxw = s.pencil_cnt[k];
    if (np == 0) continue;
    if ((variant & VARIANT_XY) && s.xy_ok) {
      PSB_L(launch_rows_t<T>(pw, np, nx, ny, nz, s.tw_zh, s.tw_z, st));
      if (nxw > 0) PSB_L(launch_xy<T>(xw, nxw, nx, s.nzh, s.tw_x, variant, st));
    } else if (s.fused_plane) {
      PSB_L(launch_plane<T>(pw, np, nx, ny, nz, s.tw_y, s.tw_zh, s.tw_z, variant, st));
      if (nxw > 0)
        PSB_L(launch_pencil<T>(xw, nxw, PENCIL_KINV, nx, 1, ny * s.nzh, s.tw_x, nx, ny, nz, variant, st));
    } else if (cluster_path(s, variant)) {
      PSB_L(launch_plane_cluster_t<T>(pw, np, nx, s.tw_y, s.tw_zh, s.tw_z, st));
      if (nxw > 0)
        PSB_L(launch_pencil<T>(xw, nxw, PENCIL_KINV, nx, 1, ny * s.nzh, s.tw_x, nx, ny, nz, variant, st));
    } else {
      PSB_L(launch_rows<T>(pw, np, nx * ny, nz, s.tw_zh, s.tw_z, st));
      if (nxw > 0) {
        if (ny > 1) PSB_L(launch_pencil<T>(xw, nxw, PENCIL_FWD, ny, nx, s.nzh, s.tw_y, nx, ny, nz, variant, st));
        PSB_L(launch_pencil<T>(xw, nxw, PENCIL_KINV, nx, 1, ny * s.nzh, s.tw_x, nx, ny, nz, variant, st));
        if (ny > 1) PSB_L(launch_pencil<T>(xw, nxw, PENCIL_INV, ny, nx, s.nzh, s.tw_y, nx, ny, nz, variant, st));
      }
    }
  }
#undef PSB_L
  return cudaSuccess;
}

// Time every kernel variant on the set's own sweeps (one warm-up and one timed
// pass each, on `st`) and return the fastest; tune_ms[v] = -1 for variants that
// do not exist for this grid.
template <typename T>
cudaError_t autotune_sweep_set(const SweepSet<T>& s, cudaStream_t st, float* tune_ms, int* best_variant) {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  float best = 1e30f;
  int best_v = 0;
  for (int v = 0; v < VARIANT_COUNT && e == cudaSuccess; ++v) {
    tune_ms[v] = -1.f;
    if ((v & VARIANT_XY) && (!s.xy_ok || (v & VARIANT_FUSE_Z))) continue;  // absent / same
    if ((v & VARIANT_CLUSTER) && (!cluster_path(s, v) || (v & VARIANT_XY))) continue;
    if (v & VARIANT_SPLIT) continue;  // a property of how an instance's sweeps are launched
    long long nl = 0;
    e = launch_sweep_set<T>(s, v, st, &nl);
    if (e == cudaSuccess) e = cudaEventRecord(a, st);
    if (e == cudaSuccess) e = launch_sweep_set<T>(s, v, st, &nl);
    if (e == cudaSuccess) e = cudaEventRecord(b, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e != cudaSuccess) break;
    tune_ms[v] = ms;
    if (ms < best) {
      best = ms;
      best_v = v;
    }
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (e == cudaSuccess) *best_variant = best_v;
  return e;
}

}  // namespace psb
