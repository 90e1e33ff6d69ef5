// Host-side launch interface of the sm_100a SCFT kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace psb {

// One propagator step of one sweep, real-space side (see prop_kernels.cu).
enum { MODE_FIRST = 0, MODE_MID = 1, MODE_LAST = 2 };

// Mean-mode carry (FP32 sweeps).  The k = 0 coefficient of each step's
// transform is a sum over all N points; summed by the FP32 FFT its rounding is
// the same for every point and accumulates over the sweep (about 1e-6 in Q
// after 200 steps at 128^3).  With the carry the plane/row pass also sums its
// forward input (one FP64 partial per CTA in dc_out[blockIdx.x], the count
// gridDim.x in *dc_count); the x pencil pass (or the x-y pass) drops the FP32
// k = 0 coefficient, and one warp of its first CTA writes the FP64 mean
// (sum of the partials) * dc_scale (= 1/N) to dc_total; the next plane/row
// pass adds that value, rounded to T, to every point of its inverse transform
// (dc_in).  The part the rounding drops (the same at every point, so it would
// accumulate over the sweep) is kept in *dc_err and added to the next step's
// mean: what one step loses, the next one puts back (reset at the sweep's
// first step, dc_first).  The partials buffer holds at least kDcMinSlots
// slots.  nullptr: no carry (FP64 sweeps, the plugins).
constexpr int kDcMinSlots = 128;

template <typename T> struct PlaneWork {
  const T* src;       // MODE_FIRST: initial q (nullptr = ones)
  c2_t<T>* spec;      // half spectrum [nx][ny][nz/2+1]
  const T* wfac_in;   // wfac of the step being finished (nullptr = 1)
  const T* wfac_out;  // wfac of the step being started (nullptr = 1)
  T* store;           // slice receiving q (FIRST: the initial q; MID/LAST: q(s+ds))
  int* status;        // error word: bit 2 set when a bulk copy did not land in time
  int mode;
  int pad;
  const double* dc_in;  // MID/LAST: the mean-mode value added after the inverse transform
  double* dc_out;       // FIRST/MID: per-CTA FP64 sums of the forward input, [blockIdx.x]
  double* dc_count;     // FIRST/MID: CTA 0 writes the number of partials (gridDim.x)
};

// Pencil pass along a strided axis of the half spectrum.
// PENCIL_KFULL_IM and PENCIL_KSPEC exist for FP64 only (the FFT plugin).
enum {
  PENCIL_FWD = 0,
  PENCIL_INV = 1,
  PENCIL_KINV = 2,
  PENCIL_KFULL = 3,
  PENCIL_KFULL_IM = 4,
  PENCIL_KSPEC = 5
};

template <typename T> struct PencilWork {
  c2_t<T>* spec;
  const T* kx;        // PENCIL_KINV: factor along the pencil axis (1/N folded in)
  const T* kyz;       // PENCIL_KINV: factor per (y, kz) column
  const double* kfull;// PENCIL_KFULL(_IM): full real k array [nx][ny][nz] (plugin path)
  const c2_t<T>* kspec;// PENCIL_KSPEC: a second, fully transformed half spectrum (same layout)
  const double* dc_parts;  // PENCIL_KINV / x-y pass: the plane pass's dc_out (mean-mode carry)
  const double* dc_count;  // ... its number of partials
  double* dc_total;        // ... and where the FP64 mean goes
  double* dc_err;          // ... the rounding the previous step's mean lost (error feedback)
  double dc_scale;         // 1 / N
  int dc_first;            // the sweep's first step: no error to feed back
};

bool extent_supported(int n);
// The fused y-z plane kernel exists for this plane and fits in shared memory.
bool plane_fused_supported(int prec_bytes, int ny, int nz);

// Twiddle tables: tw_L[m] = exp(-2 pi i m / L); tw_zh has length nz/2, tw_z length nz.
// Kernel variants (chosen by the engine's autotuner, all verified by tests):
// bit 0: the plane pass runs the inverse-z last pass, the real-space step and
// the forward-z first pass as one shared-memory round trip; bit 1: the pencil
// pass does the same with its forward last pass, the k2 multiply and the
// inverse first pass.
// bit 2: the sweeps use the row + x-y plane design (transposed half spectrum
// S[kz][x][y]) instead of the y-z plane + x pencil design.
// bit 3: each sweep of an instance runs as its own chain of launches on its
// own stream (parallel graph branches) instead of all sweeps in lockstep in
// shared launches; single-instance engine only (kernels ignore the bit).
// bit 4: 256 x 256 y-z planes (too large for one CTA) run as one plane pass on
// a cluster of eight CTAs instead of a row pass and two y pencil passes
// (cluster_plane_supported); elsewhere the bit changes nothing.
enum {
  VARIANT_FUSE_Z = 1,
  VARIANT_FUSE_K = 2,
  VARIANT_XY = 4,
  VARIANT_SPLIT = 8,
  VARIANT_CLUSTER = 16,
  VARIANT_COUNT = 32
};
bool cluster_plane_supported(int prec_bytes, int ny, int nz);
// The cluster plane pass (ny = nz = 256): grid 8 nx x nworks, eight CTAs per
// plane.
template <typename T>
cudaError_t launch_plane_cluster(const PlaneWork<T>* d_works, int nworks, int nx, const c2_t<T>* tw_y,
                                 const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st);

// The x-y plane design exists for this grid (square x-y planes that fit in
// shared memory).
bool xy_supported(int prec_bytes, int nx, int ny, int nz);

// Row (z only) pass that stores the half spectrum transposed, S[kz][x][y].
template <typename T>
cudaError_t launch_rows_t(const PlaneWork<T>* d_works, int nworks, int nx, int ny, int nz,
                          const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st);

// x-y plane pass (one CTA per kz plane of S[kz][x][y]): FFT y, FFT x, k2,
// IFFT x, IFFT y.  tw has length nx (= ny).
template <typename T>
cudaError_t launch_xy(const PencilWork<T>* d_works, int nworks, int nx, int nzh,
                      const c2_t<T>* tw, int variant, cudaStream_t st);

template <typename T>
cudaError_t launch_plane(const PlaneWork<T>* d_works, int nworks, int nx, int ny, int nz,
                         const c2_t<T>* tw_y, const c2_t<T>* tw_zh, const c2_t<T>* tw_z,
                         int variant, cudaStream_t st);

// Row (z only) pass over nrows = nx*ny flattened rows.
template <typename T>
cudaError_t launch_rows(const PlaneWork<T>* d_works, int nworks, int nrows, int nz,
                        const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st);

// Pencils of length L along an axis of stride `inner` (elements), `outer`
// independent groups of L*inner elements; dims used only by PENCIL_KFULL.
template <typename T>
cudaError_t launch_pencil(const PencilWork<T>* d_works, int nworks, int mode, int L, int outer,
                          int inner, const c2_t<T>* tw, int nx, int ny, int nz, int variant,
                          cudaStream_t st);

}  // namespace psb
