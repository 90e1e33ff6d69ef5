// Field-level kernels: Boltzmann factors, Q, contour quadrature, field updates.
//
// Everything here is FP64 except the propagator slices, which are read in the
// sweep precision T and widened before any product.  All reductions use a
// fixed grid of kRedBlocks CTAs and a fixed in-CTA tree, so results do not
// depend on scheduling (no atomics).
#include <stdint.h>
#include <math.h>

#include "field_kernels.cuh"

namespace psb {

// ---------------------------------------------------------------------------
// Reduction helpers.
// ---------------------------------------------------------------------------
template <int NQ>
__device__ __forceinline__ void block_reduce_write(double (&v)[NQ], unsigned max_mask,
                                                   double* out) {
  __shared__ double red[NQ][kRedThreads / 32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double x = v[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double y = __shfl_down_sync(0xffffffffu, x, off);
      x = ((max_mask >> q) & 1u) ? fmax(x, y) : x + y;
    }
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = (lane < kRedThreads / 32) ? red[q][lane] : (((max_mask >> q) & 1u) ? 0.0 : 0.0);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double y = __shfl_down_sync(0xffffffffu, x, off);
        x = ((max_mask >> q) & 1u) ? fmax(x, y) : x + y;
      }
      if (lane == 0) out[q] = x;
    }
  }
}

// Deterministic sum (or max) of n values by one CTA.
__device__ double cta_reduce_partials(const double* p, int n, int stride, bool is_max) {
  __shared__ double sh[kRedThreads];
  double x = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double y = p[(size_t)i * stride];
    x = is_max ? fmax(x, y) : x + y;
  }
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double a = sh[threadIdx.x], b = sh[threadIdx.x + s];
      sh[threadIdx.x] = is_max ? fmax(a, b) : a + b;
    }
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// wfac = exp(-ds/2 w)   (pspolymer/PsFlexPseudoSpec.cpp:170-177)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void wfac_kernel(const double* __restrict__ w, T* __restrict__ wfac, double ds2,
                            long long N) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    wfac[i] = (T)exp(ds2 * w[i]);
}

template <typename T>
cudaError_t launch_wfac(const double* w, T* wfac, double ds2, long long N, cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  wfac_kernel<T><<<blocks, 256, 0, st>>>(w, wfac, ds2, N);
  return cudaGetLastError();
}
template cudaError_t launch_wfac<float>(const double*, float*, double, long long, cudaStream_t);
template cudaError_t launch_wfac<double>(const double*, double*, double, long long, cudaStream_t);

template <typename T>
__global__ void junction_kernel(JunctionIn<T> in, long long N, T* __restrict__ out) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    T p = T(1);
    for (int i = 0; i < in.n; ++i) p = p * in.q[i][r];
    out[r] = p;
  }
}

template <typename T>
cudaError_t launch_junction(const JunctionIn<T>& in, long long N, T* out, cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  junction_kernel<T><<<blocks, 256, 0, st>>>(in, N, out);
  return cudaGetLastError();
}
template cudaError_t launch_junction<float>(const JunctionIn<float>&, long long, float*, cudaStream_t);
template cudaError_t launch_junction<double>(const JunctionIn<double>&, long long, double*, cudaStream_t);

__global__ void zero_kernel(double* p, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

cudaError_t launch_zero(double* p, long long n, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  zero_kernel<<<blocks, 256, 0, st>>>(p, n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Q = <qHeadInitial * qHeadFinal>  (pspolymer/PsBlock.cpp:204-237)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
    dot_partials_kernel(const T* __restrict__ a, const T* __restrict__ b, long long N,
                        double* __restrict__ partials) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < N;
       i += (long long)kRedBlocks * kRedThreads)
    v[0] += (0.0 + (double)a[i]) * (double)b[i];
  block_reduce_write<1>(v, 0u, partials + blockIdx.x);
}

template <typename T>
cudaError_t launch_dot_partials(const T* a, const T* b, long long N, double* partials,
                                cudaStream_t st) {
  dot_partials_kernel<T><<<kRedBlocks, kRedThreads, 0, st>>>(a, b, N, partials);
  return cudaGetLastError();
}
template cudaError_t launch_dot_partials<float>(const float*, const float*, long long, double*,
                                                cudaStream_t);
template cudaError_t launch_dot_partials<double>(const double*, const double*, long long, double*,
                                                 cudaStream_t);

__global__ void finalize_q_kernel(const double* partials, double N, int ip, DevScalars* sc) {
  double tot = cta_reduce_partials(partials, kRedBlocks, 1, false);
  if (threadIdx.x == 0) {
    double q = tot / (1.0 * N);
    sc->q[ip] = q;
    sc->log_q[ip] = log(q);
    if (q != q) sc->error_flags |= 1;
  }
}

cudaError_t launch_finalize_q(const double* partials, double N, int ip, DevScalars* sc,
                              cudaStream_t st) {
  finalize_q_kernel<<<1, kRedThreads, 0, st>>>(partials, N, ip, sc);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// simpleSolvent: wFactor = exp(-w / L), Q = sum(wFactor) / N, phi += (vf / Q) wFactor
// (pssolvent/PsSimpleSolvent.cpp:86-140).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double solvent_factor(double w, double neg_inv_len) {
  double v = 0.0 + w;
  v = v * neg_inv_len;
  return exp(v);
}

__global__ void solvent_partials_kernel(const double* __restrict__ w, double neg_inv_len, long long N,
                                        double* __restrict__ partials) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < N;
       i += (long long)kRedBlocks * kRedThreads)
    v[0] += solvent_factor(w[i], neg_inv_len);
  block_reduce_write<1>(v, 0u, partials + blockIdx.x);
}

__global__ void solvent_finalize_kernel(const double* partials, double N, int is, DevScalars* sc) {
  const double tot = cta_reduce_partials(partials, kRedBlocks, 1, false);
  if (threadIdx.x == 0) {
    const double q = tot / (1.0 * N);
    sc->solv_q[is] = q;
    if (q != q) sc->error_flags |= 1;
  }
}

__global__ void solvent_density_kernel(const double* __restrict__ w, double neg_inv_len, double volfrac,
                                       long long N, int is, const DevScalars* __restrict__ sc,
                                       double* __restrict__ phi) {
  const double f = volfrac / sc->solv_q[is];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x)
    phi[r] = phi[r] + solvent_factor(w[r], neg_inv_len) * f;
}

cudaError_t launch_solvent(const double* w, double neg_inv_len, double volfrac, long long N, int is,
                           double* partials, DevScalars* sc, double* phi, cudaStream_t st) {
  solvent_partials_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, neg_inv_len, N, partials);
  solvent_finalize_kernel<<<1, kRedThreads, 0, st>>>(partials, (double)N, is, sc);
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  solvent_density_kernel<<<blocks, 256, 0, st>>>(w, neg_inv_len, volfrac, N, is, sc, phi);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// chargeFlexPseudoSpec Boltzmann factor (pspolymer/PsChargeFlexPseudoSpec.cpp:97-130):
// wfac = exp(ds2 w) exp(facZ ds2 psi), facZ = za alpha L.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void wfac_charged_kernel(const double* __restrict__ w, const double* __restrict__ psi,
                                    T* __restrict__ wfac, double ds2, double facz, long long N) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    wfac[i] = (T)(exp(ds2 * w[i]) * exp(facz * ds2 * psi[i]));
}

template <typename T>
cudaError_t launch_wfac_charged(const double* w, const double* psi, T* wfac, double ds2, double facz,
                                long long N, cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  wfac_charged_kernel<T><<<blocks, 256, 0, st>>>(w, psi, wfac, ds2, facz, N);
  return cudaGetLastError();
}
template cudaError_t launch_wfac_charged<float>(const double*, const double*, float*, double, double,
                                                long long, cudaStream_t);
template cudaError_t launch_wfac_charged<double>(const double*, const double*, double*, double, double,
                                                 long long, cudaStream_t);

// ---------------------------------------------------------------------------
// simpleIons (pssolvent/PsSimpleIons.cpp:90-160): e = exp(-zc psi),
// Q = sum(e) / N, e *= -neutralFactor / (Q zc); blockfield = e; rho += zc e.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ion_factor(double psi, double negfac) {
  double v = 0.0 + psi;
  v = v * negfac;
  return exp(v);
}

__global__ void ions_partials_kernel(const double* __restrict__ psi, double negfac, long long N,
                                     double* __restrict__ partials) {
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < N;
       i += (long long)kRedBlocks * kRedThreads)
    v[0] += ion_factor(psi[i], negfac);
  block_reduce_write<1>(v, 0u, partials + blockIdx.x);
}

__global__ void ions_density_kernel(const double* __restrict__ psi, double zc, double neutral_factor,
                                    long long N, int is, const DevScalars* __restrict__ sc,
                                    double* __restrict__ rho, double* __restrict__ block_rho) {
  const double cfac = -neutral_factor / (sc->solv_q[is] * zc);
  const double negfac = -1.0 * zc;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    const double e = ion_factor(psi[r], negfac) * cfac;
    if (block_rho) block_rho[r] = 0.0 + e;
    rho[r] = rho[r] + e * zc;
  }
}

cudaError_t launch_ions(const double* psi, double zc, double neutral_factor, long long N, int is,
                        double* partials, DevScalars* sc, double* rho, double* block_rho,
                        cudaStream_t st) {
  ions_partials_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(psi, -1.0 * zc, N, partials);
  solvent_finalize_kernel<<<1, kRedThreads, 0, st>>>(partials, (double)N, is, sc);
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  ions_density_kernel<<<blocks, 256, 0, st>>>(psi, zc, neutral_factor, N, is, sc, rho, block_rho);
  return cudaGetLastError();
}

// rho += (phi alpha) za   (pspolymer/PsChargeFlexPseudoSpec.cpp:136-165)
__global__ void charge_accum_kernel(const double* __restrict__ phi, double alpha, double za, long long N,
                                    double* __restrict__ rho) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    double t = 0.0 + phi[r];
    t = t * alpha;
    t = t * za;
    rho[r] = rho[r] + t;
  }
}

cudaError_t launch_charge_accum(const double* phi, double alpha, double za, long long N, double* rho,
                                cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  charge_accum_kernel<<<blocks, 256, 0, st>>>(phi, alpha, za, N, rho);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Contour quadrature (pspolymer/PsBlock.cpp:255-380) and density update
// (pspolymer/PsBlock.cpp:153-196): extended Simpson with the reference's
// 0.33333 factor, trapezoid on the last interval for an even point count.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void quadrature_kernel(const T* __restrict__ qs, const T* __restrict__ qts, int steps,
                                  long long N, double simp, double trap, double densfac,
                                  const DevScalars* __restrict__ sc, int ip,
                                  double* __restrict__ phi) {
  const long long num = steps + 1;
  const long long npts = num - 1;
  const bool even = (num % 2) == 0;
  const long long numstail = even ? npts - 3 : npts - 2;
  const double inv_bq = 1.0 / sc->q[ip];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
#pragma unroll 2
    for (long long n = 0; n <= numstail; n += 2) {
      double p1 = (double)qs[n * N + r] * (double)qts[(num - n - 1) * N + r];
      double p2 = (double)qs[(n + 1) * N + r] * (double)qts[(num - n - 2) * N + r];
      double p3 = (double)qs[(n + 2) * N + r] * (double)qts[(num - n - 3) * N + r];
      p2 = p2 * 4.0;
      acc = acc + p1;
      acc = acc + p2;
      acc = acc + p3;
    }
    acc = acc * simp;
    if (even) {
      double p1 = (double)qs[(num - 2) * N + r] * (double)qts[1 * N + r];
      double p2 = (double)qs[(num - 1) * N + r] * (double)qts[r];
      double t = 0.0;
      t = t + p1;
      t = t + p2;
      t = t * trap;
      acc = acc + t;
    }
    double qqt = inv_bq * acc;
    double v = densfac * qqt;
    phi[r] = phi[r] + v;
  }
}

// FP32 slices with N % 4 == 0: four points per thread with 16-byte loads, the
// same arithmetic per point as quadrature_kernel (bitwise the same result).
__global__ void quadrature4_kernel(const float4* __restrict__ qs, const float4* __restrict__ qts, int steps,
                                   long long N4, double simp, double trap, double densfac,
                                   const DevScalars* __restrict__ sc, int ip, double2* __restrict__ phi) {
  const long long num = steps + 1;
  const long long npts = num - 1;
  const bool even = (num % 2) == 0;
  const long long numstail = even ? npts - 3 : npts - 2;
  const double inv_bq = 1.0 / sc->q[ip];
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N4;
       r += (long long)gridDim.x * blockDim.x) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 2
    for (long long n = 0; n <= numstail; n += 2) {
      const float4 a1 = qs[n * N4 + r], b1 = qts[(num - n - 1) * N4 + r];
      const float4 a2 = qs[(n + 1) * N4 + r], b2 = qts[(num - n - 2) * N4 + r];
      const float4 a3 = qs[(n + 2) * N4 + r], b3 = qts[(num - n - 3) * N4 + r];
      const float x1[4] = {a1.x, a1.y, a1.z, a1.w}, y1[4] = {b1.x, b1.y, b1.z, b1.w};
      const float x2[4] = {a2.x, a2.y, a2.z, a2.w}, y2[4] = {b2.x, b2.y, b2.z, b2.w};
      const float x3[4] = {a3.x, a3.y, a3.z, a3.w}, y3[4] = {b3.x, b3.y, b3.z, b3.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double p1 = (double)x1[c] * (double)y1[c];
        double p2 = (double)x2[c] * (double)y2[c];
        double p3 = (double)x3[c] * (double)y3[c];
        p2 = p2 * 4.0;
        acc[c] = acc[c] + p1;
        acc[c] = acc[c] + p2;
        acc[c] = acc[c] + p3;
      }
    }
    double tail[4] = {0.0, 0.0, 0.0, 0.0};
    if (even) {
      const float4 a1 = qs[(num - 2) * N4 + r], b1 = qts[1 * N4 + r];
      const float4 a2 = qs[(num - 1) * N4 + r], b2 = qts[r];
      const float x1[4] = {a1.x, a1.y, a1.z, a1.w}, y1[4] = {b1.x, b1.y, b1.z, b1.w};
      const float x2[4] = {a2.x, a2.y, a2.z, a2.w}, y2[4] = {b2.x, b2.y, b2.z, b2.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double p1 = (double)x1[c] * (double)y1[c];
        double p2 = (double)x2[c] * (double)y2[c];
        double t = 0.0;
        t = t + p1;
        t = t + p2;
        tail[c] = t * trap;
      }
    }
    double v[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double a = acc[c] * simp;
      if (even) a = a + tail[c];
      const double qqt = inv_bq * a;
      v[c] = densfac * qqt;
    }
    const double2 f0 = phi[2 * r], f1 = phi[2 * r + 1];
    phi[2 * r] = make_double2(f0.x + v[0], f0.y + v[1]);
    phi[2 * r + 1] = make_double2(f1.x + v[2], f1.y + v[3]);
  }
}

template <typename T>
cudaError_t launch_quadrature(const T* qs, const T* qts, int steps, long long N, double ds,
                              double densfac, const DevScalars* sc, int ip, double* phi,
                              cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  const double simp = 0.33333 * ds;
  const double trap = ds * 0.5;
  if (sizeof(T) == 4 && N % 4 == 0 && ((uintptr_t)qs % 16) == 0 && ((uintptr_t)qts % 16) == 0 &&
      ((uintptr_t)phi % 16) == 0) {
    const long long N4 = N / 4;
    int b4 = (int)((N4 + 255) / 256);
    if (b4 > 148 * 8) b4 = 148 * 8;
    quadrature4_kernel<<<b4, 256, 0, st>>>(reinterpret_cast<const float4*>(qs),
                                           reinterpret_cast<const float4*>(qts), steps, N4, simp, trap,
                                           densfac, sc, ip, reinterpret_cast<double2*>(phi));
    return cudaGetLastError();
  }
  quadrature_kernel<T><<<blocks, 256, 0, st>>>(qs, qts, steps, N, simp, trap, densfac, sc, ip, phi);
  return cudaGetLastError();
}
template cudaError_t launch_quadrature<float>(const float*, const float*, int, long long, double,
                                              double, const DevScalars*, int, double*, cudaStream_t);
template cudaError_t launch_quadrature<double>(const double*, const double*, int, long long, double,
                                               double, const DevScalars*, int, double*,
                                               cudaStream_t);

// ---------------------------------------------------------------------------
// Field update pieces shared by the steepest-descent and Anderson updaters.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool int_has(const FieldModel& fm, int it, int f) {
  return fm.int_a[it] == f || fm.int_b[it] == f;
}

// Per-point field arrays of NF (2 or 3) entries stay in registers: loops over
// fields are unrolled, and an entry picked by a runtime field index goes
// through pick().  The arithmetic and its order are those of the reference.
template <int NF>
__device__ __forceinline__ double pick(const double (&a)[NF], int i) {
  double v = a[0];
#pragma unroll
  for (int q = 1; q < NF; ++q)
    if (i == q) v = a[q];
  return v;
}

// dH_i = p - w_i + sum_{int ∋ i} chiN (phi_other - avg_other)
// (pseffhamil/PsSteepDUpdater.cpp:174-184, :208-236; pseffhamil/PsFloryInteraction.cpp:204-269)
template <int NF>
__device__ __forceinline__ void compute_dh(const FieldModel& fm, const FieldPtrs& fp, long long r,
                                           double (&dh)[NF], double (&phi_r)[NF]) {
  const double pr = fp.p[r];
#pragma unroll
  for (int i = 0; i < NF; ++i) phi_r[i] = fp.phi[i][r];
#pragma unroll
  for (int i = 0; i < NF; ++i) {
    double d = 0.0;
    d = d + pr;
    d = d - fp.w[i][r];
    for (int it = 0; it < fm.n_int; ++it) {
      if (!int_has(fm, it, i)) continue;
      const int other = (i == fm.int_a[it]) ? fm.int_b[it] : fm.int_a[it];
      const double mask = -1.0 * fm.dens_avg[other];
      double x = 0.0;
      x = x + pick(phi_r, other);
      x = x + mask;
      x = x * fm.chin[it];
      d = d + x;
    }
    dh[i] = d;
  }
}

// SD direction: dH_i - lambda1 * sum_{j != i} dH_j (pseffhamil/PsSteepDUpdater.cpp:264-278, :368-393)
template <int NF>
__device__ __forceinline__ void sd_direction(const FieldModel& fm, const double (&dh)[NF], double (&dir)[NF]) {
#pragma unroll
  for (int i = 0; i < NF; ++i) {
    double x = 0.0;
#pragma unroll
    for (int j = 0; j < NF; ++j)
      if (j != i) x = x + dh[j];
    x = x * (-1.0 * fm.lambda1);
    x = x + dh[i];
    dir[i] = x;
  }
}

// Noise, pressure rebuild (pseffhamil/PsSteepDUpdater.cpp:283-332, :398-452) and
// the free-energy density (pseffhamil/PsPolymerUpdater.cpp:172-226, 302-341;
// pseffhamil/PsFloryInteraction.cpp:274-321) at one point, given the new w.
template <int NF>
__device__ __forceinline__ void finish_point(const FieldModel& fm, const FieldPtrs& fp,
                                             long long r, double (&wn)[NF], const double (&phi_r)[NF],
                                             double& psum, double& fe, double& fe_nd) {
  if (fp.noise) {
#pragma unroll
    for (int i = 0; i < NF; ++i) {
      double v = 0.0 + fp.noise[(size_t)i * fm.N + r];
      v = v * 1.0;
      wn[i] = wn[i] + v;
    }
  }
#pragma unroll
  for (int i = 0; i < NF; ++i) fp.w[i][r] = wn[i];
  double pr = 0.0;
#pragma unroll
  for (int i = 0; i < NF; ++i) pr = pr + wn[i];
  if (NF == 2) {
    for (int it = 0; it < fm.n_int; ++it) {
      if (int_has(fm, it, 0) && int_has(fm, it, 1)) {
        double x = 0.0;
        x = x * fm.chin[it];
        pr = pr + x;
      }
    }
    pr = 0.5 * pr;
  } else {
    for (int it = 0; it < fm.n_int; ++it) {
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        if (int_has(fm, it, n)) continue;
        double x = 0.0;
        x = x + (phi_r[n] - fm.dens_avg[n]);
        x = x + 0.0;
        x = x * fm.chin[it];
        pr = pr + x;
      }
    }
    const double inv = 1.0 / 3.0;
    pr = inv * pr;
  }
  fp.p[r] = pr;
  psum += pr;
  const double inv_vol = 1.0 / (double)fm.N;
  double f = 0.0;
#pragma unroll
  for (int i = 0; i < NF; ++i) {
    double prod = (0.0 + phi_r[i]) * wn[i];
    prod = -1.0 * prod;
    f = f + prod;
  }
  f = f * 1.0;
  f = inv_vol * f;
  double ft = 0.0 + f, ftn = 0.0 + f;
  for (int it = 0; it < fm.n_int; ++it) {
    const double a0 = fm.dens_avg[fm.int_a[it]], a1 = fm.dens_avg[fm.int_b[it]];
    double dis = (((0.0 + 1.0) * 1.0) * a0) * a1;
    dis = dis * fm.chin[it];
    double v = (0.0 + pick(phi_r, fm.int_a[it])) * pick(phi_r, fm.int_b[it]);
    v = v * fm.chin[it];
    const double vd = v - dis;
    ft = ft + inv_vol * vd;
    ftn = ftn + inv_vol * v;
  }
  fe += ft;
  fe_nd += ftn;
}

template <int NF>
__device__ __forceinline__ double incomp(const double (&phi_r)[NF]) {
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < NF; ++i) t += phi_r[i];
  return fabs(t - 1.0);
}

template <int NF>
__global__ void __launch_bounds__(kRedThreads)
    sd_update_kernel(FieldModel fm, FieldPtrs fp, double* __restrict__ partials) {
  double acc[kUpdQ] = {0, 0, 0, 0, 0, 0};
  for (long long r = blockIdx.x * (long long)kRedThreads + threadIdx.x; r < fm.N;
       r += (long long)kRedBlocks * kRedThreads) {
    double dh[NF], phi_r[NF], dir[NF], wn[NF];
    compute_dh<NF>(fm, fp, r, dh, phi_r);
#pragma unroll
    for (int i = 0; i < NF; ++i) acc[3] += dh[i] * dh[i];
    acc[4] = fmax(acc[4], incomp<NF>(phi_r));
    sd_direction<NF>(fm, dh, dir);
#pragma unroll
    for (int i = 0; i < NF; ++i) {
      const double x = dir[i] * fm.lambda0;
      wn[i] = fp.w[i][r] + x;
    }
    finish_point<NF>(fm, fp, r, wn, phi_r, acc[0], acc[1], acc[2]);
  }
  block_reduce_write<kUpdQ>(acc, 1u << 4, partials + (size_t)blockIdx.x * kUpdQ);
}

cudaError_t launch_sd_update(const FieldModel& fm, const FieldPtrs& fp, double* partials,
                             cudaStream_t st) {
  if (fm.nf == 3)
    sd_update_kernel<3><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, partials);
  else
    sd_update_kernel<2><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, partials);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Anderson mixing (no reference counterpart): history of (w, D) with
// D = steepest-descent direction; Gram-matrix normal equations in FP64.
// ---------------------------------------------------------------------------
template <int NF>
__global__ void __launch_bounds__(kRedThreads)
    am_residual_kernel(FieldModel fm, FieldPtrs fp, double* __restrict__ hist_w,
                       double* __restrict__ hist_d, int slots, const DevScalars* __restrict__ sc,
                       double* __restrict__ partials) {
  const int cur = (int)(sc->am_k % slots);
  const size_t nfN = (size_t)fm.nf * fm.N;
  double* Wc = hist_w + (size_t)cur * nfN;
  double* Dc = hist_d + (size_t)cur * nfN;
  double acc[2] = {0.0, 0.0};
  for (long long r = blockIdx.x * (long long)kRedThreads + threadIdx.x; r < fm.N;
       r += (long long)kRedBlocks * kRedThreads) {
    double dh[NF], phi_r[NF], dir[NF];
    compute_dh<NF>(fm, fp, r, dh, phi_r);
#pragma unroll
    for (int i = 0; i < NF; ++i) acc[0] += dh[i] * dh[i];
    acc[1] = fmax(acc[1], incomp<NF>(phi_r));
    sd_direction<NF>(fm, dh, dir);
#pragma unroll
    for (int i = 0; i < NF; ++i) {
      Wc[(size_t)i * fm.N + r] = fp.w[i][r];
      Dc[(size_t)i * fm.N + r] = dir[i];
    }
  }
  double out[2];
  block_reduce_write<2>(acc, 2u, out);
  if (threadIdx.x == 0) {
    partials[(size_t)blockIdx.x * kUpdQ + 3] = out[0];
    partials[(size_t)blockIdx.x * kUpdQ + 4] = out[1];
  }
}

cudaError_t launch_am_residual(const FieldModel& fm, const FieldPtrs& fp, double* hist_w,
                               double* hist_d, int slots, DevScalars* sc, double* partials,
                               cudaStream_t st) {
  if (fm.nf == 3)
    am_residual_kernel<3><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, hist_w, hist_d, slots, sc, partials);
  else
    am_residual_kernel<2><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, hist_w, hist_d, slots, sc, partials);
  return cudaGetLastError();
}

constexpr int kAmMax = 33;  // depth <= 32

// MAXJ >= m + 1 accumulators: a small depth keeps them in few registers (more
// blocks per SM); each Gram entry's sum and reduction tree do not depend on MAXJ.
template <int MAXJ>
__global__ void __launch_bounds__(kRedThreads)
    am_gram_kernel(long long nfN, const double* __restrict__ hist_d, int slots, int m,
                   const DevScalars* __restrict__ sc, double* __restrict__ gram_partials) {
  const long long k = sc->am_k;
  const int nh = (int)(k < m ? k : m);
  const int cur = (int)(k % slots);
  const double* Dc = hist_d + (size_t)cur * nfN;
  __shared__ const double* Dj[MAXJ];
  if (threadIdx.x < MAXJ) {
    const int j = threadIdx.x;
    Dj[j] = hist_d + (size_t)((k - (j <= nh ? j : 0)) % slots) * nfN;
  }
  __syncthreads();
  double acc[MAXJ];
#pragma unroll
  for (int j = 0; j < MAXJ; ++j) acc[j] = 0.0;
  for (long long t = blockIdx.x * (long long)kRedThreads + threadIdx.x; t < nfN;
       t += (long long)kRedBlocks * kRedThreads) {
    const double d = Dc[t];
#pragma unroll
    for (int j = 0; j < MAXJ; ++j)
      if (j <= nh) acc[j] += d * Dj[j][t];
  }
  block_reduce_write<MAXJ>(acc, 0u, gram_partials + (size_t)blockIdx.x * kAmMax);
}

cudaError_t launch_am_gram(long long nfN, const double* hist_d, int slots, int m, DevScalars* sc,
                           double* gram_partials, cudaStream_t st) {
  if (m + 1 > kAmMax) return cudaErrorInvalidValue;
  if (m + 1 <= 8)
    am_gram_kernel<8><<<kRedBlocks, kRedThreads, 0, st>>>(nfN, hist_d, slots, m, sc, gram_partials);
  else if (m + 1 <= 12)
    am_gram_kernel<12><<<kRedBlocks, kRedThreads, 0, st>>>(nfN, hist_d, slots, m, sc, gram_partials);
  else if (m + 1 <= 16)
    am_gram_kernel<16><<<kRedBlocks, kRedThreads, 0, st>>>(nfN, hist_d, slots, m, sc, gram_partials);
  else
    am_gram_kernel<kAmMax><<<kRedBlocks, kRedThreads, 0, st>>>(nfN, hist_d, slots, m, sc, gram_partials);
  return cudaGetLastError();
}

// One CTA: finish the Gram row, build U c = V and solve it (partial pivoting,
// the same elimination order as the oracle's restatement).
__global__ void am_solve_kernel(const double* __restrict__ gram_partials, double* __restrict__ gram,
                                int slots, int m, int start, double mix, double lambda0,
                                DevScalars* __restrict__ sc) {
  __shared__ double A[32 * 32];
  __shared__ double V[32];
  __shared__ double row[kAmMax];
  const long long k = sc->am_k;
  const int nh_all = (int)(k < m ? k : m);
  const int cur = (int)(k % slots);
  for (int j = 0; j <= nh_all; ++j) {
    double g = cta_reduce_partials(gram_partials + j, kRedBlocks, kAmMax, false);
    if (threadIdx.x == 0) row[j] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 0; j <= nh_all; ++j) {
      const int sj = (int)((k - j) % slots);
      gram[cur * slots + sj] = row[j];
      gram[sj * slots + cur] = row[j];
    }
    const int use = (k >= start) && nh_all > 0;
    int nh = use ? nh_all : 0;
    if (use) {
      const double gkk = gram[cur * slots + cur];
      for (int a = 1; a <= nh; ++a) {
        const int sa = (int)((k - a) % slots);
        V[a - 1] = gkk - gram[cur * slots + sa];
        for (int b = 1; b <= nh; ++b) {
          const int sb = (int)((k - b) % slots);
          A[(a - 1) * nh + (b - 1)] =
              gkk - gram[cur * slots + sa] - gram[cur * slots + sb] + gram[sa * slots + sb];
        }
      }
      int singular = 0;
      for (int kk = 0; kk < nh && !singular; ++kk) {
        int piv = kk;
        double best = fabs(A[kk * nh + kk]);
        for (int i = kk + 1; i < nh; ++i)
          if (fabs(A[i * nh + kk]) > best) { best = fabs(A[i * nh + kk]); piv = i; }
        if (!(best > 0.0)) { singular = 1; break; }
        if (piv != kk) {
          for (int j = 0; j < nh; ++j) {
            double t = A[kk * nh + j]; A[kk * nh + j] = A[piv * nh + j]; A[piv * nh + j] = t;
          }
          double t = V[kk]; V[kk] = V[piv]; V[piv] = t;
        }
        for (int i = kk + 1; i < nh; ++i) {
          double f = A[i * nh + kk] / A[kk * nh + kk];
          for (int j = kk; j < nh; ++j) A[i * nh + j] = A[i * nh + j] - f * A[kk * nh + j];
          V[i] = V[i] - f * V[kk];
        }
      }
      if (!singular) {
        for (int i = nh - 1; i >= 0; --i) {
          double t = V[i];
          for (int j = i + 1; j < nh; ++j) t = t - A[i * nh + j] * V[j];
          V[i] = t / A[i * nh + i];
        }
      }
      for (int a = 0; a < nh; ++a) sc->am_c[a] = singular ? 0.0 : V[a];
    }
    sc->am_nh = nh;
    sc->am_use = use;
    sc->am_mix = use ? mix : lambda0;
  }
}

cudaError_t launch_am_solve(const double* gram_partials, double* gram, int slots, int m, int start,
                            double mix, double lambda0, DevScalars* sc, cudaStream_t st) {
  if (m > 32) return cudaErrorInvalidValue;
  am_solve_kernel<<<1, kRedThreads, 0, st>>>(gram_partials, gram, slots, m, start, mix, lambda0, sc);
  return cudaGetLastError();
}

template <int NF>
__global__ void __launch_bounds__(kRedThreads)
    am_mix_kernel(FieldModel fm, FieldPtrs fp, const double* __restrict__ hist_w,
                  const double* __restrict__ hist_d, int slots, const DevScalars* __restrict__ sc,
                  double* __restrict__ partials) {
  const long long k = sc->am_k;
  const int cur = (int)(k % slots);
  const int nh = sc->am_nh;
  const double mix = sc->am_mix;
  const size_t nfN = (size_t)fm.nf * fm.N;
  double acc[3] = {0.0, 0.0, 0.0};
  for (long long r = blockIdx.x * (long long)kRedThreads + threadIdx.x; r < fm.N;
       r += (long long)kRedBlocks * kRedThreads) {
    double wn[NF], phi_r[NF];
#pragma unroll
    for (int i = 0; i < NF; ++i) phi_r[i] = fp.phi[i][r];
#pragma unroll
    for (int i = 0; i < NF; ++i) {
      const size_t off = (size_t)i * fm.N + r;
      const double wk = hist_w[(size_t)cur * nfN + off];
      const double dk = hist_d[(size_t)cur * nfN + off];
      double wh = wk, dhh = dk;
      // history terms four at a time: all eight loads in flight before the
      // (unchanged, sequential) accumulation
      for (int a0 = 1; a0 <= nh; a0 += 4) {
        double hw[4], hd[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int a = a0 + j;
          if (a <= nh) {
            const size_t sa = (size_t)((k - a) % slots);
            hw[j] = hist_w[sa * nfN + off];
            hd[j] = hist_d[sa * nfN + off];
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int a = a0 + j;
          if (a <= nh) {
            const double ca = sc->am_c[a - 1];
            wh = wh + ca * (hw[j] - wk);
            dhh = dhh + ca * (hd[j] - dk);
          }
        }
      }
      wn[i] = wh + mix * dhh;
    }
    finish_point<NF>(fm, fp, r, wn, phi_r, acc[0], acc[1], acc[2]);
  }
  double out[3];
  block_reduce_write<3>(acc, 0u, out);
  if (threadIdx.x == 0) {
    for (int q = 0; q < 3; ++q) partials[(size_t)blockIdx.x * kUpdQ + q] = out[q];
  }
}

cudaError_t launch_am_mix(const FieldModel& fm, const FieldPtrs& fp, const double* hist_w,
                          const double* hist_d, int slots, DevScalars* sc, double* partials,
                          cudaStream_t st) {
  if (fm.nf == 3)
    am_mix_kernel<3><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, hist_w, hist_d, slots, sc, partials);
  else
    am_mix_kernel<2><<<kRedBlocks, kRedThreads, 0, st>>>(fm, fp, hist_w, hist_d, slots, sc, partials);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Finalisation: mean pressure, F, diagnostics.
// ---------------------------------------------------------------------------
__global__ void update_finalize_kernel(FieldModel fm, const double* __restrict__ partials,
                                       DevScalars* __restrict__ sc, int anderson) {
  const double psum = cta_reduce_partials(partials + 0, kRedBlocks, kUpdQ, false);
  const double fe = cta_reduce_partials(partials + 1, kRedBlocks, kUpdQ, false);
  const double fend = cta_reduce_partials(partials + 2, kRedBlocks, kUpdQ, false);
  const double dh2 = cta_reduce_partials(partials + 3, kRedBlocks, kUpdQ, false);
  const double mx = cta_reduce_partials(partials + 4, kRedBlocks, kUpdQ, true);
  if (threadIdx.x == 0) {
    double sum_tmp = 0.0;
    for (int ip = 0; ip < fm.npol; ++ip) {
      const double logq = sc->log_q[ip];
      sum_tmp = sum_tmp - ((fm.vf[ip] * logq) / fm.alpha[ip]);
    }
    for (int is = 0; is < fm.nsolv; ++is) {
      const double logq = log(sc->solv_q[is]);
      sum_tmp = sum_tmp - ((fm.solv_vf[is] * logq) / (1.0 / fm.scale_len));
    }
    sc->pressure_mean = psum / ((double)fm.N * 1.0);
    sc->free_energy = sum_tmp + fe;
    sc->free_energy_nodis = sum_tmp + fend;
    sc->dh_norm = sqrt(dh2 / (double)fm.N);
    sc->max_incomp = mx;
    if (!(sc->free_energy == sc->free_energy)) sc->error_flags |= 2;
    sc->iteration += 1;
    if (anderson) sc->am_k += 1;
  }
}

cudaError_t launch_update_finalize(const FieldModel& fm, const double* partials, DevScalars* sc,
                                   cudaStream_t st) {
  update_finalize_kernel<<<1, kRedThreads, 0, st>>>(fm, partials, sc, 0);
  return cudaGetLastError();
}

cudaError_t launch_update_finalize_am(const FieldModel& fm, const double* partials, DevScalars* sc,
                                      cudaStream_t st) {
  update_finalize_kernel<<<1, kRedThreads, 0, st>>>(fm, partials, sc, 1);
  return cudaGetLastError();
}

__global__ void pressure_shift_kernel(double* __restrict__ p, long long N,
                                      const DevScalars* __restrict__ sc) {
  const double mean = sc->pressure_mean;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = p[i] - mean;
}

cudaError_t launch_pressure_shift(double* p, long long N, const DevScalars* sc, cudaStream_t st) {
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  pressure_shift_kernel<<<blocks, 256, 0, st>>>(p, N, sc);
  return cudaGetLastError();
}

}  // namespace psb
