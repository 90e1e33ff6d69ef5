// Propagator-step kernels for sm_100a.
//
// One step of PsFlexPseudoSpec::solveQ (pspolymer/PsFlexPseudoSpec.cpp:267-289)
//     q(s+ds) = wfac * Re(IFFT(k2 * FFT(wfac * q(s)))) / N
// is split into two passes over a half spectrum S[x][y][kz] (kz <= nz/2) that
// stays resident in L2 between passes:
//   plane pass  (one CTA per x-plane, whole y-z plane in shared memory):
//       inverse y FFT -> inverse z c2r -> q = a*wfac_in -> store q(s+ds)
//       -> a = q*wfac_out -> forward z r2c -> forward y FFT
//     i.e. the end of step s and the start of step s+1 fused in one launch;
//   pencil pass (TK adjacent (y,kz) columns per CTA): forward x FFT,
//       multiply by exp(-ds b^2 k^2)/N from separable 1D tables, inverse x FFT.
// When a plane does not fit in shared memory the plane pass becomes a row pass
// (z only) plus y pencil passes.  Real <-> half-spectrum transforms use the
// half-length complex FFT of the even/odd samples with an in-place pairwise
// post-/pre-processing step (k with h-k of the same row).
#include <cstdio>

#include "fft_smem.cuh"
#include "kernels.h"

namespace psb {

template <typename T>
__device__ __forceinline__ T ld_or_one(const T* p, size_t i) {
  return p ? __ldg(p + i) : T(1);
}

// Forward post-processing of one row: slots hold C = FFT_h(a_even + i a_odd),
// rewritten in place to the half spectrum A[0..h] (slot h = Nyquist).
template <int NZ, int ROWS, int TH, typename C>
__device__ __forceinline__ void r2c_post(C* buf, const C* twn, int rows) {
  constexpr int H = NZ / 2;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int KP = H / 2 + 1;  // pairs (k, h-k), k = 0..h/2
  using S = decltype(buf[0].x);
  for (int e = threadIdx.x; e < ROWS * KP; e += TH) {
    const int r = e / KP;
    const int k = e - r * KP;
    if (r >= rows) continue;
    C* row = buf + r * NZH;
    const int km = (H - k) % H;
    const C c = row[k];
    const C d = row[km];
    // E = (C[k] + conj(C[km]))/2 ; O = -i (C[k] - conj(C[km]))/2
    const C E = {S(0.5) * (c.x + d.x), S(0.5) * (c.y - d.y)};
    const C O = {S(0.5) * (c.y + d.y), S(0.5) * (d.x - c.x)};
    const C wo = cmul(twn[k], O);
    row[k] = cadd(E, wo);
    const C m = csub(E, wo);
    row[H - k] = {m.x, -m.y};
  }
}

// Inverse pre-processing: half spectrum A[0..h] -> C' with IFFT_h(C') = a_even + i a_odd.
template <int NZ, int ROWS, int TH, typename C>
__device__ __forceinline__ void c2r_pre(C* buf, const C* twn, int rows) {
  constexpr int H = NZ / 2;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int KP = H / 2 + 1;
  for (int e = threadIdx.x; e < ROWS * KP; e += TH) {
    const int r = e / KP;
    const int k = e - r * KP;
    if (r >= rows) continue;
    C* row = buf + r * NZH;
    const C a = row[k];
    const C b = row[H - k];
    const C w = twn[k];  // W^k = exp(-2 pi i k / NZ)
    {
      // C'[k] = (A[k] + conj(A[h-k])) + i conj(W^k) (A[k] - conj(A[h-k]))
      const C ep = {a.x + b.x, a.y - b.y};
      const C dm = {a.x - b.x, a.y + b.y};
      const C op = cmulc(dm, w);
      row[k] = {ep.x - op.y, ep.y + op.x};
    }
    if (k > 0 && H - k != k) {
      // C'[h-k] = (A[h-k] + conj(A[k])) + i (-W^k) (A[h-k] - conj(A[k]))
      const C ep = {b.x + a.x, b.y - a.y};
      const C dm = {b.x - a.x, b.y + a.y};
      const C op = cmul(dm, w);
      row[H - k] = {ep.x + op.y, ep.y - op.x};
    }
  }
}

// ---------------------------------------------------------------------------
// Plane / row pass.  DO_Y: tile = one whole x-plane (ROWS = ny) and the y FFT
// is done here; otherwise tile = ROWS consecutive (x,y) rows, z only.
// ---------------------------------------------------------------------------
template <typename T, int ROWS, int NZ, int TH, bool DO_Y>
__global__ void __launch_bounds__(TH)
    plane_kernel(const PlaneWork<T>* __restrict__ works, int nrows_total,
                 const c2_t<T>* __restrict__ tw_y, const c2_t<T>* __restrict__ tw_zh,
                 const c2_t<T>* __restrict__ tw_z) {
  using C = c2_t<T>;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int H = (NZ > 1) ? NZ / 2 : 1;
  constexpr int SPEC = ROWS * NZH;
  constexpr int RS = 2 * NZH;  // real row stride inside the buffer
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_tw_zh = reinterpret_cast<C*>(smem_raw);
  C* s_tw_z = s_tw_zh + H;
  C* s_tw_y = s_tw_z + NZ;
  C* buf = s_tw_y + (DO_Y ? ROWS : 0);
  T* rbuf = reinterpret_cast<T*>(buf);

  const PlaneWork<T> w = works[blockIdx.y];
  const int tid = threadIdx.x;
  const int row0 = blockIdx.x * ROWS;
  const int rows = min(ROWS, nrows_total - row0);
  const size_t roff = (size_t)row0 * NZ;
  const size_t soff = (size_t)row0 * NZH;

  if constexpr (NZ > 1) {
    for (int i = tid; i < H; i += TH) s_tw_zh[i] = tw_zh[i];
    for (int i = tid; i < NZ; i += TH) s_tw_z[i] = tw_z[i];
  }
  if constexpr (DO_Y) {
    for (int i = tid; i < ROWS; i += TH) s_tw_y[i] = tw_y[i];
  }

  if (w.mode != MODE_FIRST) {
    for (int i = tid; i < SPEC; i += TH) {
      const int r = i / NZH;
      buf[i] = (r < rows) ? w.spec[soff + i] : C{T(0), T(0)};
    }
    __syncthreads();
    if constexpr (DO_Y) smem_fft<ROWS, NZH, TH, true, true>(buf, 1, NZH, s_tw_y);
    if constexpr (NZ > 1) {
      c2r_pre<NZ, ROWS, TH>(buf, s_tw_z, rows);
      __syncthreads();
      smem_fft<H, ROWS, TH, true, false>(buf, NZH, 1, s_tw_zh);
    }
    const bool mid = (w.mode == MODE_MID);
    for (int e = tid; e < ROWS * NZ; e += TH) {
      const int r = e / NZ;
      const int z = e - r * NZ;
      if (r >= rows) continue;
      const size_t g = roff + (size_t)e;
      const T a = rbuf[r * RS + z];
      const T q = a * ld_or_one(w.wfac_in, g);
      w.store[g] = q;
      if (mid) rbuf[r * RS + z] = q * ld_or_one(w.wfac_out, g);
    }
    if (!mid) return;  // uniform over the CTA
  } else {
    for (int e = tid; e < ROWS * NZ; e += TH) {
      const int r = e / NZ;
      const int z = e - r * NZ;
      T a = T(0);
      if (r < rows) {
        const size_t g = roff + (size_t)e;
        a = w.src ? w.src[g] : T(1);
        if (w.store) w.store[g] = a;
        a = a * ld_or_one(w.wfac_out, g);
      }
      rbuf[r * RS + z] = a;
    }
  }
  if constexpr (NZ == 1) {
    // one real per row: make it a complex number with zero imaginary part
    for (int r = tid; r < ROWS; r += TH) buf[r].y = T(0);
  }
  __syncthreads();
  if constexpr (NZ > 1) {
    smem_fft<H, ROWS, TH, false, false>(buf, NZH, 1, s_tw_zh);
    r2c_post<NZ, ROWS, TH>(buf, s_tw_z, rows);
    __syncthreads();
  }
  if constexpr (DO_Y) smem_fft<ROWS, NZH, TH, false, true>(buf, 1, NZH, s_tw_y);
  for (int i = tid; i < SPEC; i += TH) {
    if (i / NZH < rows) w.spec[soff + i] = buf[i];
  }
}

// ---------------------------------------------------------------------------
// Pencil pass along a strided axis.  Tile = TK adjacent columns of `inner`.
// ---------------------------------------------------------------------------
template <typename T, int L, int TK, int TH, int MODE>
__global__ void __launch_bounds__(TH)
    pencil_kernel(const PencilWork<T>* __restrict__ works, int inner, int tiles,
                  const c2_t<T>* __restrict__ tw, int nx, int ny, int nz) {
  using C = c2_t<T>;
  constexpr int TKP = TK;  // row stride in shared memory
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_tw = reinterpret_cast<C*>(smem_raw);
  C* buf = s_tw + L;
  const PencilWork<T> w = works[blockIdx.y];
  const int tid = threadIdx.x;
  const int o = blockIdx.x / tiles;
  const int c0 = (blockIdx.x - o * tiles) * TK;
  C* base = w.spec + (size_t)o * L * inner;
  for (int i = tid; i < L; i += TH) s_tw[i] = tw[i];
  for (int e = tid; e < L * TK; e += TH) {
    const int i = e / TK;
    const int cc = e - i * TK;
    const int c = c0 + cc;
    buf[i * TKP + cc] = (c < inner) ? base[(size_t)i * inner + c] : C{T(0), T(0)};
  }
  __syncthreads();
  if (MODE != PENCIL_INV) smem_fft<L, TK, TH, false, true>(buf, 1, TKP, s_tw);
  if (MODE == PENCIL_KINV) {
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      if (c < inner) {
        const T f = __ldg(w.kx + i) * __ldg(w.kyz + c);
        C v = buf[i * TKP + cc];
        buf[i * TKP + cc] = {v.x * f, v.y * f};
      }
    }
    __syncthreads();
  } else if (MODE == PENCIL_KFULL) {
    // scaledFFTPair with an arbitrary real kdata: Re(IFFT(kdata*X)) equals the
    // c2r of X * (kdata(k) + kdata(-k))/2 for a Hermitian X.
    const int nzh = nz / 2 + 1;
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      if (c < inner) {
        const int y = c / nzh;
        const int kz = c - y * nzh;
        const int xm = (nx - i) % nx, ym = (ny - y) % ny, zm = (nz - kz) % nz;
        const double k1 = w.kfull[((size_t)i * ny + y) * nz + kz];
        const double k2 = w.kfull[((size_t)xm * ny + ym) * nz + zm];
        const T f = T(0.5 * (k1 + k2));
        C v = buf[i * TKP + cc];
        buf[i * TKP + cc] = {v.x * f, v.y * f};
      }
    }
    __syncthreads();
  }
  if (MODE != PENCIL_FWD) smem_fft<L, TK, TH, true, true>(buf, 1, TKP, s_tw);
  for (int e = tid; e < L * TK; e += TH) {
    const int i = e / TK;
    const int cc = e - i * TK;
    const int c = c0 + cc;
    if (c < inner) base[(size_t)i * inner + c] = buf[i * TKP + cc];
  }
}

// ---------------------------------------------------------------------------
// Dispatch.
// ---------------------------------------------------------------------------
// Opt in to large dynamic shared memory once per (kernel, device).
template <typename K>
static cudaError_t ensure_smem_attr(K kern, size_t smem, unsigned* done_mask) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned bit = 1u << (dev & 31);
  if (*done_mask & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) *done_mask |= bit;
  return e;
}

static const int kExtents[] = {1, 4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 256};

bool extent_supported(int n) {
  for (int e : kExtents)
    if (e == n) return true;
  return false;
}

template <typename T, int ROWS, int NZ, int TH, bool DO_Y>
static cudaError_t launch_plane_t(const PlaneWork<T>* d_works, int nworks, int ntiles,
                                  int nrows_total, const c2_t<T>* tw_y, const c2_t<T>* tw_zh,
                                  const c2_t<T>* tw_z, cudaStream_t st) {
  using C = c2_t<T>;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int H = (NZ > 1) ? NZ / 2 : 1;
  const size_t smem = sizeof(C) * ((size_t)H + NZ + (DO_Y ? ROWS : 0) + (size_t)ROWS * NZH);
  auto kern = plane_kernel<T, ROWS, NZ, TH, DO_Y>;
  static unsigned attr_mask = 0;
  cudaError_t ea = ensure_smem_attr(kern, smem, &attr_mask);
  if (ea != cudaSuccess) return ea;
  dim3 grid(ntiles, nworks);
  kern<<<grid, TH, smem, st>>>(d_works, nrows_total, tw_y, tw_zh, tw_z);
  return cudaGetLastError();
}

// (ny, nz) planes with a fused y-z kernel instantiation.
static const int kPlaneShapes[][2] = {{8, 8},   {12, 12}, {16, 16}, {24, 24}, {32, 32},
                                      {48, 48}, {64, 64}, {96, 96}, {128, 128}, {16, 1},
                                      {32, 1},  {64, 1},  {128, 1}};

bool plane_fused_supported(int prec_bytes, int ny, int nz) {
  bool listed = false;
  for (auto& s : kPlaneShapes) listed |= (s[0] == ny && s[1] == nz);
  if (!listed) return false;
  size_t nzh = nz / 2 + 1;
  size_t bytes = (size_t)2 * prec_bytes * ((size_t)nz + nz + ny + (size_t)ny * nzh);
  return bytes <= 200 * 1024;
}

#define PSB_PLANE_CASE(T, NY, NZ, TH)                                                     \
  if (ny == NY && nz == NZ)                                                               \
    return launch_plane_t<T, NY, NZ, TH, true>(d_works, nworks, nx, nx * ny, tw_y, tw_zh, \
                                               tw_z, st);

template <typename T>
cudaError_t launch_plane_impl(const PlaneWork<T>* d_works, int nworks, int nx, int ny, int nz,
                              const c2_t<T>* tw_y, const c2_t<T>* tw_zh, const c2_t<T>* tw_z,
                              cudaStream_t st) {
  PSB_PLANE_CASE(T, 8, 8, 64)
  PSB_PLANE_CASE(T, 12, 12, 64)
  PSB_PLANE_CASE(T, 16, 16, 128)
  PSB_PLANE_CASE(T, 24, 24, 128)
  PSB_PLANE_CASE(T, 32, 32, 256)
  PSB_PLANE_CASE(T, 48, 48, 256)
  PSB_PLANE_CASE(T, 64, 64, 256)
  PSB_PLANE_CASE(T, 96, 96, 512)
  PSB_PLANE_CASE(T, 128, 128, 512)
  PSB_PLANE_CASE(T, 16, 1, 64)
  PSB_PLANE_CASE(T, 32, 1, 64)
  PSB_PLANE_CASE(T, 64, 1, 64)
  PSB_PLANE_CASE(T, 128, 1, 128)
  return cudaErrorInvalidValue;
}

#define PSB_ROW_CASE(T, NZ, ROWS, TH)                                                      \
  if (nz == NZ)                                                                            \
    return launch_plane_t<T, ROWS, NZ, TH, false>(d_works, nworks, (nrows + ROWS - 1) / ROWS, \
                                                  nrows, nullptr, tw_zh, tw_z, st);

template <typename T>
cudaError_t launch_rows_impl(const PlaneWork<T>* d_works, int nworks, int nrows, int nz,
                             const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st) {
  PSB_ROW_CASE(T, 1, 256, 256)
  PSB_ROW_CASE(T, 4, 64, 128)
  PSB_ROW_CASE(T, 8, 32, 128)
  PSB_ROW_CASE(T, 12, 32, 128)
  PSB_ROW_CASE(T, 16, 16, 128)
  PSB_ROW_CASE(T, 24, 16, 128)
  PSB_ROW_CASE(T, 32, 16, 256)
  PSB_ROW_CASE(T, 48, 8, 128)
  PSB_ROW_CASE(T, 64, 8, 256)
  PSB_ROW_CASE(T, 96, 8, 256)
  PSB_ROW_CASE(T, 128, 8, 256)
  PSB_ROW_CASE(T, 256, 4, 256)
  return cudaErrorInvalidValue;
}

template <typename T, int L, int TK, int TH, int MODE>
static cudaError_t launch_pencil_t(const PencilWork<T>* d_works, int nworks, int outer, int inner,
                                   const c2_t<T>* tw, int nx, int ny, int nz, cudaStream_t st) {
  using C = c2_t<T>;
  const size_t smem = sizeof(C) * ((size_t)L + (size_t)L * TK);
  auto kern = pencil_kernel<T, L, TK, TH, MODE>;
  static unsigned attr_mask = 0;
  cudaError_t ea = ensure_smem_attr(kern, smem, &attr_mask);
  if (ea != cudaSuccess) return ea;
  const int tiles = (inner + TK - 1) / TK;
  dim3 grid(outer * tiles, nworks);
  kern<<<grid, TH, smem, st>>>(d_works, inner, tiles, tw, nx, ny, nz);
  return cudaGetLastError();
}

template <typename T, int L, int TK, int TH>
static cudaError_t launch_pencil_modes(const PencilWork<T>* d_works, int nworks, int mode, int outer,
                                       int inner, const c2_t<T>* tw, int nx, int ny, int nz,
                                       cudaStream_t st) {
  switch (mode) {
    case PENCIL_FWD:
      return launch_pencil_t<T, L, TK, TH, PENCIL_FWD>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_INV:
      return launch_pencil_t<T, L, TK, TH, PENCIL_INV>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_KINV:
      return launch_pencil_t<T, L, TK, TH, PENCIL_KINV>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_KFULL:
      return launch_pencil_t<T, L, TK, TH, PENCIL_KFULL>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
  }
  return cudaErrorInvalidValue;
}

template <typename T> struct PencilTK { static constexpr int v = 16; };
template <> struct PencilTK<double> { static constexpr int v = 8; };

#define PSB_PENCIL_CASE(T, L, TH)                                                          \
  if (len == L)                                                                             \
    return launch_pencil_modes<T, L, PencilTK<T>::v, TH>(d_works, nworks, mode, outer, inner, tw, \
                                                         nx, ny, nz, st);

template <typename T>
cudaError_t launch_pencil_impl(const PencilWork<T>* d_works, int nworks, int mode, int len,
                               int outer, int inner, const c2_t<T>* tw, int nx, int ny, int nz,
                               cudaStream_t st) {
  PSB_PENCIL_CASE(T, 1, 64)
  PSB_PENCIL_CASE(T, 4, 64)
  PSB_PENCIL_CASE(T, 8, 64)
  PSB_PENCIL_CASE(T, 12, 64)
  PSB_PENCIL_CASE(T, 16, 64)
  PSB_PENCIL_CASE(T, 24, 64)
  PSB_PENCIL_CASE(T, 32, 128)
  PSB_PENCIL_CASE(T, 48, 128)
  PSB_PENCIL_CASE(T, 64, 128)
  PSB_PENCIL_CASE(T, 96, 128)
  PSB_PENCIL_CASE(T, 128, 256)
  PSB_PENCIL_CASE(T, 256, 256)
  return cudaErrorInvalidValue;
}

// Explicit entry points.
template <>
cudaError_t launch_plane<float>(const PlaneWork<float>* w, int nw, int nx, int ny, int nz,
                                const float2* ty, const float2* tzh, const float2* tz,
                                cudaStream_t st) {
  return launch_plane_impl<float>(w, nw, nx, ny, nz, ty, tzh, tz, st);
}
template <>
cudaError_t launch_plane<double>(const PlaneWork<double>* w, int nw, int nx, int ny, int nz,
                                 const double2* ty, const double2* tzh, const double2* tz,
                                 cudaStream_t st) {
  return launch_plane_impl<double>(w, nw, nx, ny, nz, ty, tzh, tz, st);
}
template <>
cudaError_t launch_rows<float>(const PlaneWork<float>* w, int nw, int nrows, int nz,
                               const float2* tzh, const float2* tz, cudaStream_t st) {
  return launch_rows_impl<float>(w, nw, nrows, nz, tzh, tz, st);
}
template <>
cudaError_t launch_rows<double>(const PlaneWork<double>* w, int nw, int nrows, int nz,
                                const double2* tzh, const double2* tz, cudaStream_t st) {
  return launch_rows_impl<double>(w, nw, nrows, nz, tzh, tz, st);
}
template <>
cudaError_t launch_pencil<float>(const PencilWork<float>* w, int nw, int mode, int L, int outer,
                                 int inner, const float2* tw, int nx, int ny, int nz,
                                 cudaStream_t st) {
  return launch_pencil_impl<float>(w, nw, mode, L, outer, inner, tw, nx, ny, nz, st);
}
template <>
cudaError_t launch_pencil<double>(const PencilWork<double>* w, int nw, int mode, int L, int outer,
                                  int inner, const double2* tw, int nx, int ny, int nz,
                                  cudaStream_t st) {
  return launch_pencil_impl<double>(w, nw, mode, L, outer, inner, tw, nx, ny, nz, st);
}

}  // namespace psb
