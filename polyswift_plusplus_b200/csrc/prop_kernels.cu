// Propagator-step kernels for sm_100a.
//
// One step of PsFlexPseudoSpec::solveQ (pspolymer/PsFlexPseudoSpec.cpp:267-289)
//     q(s+ds) = wfac * Re(IFFT(k2 * FFT(wfac * q(s)))) / N
// is split into two passes over a half spectrum S[x][y][kz] (kz <= nz/2) that
// stays resident in L2 between passes:
//   plane pass  (one CTA per x-plane, whole y-z plane in shared memory, loaded
//       and stored with one bulk TMA copy each):
//       inverse y FFT -> inverse z c2r -> q = a*wfac_in -> store q(s+ds)
//       -> a = q*wfac_out -> forward z r2c -> forward y FFT
//     i.e. the end of step s and the start of step s+1 fused in one launch;
//   pencil pass (TK adjacent (y,kz) columns per CTA): forward x FFT,
//       multiply by exp(-ds b^2 k^2)/N from separable 1D tables, inverse x FFT.
// When a plane does not fit in shared memory the plane pass becomes a row pass
// (z only) plus y pencil passes.  Real <-> half-spectrum transforms use the
// half-length complex FFT of the even/odd samples with an in-place pairwise
// post-/pre-processing step (k with h-k of the same row).
#include <stdlib.h>
#include <cstdio>

#include "../../include/pswift.h"
#include "fft_smem.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace psb {

// Poll limit of the plane pass's first wait on its bulk spectrum copy (the
// wait in the timeout path that drains a copy still in flight keeps kMaxPolls).
// Lowered only by ps_gpu_set_bulk_wait_limit, to test the timeout path.
__constant__ uint32_t c_bulk_wait_polls = kMaxPolls;

template <typename T>
__device__ __forceinline__ T ld_or_one(const T* p, size_t i) {
  return p ? __ldg(p + i) : T(1);
}

// ---------------------------------------------------------------------------
// Mean-mode carry (see PlaneWork in kernels.h).
// ---------------------------------------------------------------------------
// Per-warp FP64 sums of the forward input, summed into one CTA partial.
__shared__ double s_dc_warp[32];
// The mean-mode value of the inverse transform rounded to T; written by
// thread 0 after pdl_wait(), read after the barriers that precede the inverse
// step (kept in shared memory, not in registers, through the FFT passes).  What
// the rounding drops comes back through the next step's mean (dc_err).
__shared__ __align__(16) double s_dc_hilo[2];

template <typename T>
__device__ __forceinline__ void dc_hilo_store(const double* dc_in) {
  if (threadIdx.x == 0 && dc_in) reinterpret_cast<T*>(s_dc_hilo)[0] = T(*dc_in);
}

// x + mean-mode value
template <typename T>
__device__ __forceinline__ c2_t<T> dc_add2(c2_t<T> x) {
  const T m = reinterpret_cast<const T*>(s_dc_hilo)[0];
  return cadd(x, c2_t<T>{m, m});
}
template <typename T>
__device__ __forceinline__ T dc_add(T x) {
  return x + reinterpret_cast<const T*>(s_dc_hilo)[0];
}

// Every thread of the CTA calls this (CTA-uniform): lane 0 keeps its warp's sum.
__device__ __forceinline__ void dc_warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) s_dc_warp[threadIdx.x >> 5] = v;
}

// After a __syncthreads() that follows dc_warp_sum: thread 0 stores the CTA's
// partial (warps in order) and CTA 0 the number of partials.  The pointers are
// read from the descriptor here, not kept in registers through the kernel.
template <typename T>
__device__ __forceinline__ void dc_cta_store(const PlaneWork<T>* wp) {
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += s_dc_warp[i];
    double* out = reinterpret_cast<double*>(
        __ldg(reinterpret_cast<const unsigned long long*>(&wp->dc_out)));
    out[blockIdx.x] = s;
    if (blockIdx.x == 0) {
      double* cnt = reinterpret_cast<double*>(
          __ldg(reinterpret_cast<const unsigned long long*>(&wp->dc_count)));
      *cnt = (double)gridDim.x;
    }
  }
}

// Spectral pass side: one warp sums the plane pass's partials in a fixed order
// (lane l takes slots l, l + 32, ...; then a butterfly) and stores the mean.
// load() issues the count and the first kDcMinSlots slots (before the count is
// known) so that they travel with the tile loads; finish() sums them.
template <typename T> struct DcFinish {
  double cnt;
  double v[kDcMinSlots / 32];
  __device__ __forceinline__ void load(const PencilWork<T>& w) {
    const int lane = threadIdx.x & 31;
    cnt = *w.dc_count;
#pragma unroll
    for (int k = 0; k < kDcMinSlots / 32; ++k) v[k] = w.dc_parts[lane + 32 * k];
  }
  __device__ __forceinline__ void finish(const PencilWork<T>& w) const {
    const int lane = threadIdx.x & 31;
    const int n = (int)cnt;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kDcMinSlots / 32; ++k)
      if (lane + 32 * k < n) s += v[k];
    for (int i = kDcMinSlots + lane; i < n; i += 32) s += w.dc_parts[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
      // error feedback: add what the previous step's rounding to T dropped
      const double m = s * w.dc_scale + (w.dc_first ? 0.0 : *w.dc_err);
      *w.dc_total = m;
      *w.dc_err = m - (double)T(m);
    }
  }
};

// 16-byte vector of T: 4 floats or 2 doubles.
template <typename T> struct Vec16;
template <> struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <> struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <typename V, typename T>
__device__ __forceinline__ T vget(const V& v, int i) {
  return reinterpret_cast<const T*>(&v)[i];
}
template <typename V, typename T>
__device__ __forceinline__ void vset(V& v, int i, T x) {
  reinterpret_cast<T*>(&v)[i] = x;
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
// nz = 128 rows (half length H = 64 = 8 x 8): the c2r pre-processing is folded
// into the first inverse z pass and the r2c post-processing into the last
// forward z pass, removing two shared-memory round trips.  Thread -> (row
// b = t % ROWS, pair p = t / ROWS): butterflies j1 = p and j2 = 8 - p
// (p = 1..3), or 0 and 4 (p = 0).  The elements {j + 8r} of the two butterflies
// hold every partner pair (k, 64 - k) that the pre- and post-processing combine.
// ---------------------------------------------------------------------------
template <typename C>
__device__ __forceinline__ C c2r_pre_one(C a, C b, C w) {
  // C'[k] = (A[k] + conj(A[h-k])) + i conj(W^k) (A[k] - conj(A[h-k]))
  const C ep = {a.x + b.x, a.y - b.y};
  const C dm = {a.x - b.x, a.y + b.y};
  const C op = cmulc(dm, w);
  return {ep.x - op.y, ep.y + op.x};
}

template <typename C>
__device__ __forceinline__ C r2c_post_one(C c, C d, C w) {
  // E = (C[k] + conj(C[km]))/2, O = -i (C[k] - conj(C[km]))/2, A[k] = E + W^k O
  using S = decltype(c.x);
  const C E = {S(0.5) * (c.x + d.x), S(0.5) * (c.y - d.y)};
  const C O = {S(0.5) * (c.y + d.y), S(0.5) * (d.x - c.x)};
  return cadd(E, cmul(w, O));
}

template <int ROWS, int TH, typename C>
__device__ __forceinline__ void z64_inverse_first(C* buf, const C* tw_z) {
  static_assert(ROWS * 4 == TH, "one butterfly pair per thread");
  constexpr int NZH = 65;
  const int b = threadIdx.x % ROWS;
  const int p = threadIdx.x / ROWS;  // uniform over a warp
  const int j1 = p, j2 = (p == 0) ? 4 : 8 - p;
  C* row = buf + b * NZH;
  C a1[8], a2[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    a1[r] = row[j1 + 8 * r];
    a2[r] = row[j2 + 8 * r];
  }
  if (p == 0) {
    const C nyq = row[64];
    a1[0] = c2r_pre_one(a1[0], nyq, tw_z[0]);
#pragma unroll
    for (int r = 1; r < 4; ++r) {
      const C x = a1[r], y = a1[8 - r];
      a1[r] = c2r_pre_one(x, y, tw_z[8 * r]);
      a1[8 - r] = c2r_pre_one(y, x, tw_z[8 * (8 - r)]);
    }
    a1[4] = c2r_pre_one(a1[4], a1[4], tw_z[32]);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const C x = a2[r], y = a2[7 - r];
      a2[r] = c2r_pre_one(x, y, tw_z[4 + 8 * r]);
      a2[7 - r] = c2r_pre_one(y, x, tw_z[4 + 8 * (7 - r)]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const C x = a1[r], y = a2[7 - r];
      a1[r] = c2r_pre_one(x, y, tw_z[j1 + 8 * r]);
      a2[7 - r] = c2r_pre_one(y, x, tw_z[j2 + 8 * (7 - r)]);
    }
  }
  __syncthreads();  // every element read before any is overwritten
  Dft<8, true, C>::run(a1);
  Dft<8, true, C>::run(a2);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    row[8 * j1 + r] = a1[r];
    row[8 * j2 + r] = a2[r];
  }
  __syncthreads();
}

template <int ROWS, int TH, typename C>
__device__ __forceinline__ void z64_forward_last(C* buf, const C* tw_zh, const C* tw_z) {
  static_assert(ROWS * 4 == TH, "one butterfly pair per thread");
  constexpr int NZH = 65;
  const int b = threadIdx.x % ROWS;
  const int p = threadIdx.x / ROWS;
  const int j1 = p, j2 = (p == 0) ? 4 : 8 - p;
  C* row = buf + b * NZH;
  C v1[8], v2[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    v1[r] = row[j1 + 8 * r];
    v2[r] = row[j2 + 8 * r];
  }
  __syncthreads();
  // last Stockham pass of the 64-point forward FFT (radix 8, 8 already applied)
#pragma unroll
  for (int r = 1; r < 8; ++r) {
    v1[r] = cmul(v1[r], tw_zh[r * j1]);
    v2[r] = cmul(v2[r], tw_zh[r * j2]);
  }
  Dft<8, false, C>::run(v1);
  Dft<8, false, C>::run(v2);
  // v1[r] = C[j1 + 8r], v2[r] = C[j2 + 8r] (natural order); post-process pairs
  if (p == 0) {
    using S = decltype(v1[0].x);
    const C c0 = v1[0];
    const C E = {c0.x, S(0)};
    const C O = {c0.y, S(0)};
    row[64] = C{E.x - O.x, S(0)};
    row[0] = C{E.x + O.x, S(0)};
#pragma unroll
    for (int r = 1; r < 4; ++r) {
      const C x = v1[r], y = v1[8 - r];
      row[8 * r] = r2c_post_one(x, y, tw_z[8 * r]);
      row[8 * (8 - r)] = r2c_post_one(y, x, tw_z[8 * (8 - r)]);
    }
    row[32] = r2c_post_one(v1[4], v1[4], tw_z[32]);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const C x = v2[r], y = v2[7 - r];
      row[4 + 8 * r] = r2c_post_one(x, y, tw_z[4 + 8 * r]);
      row[4 + 8 * (7 - r)] = r2c_post_one(y, x, tw_z[4 + 8 * (7 - r)]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const C x = v1[r], y = v2[7 - r];
      row[j1 + 8 * r] = r2c_post_one(x, y, tw_z[j1 + 8 * r]);
      row[j2 + 8 * (7 - r)] = r2c_post_one(y, x, tw_z[j2 + 8 * (7 - r)]);
    }
  }
  __syncthreads();
}

// Radix plan of the y FFT of a plane: 128 = 16 x 8 (two passes; with the kz = 0
// and kz = nz/2 columns packed the 512 threads each take one radix-16 and two
// radix-8 butterflies).
template <int L> struct PlanY { using type = typename Plan<L>::type; };
template <> struct PlanY<128> { using type = RadixList<16, 8>; };

// y FFTs of a whole plane S[y][kz].  In y-space the kz = 0 and kz = nz/2
// columns are real (the DC and Nyquist bins of a real z transform), so the two
// share one complex transform: the inverse of A_0 + i A_h is a_0 + i a_h, and
// the forward transform of x_0 + i x_h is split by Hermitian symmetry,
// A_0[k] = (C[k] + conj(C[-k]))/2, A_h[k] = -i (C[k] - conj(C[-k]))/2.  The y
// FFT then runs over nz/2 columns instead of nz/2 + 1.
// The packing and unpacking are loops of their own: folded into the first and
// last Stockham passes (pencil 0's reads and writes) they made one thread in
// every other warp diverge, and the 128^3 step took 16.1 instead of 15.4 us.
template <int ROWS, int NZH, int TH, typename C>
__device__ __forceinline__ void plane_y_inverse(C* buf, const C* tw) {
  if constexpr (NZH > 1 && ROWS > 1) {
    for (int y = threadIdx.x; y < ROWS; y += TH) {
      const C a = buf[y * NZH], b = buf[y * NZH + NZH - 1];
      buf[y * NZH] = C{a.x - b.y, a.y + b.x};
    }
    __syncthreads();
    smem_fft<ROWS, NZH - 1, TH, true, true, C, typename PlanY<ROWS>::type>(buf, 1, NZH, tw);
    using S = decltype(buf[0].x);
    for (int y = threadIdx.x; y < ROWS; y += TH) {
      const C c = buf[y * NZH];
      buf[y * NZH] = C{c.x, S(0)};
      buf[y * NZH + NZH - 1] = C{c.y, S(0)};
    }
    __syncthreads();
  } else {
    smem_fft<ROWS, NZH, TH, true, true>(buf, 1, NZH, tw);
  }
}

template <int ROWS, int NZH, int TH, typename C>
__device__ __forceinline__ void plane_y_forward(C* buf, const C* tw) {
  if constexpr (NZH > 1 && ROWS > 1) {
    for (int y = threadIdx.x; y < ROWS; y += TH) buf[y * NZH] = C{buf[y * NZH].x, buf[y * NZH + NZH - 1].x};
    __syncthreads();
    smem_fft<ROWS, NZH - 1, TH, false, true, C, typename PlanY<ROWS>::type>(buf, 1, NZH, tw);
    using S = decltype(buf[0].x);
    for (int k = threadIdx.x; k <= ROWS / 2; k += TH) {
      const int km = (ROWS - k) % ROWS;
      const C c = buf[k * NZH], d = buf[km * NZH];
      const C a0 = {S(0.5) * (c.x + d.x), S(0.5) * (c.y - d.y)};
      const C ah = {S(0.5) * (c.y + d.y), S(0.5) * (d.x - c.x)};
      buf[k * NZH] = a0;
      buf[k * NZH + NZH - 1] = ah;
      if (km != k) {
        buf[km * NZH] = C{a0.x, -a0.y};
        buf[km * NZH + NZH - 1] = C{ah.x, -ah.y};
      }
    }
    __syncthreads();
  } else {
    smem_fft<ROWS, NZH, TH, false, true>(buf, 1, NZH, tw);
  }
}

// Real-space part of a step on the tile held in shared memory (row stride RS
// reals): MID: q = a*wfac_in, store q, a = q*wfac_out; LAST: q = a*wfac_in,
// store q; FIRST: a = src (or 1), store a, a = a*wfac_out.
// Pairs of reals: one 8-byte (FP32) or 16-byte (FP64) access, aligned in the
// shared tile (rows of 2*(nz/2+1) reals) and conflict-free for consecutive threads.
template <typename T> struct RVec;
template <> struct RVec<float> {
  using type = float2;
  static constexpr int n = 2;
};
template <> struct RVec<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <typename T, int ROWS, int NZ, int TH, int UCMAX = 4>
__device__ __forceinline__ void real_space(const PlaneWork<T>& w, T* rbuf, size_t roff, int rows) {
  constexpr int RS = 2 * (NZ / 2 + 1);
  using VT = RVec<T>;
  using V = typename VT::type;
  constexpr int VN = VT::n;
  if constexpr (NZ % VN == 0 && (ROWS * NZ / VN) % TH == 0) {
    // vectorised, in chunks of UC vectors per thread whose global loads are all
    // issued before any of them is used
    constexpr int G = ROWS * NZ / VN;
    constexpr int U = G / TH;
    constexpr int UC = (UCMAX >= 8 && U % 8 == 0)
                           ? 8
                           : ((U % 4 == 0) ? 4 : ((U % 3 == 0) ? 3 : ((U % 2 == 0) ? 2 : 1)));
    constexpr int ZV = NZ / VN;
    static_assert(U % UC == 0, "chunking");
    const bool same = (w.wfac_in == w.wfac_out);
    const bool need_in = (w.mode != MODE_FIRST) && w.wfac_in;
    const bool need_out = (w.mode != MODE_LAST) && w.wfac_out && !(w.mode == MODE_MID && same);
    const bool need_src = (w.mode == MODE_FIRST) && w.src;
    const bool dc_in = (w.mode != MODE_FIRST) && w.dc_in;
    const bool dc_sum = (w.mode != MODE_LAST) && w.dc_out;
    T acc = T(0);
#pragma unroll 1
    for (int u0 = 0; u0 < U; u0 += UC) {
      V a[UC], b[UC];
#pragma unroll
      for (int c = 0; c < UC; ++c) {
        const int g = threadIdx.x + (u0 + c) * TH;
        const int r = g / ZV;
        const size_t gi = roff + (size_t)r * NZ + (size_t)(g - r * ZV) * VN;
        if (r < rows) {
          if (need_in) a[c] = __ldg(reinterpret_cast<const V*>(w.wfac_in + gi));
          else if (need_src) a[c] = *reinterpret_cast<const V*>(w.src + gi);
          if (need_out) b[c] = __ldg(reinterpret_cast<const V*>(w.wfac_out + gi));
        }
      }
#pragma unroll
      for (int c = 0; c < UC; ++c) {
        const int g = threadIdx.x + (u0 + c) * TH;
        const int r = g / ZV;
        const int z = (g - r * ZV) * VN;
        if (r >= rows) continue;
        const size_t gi = roff + (size_t)r * NZ + z;
        V* sp = reinterpret_cast<V*>(rbuf + r * RS + z);
        const V cur = (w.mode == MODE_FIRST) ? V{} : *sp;
        V q;
#pragma unroll
        for (int i = 0; i < VN; ++i) {
          T v;
          if (w.mode == MODE_FIRST) v = need_src ? vget<V, T>(a[c], i) : T(1);
          else {
            T x = vget<V, T>(cur, i);
            if (dc_in) x = dc_add(x);
            v = x * (need_in ? vget<V, T>(a[c], i) : T(1));
          }
          vset(q, i, v);
        }
        if (w.store) *reinterpret_cast<V*>(w.store + gi) = q;
        if (w.mode != MODE_LAST) {
          V o;
#pragma unroll
          for (int i = 0; i < VN; ++i) {
            T f = T(1);
            if (need_out) f = vget<V, T>(b[c], i);
            else if (w.mode == MODE_MID && same && need_in) f = vget<V, T>(a[c], i);
            vset(o, i, vget<V, T>(q, i) * f);
            acc += vget<V, T>(o, i);
          }
          *sp = o;
        }
      }
    }
    if (dc_sum) dc_warp_sum((double)acc);
  } else {
    const bool dc_in = (w.mode != MODE_FIRST) && w.dc_in;
    T acc = T(0);
    for (int e = threadIdx.x; e < ROWS * NZ; e += TH) {
      const int r = e / NZ;
      const int z = e - r * NZ;
      if (r >= rows) continue;
      const size_t g = roff + (size_t)e;
      T q;
      if (w.mode == MODE_FIRST) q = w.src ? w.src[g] : T(1);
      else q = (dc_in ? dc_add(rbuf[r * RS + z]) : rbuf[r * RS + z]) * ld_or_one(w.wfac_in, g);
      if (w.store) w.store[g] = q;
      if (w.mode != MODE_LAST) {
        const T o = q * ld_or_one(w.wfac_out, g);
        rbuf[r * RS + z] = o;
        acc += o;
      }
    }
    if ((w.mode != MODE_LAST) && w.dc_out) dc_warp_sum((double)acc);
  }
}

// Real-space step of a MID pass inside one block (wfac_in == wfac_out),
// applied inside the fused z pass: slot p of row b holds (a[2p], a[2p+1]);
// q = a*wfac is stored and a = q*wfac goes on to the forward transform.
template <typename T, int NZ, int R>
struct RealStepOp {
  using T2 = c2_t<T>;
  static constexpr int M = (NZ / 2) / R;
  const T* wfac;
  T* store;
  size_t roff;
  int rows;
  bool dc_on = false;  // add the mean-mode value (s_dc_hilo) after the inverse transform
  T acc = T(0);        // sum of the forward input (mean-mode carry)
  T2 wf[R];
  __device__ __forceinline__ void prefetch(int b, int j) {
    if (b >= rows) return;
    const T* wi = wfac + roff + (size_t)b * NZ;
#pragma unroll
    for (int r = 0; r < R; ++r) wf[r] = __ldg(reinterpret_cast<const T2*>(wi + 2 * (j + r * M)));
  }
  __device__ __forceinline__ void apply(int b, int j, T2 (&v)[R]) {
    if (b >= rows) return;
    T* st = store + roff + (size_t)b * NZ;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T2 x = dc_on ? dc_add2<T>(v[r]) : v[r];
      const T q0 = x.x * wf[r].x;
      const T q1 = x.y * wf[r].y;
      *reinterpret_cast<T2*>(st + 2 * (j + r * M)) = T2{q0, q1};
      v[r] = T2{q0 * wf[r].x, q1 * wf[r].y};
    }
  }
  // s = the sum of this butterfly's forward inputs (a local FP32 sum: its
  // rounding differs from butterfly to butterfly)
  __device__ __forceinline__ void after(int b, T2 s) {
    if (b < rows) acc += s.x + s.y;
  }
};

// ---------------------------------------------------------------------------
// Plane / row pass.  DO_Y: tile = one whole x-plane (ROWS = ny), moved in and
// out with bulk TMA copies, and the y FFT is done here; otherwise tile = ROWS
// consecutive (x,y) rows, z only.
// ---------------------------------------------------------------------------
// Two resident CTAs per SM for the FP32 512-thread planes (64 registers each).
template <typename T, int TH> struct PlaneMinBlocks {
  static constexpr int v = (sizeof(T) == 4 && TH == 512) ? 2 : 1;
};

// LT (row mode only): the half spectrum is stored transposed, S[kz][x][y], for
// the x-y plane pass; a tile is ROWS consecutive y of one x (ROWS divides ny).
template <typename T, int ROWS, int NZ, int TH, bool DO_Y, bool FZ, bool LT>
__global__ void __launch_bounds__(TH, (PlaneMinBlocks<T, TH>::v))
    plane_kernel(const PlaneWork<T>* __restrict__ works, int nrows_total,
                 const c2_t<T>* __restrict__ tw_y, const c2_t<T>* __restrict__ tw_zh,
                 const c2_t<T>* __restrict__ tw_z, int lt_nx, int lt_ny) {
  using C = c2_t<T>;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int H = (NZ > 1) ? NZ / 2 : 1;
  constexpr int SPEC = ROWS * NZH;
  constexpr uint32_t SPEC_BYTES = (uint32_t)(SPEC * sizeof(C));
  constexpr bool BULK = DO_Y && (SPEC_BYTES % 16 == 0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* s_tw_zh = buf + SPEC;
  C* s_tw_z = s_tw_zh + H;
  C* s_tw_y = s_tw_z + NZ;
  uint64_t* bar = reinterpret_cast<uint64_t*>(s_tw_y + (DO_Y ? ROWS : 0));
  T* rbuf = reinterpret_cast<T*>(buf);

  const PlaneWork<T> w = works[blockIdx.y];
  const int tid = threadIdx.x;
  const int row0 = blockIdx.x * ROWS;
  const int rows = min(ROWS, nrows_total - row0);
  const size_t roff = (size_t)row0 * NZ;
  const size_t soff = (size_t)row0 * NZH;
  const bool load_spec = (w.mode != MODE_FIRST);
  const bool dc_sum = (w.mode != MODE_LAST) && (w.dc_out != nullptr);  // mean-mode carry

  if (BULK && load_spec && tid == 0) {
    pdl_wait();
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(bar, SPEC_BYTES);
    bulk_g2s(buf, w.spec + soff, SPEC_BYTES, bar);
  }
  if constexpr (NZ > 1) {
    for (int i = tid; i < H; i += TH) s_tw_zh[i] = tw_zh[i];
    for (int i = tid; i < NZ; i += TH) s_tw_z[i] = tw_z[i];
  }
  if constexpr (DO_Y) {
    for (int i = tid; i < ROWS; i += TH) s_tw_y[i] = tw_y[i];
  }
  pdl_wait();  // before any read of the spectrum, src or wfac, and any write
  if (load_spec) dc_hilo_store<T>(w.dc_in);  // used after the barriers below

  if (load_spec) {
    if constexpr (BULK) {
      __syncthreads();  // the mbarrier is initialised before anyone polls it
      // every thread waits (bounded); the CTA then agrees on the outcome
      const int ok = __syncthreads_and(mbar_wait_bounded(bar, 0, c_bulk_wait_polls) ? 1 : 0);
      if (!ok) {
        // the copy did not land in time: flag it, give the copy in flight one
        // more bounded wait, and leave without touching the buffer
        if (tid == 0) {
          if (w.status) atomicOr(w.status, 4);
          mbar_wait_bounded(bar, 0);
        }
        return;
      }
    } else {
      if constexpr (LT) {
        // element (row yy, kz) sits at S[kz][x][y0 + yy]: consecutive threads
        // take consecutive y, so every kz reads one contiguous segment
        const int x = row0 / lt_ny;
        const int y0 = row0 - x * lt_ny;
        for (int i = tid; i < SPEC; i += TH) {
          const int kz = i / ROWS;
          const int yy = i - kz * ROWS;
          buf[yy * NZH + kz] = (yy < rows)
                                   ? w.spec[((size_t)kz * lt_nx + x) * lt_ny + y0 + yy]
                                   : C{T(0), T(0)};
        }
      } else {
        for (int i = tid; i < SPEC; i += TH) {
          const int r = i / NZH;
          buf[i] = (r < rows) ? w.spec[soff + i] : C{T(0), T(0)};
        }
      }
    }
    __syncthreads();
    if constexpr (DO_Y) plane_y_inverse<ROWS, NZH, TH>(buf, s_tw_y);
    if constexpr (NZ > 1) {
      if (FZ && w.mode == MODE_MID && w.wfac_in && w.wfac_in == w.wfac_out && w.store) {
        if constexpr (NZ == 128 && DO_Y && ROWS * 4 == TH) {
          // pre-processing + first inverse pass; last inverse pass + real-space
          // step + first forward pass (index-fastest: each warp covers 4 rows x
          // 8 butterflies, so the wfac loads and q stores are 64-byte segments);
          // last forward pass + post-processing
          z64_inverse_first<ROWS, TH>(buf, s_tw_z);
          RealStepOp<T, NZ, 8> op;
          op.wfac = w.wfac_in;
          op.store = w.store;
          op.roff = roff;
          op.rows = rows;
          op.dc_on = (w.dc_in != nullptr);
          fused_pass_pair<H, 8, ROWS, TH, true, false, false>(buf, NZH, 1, s_tw_zh, op);
          if (dc_sum) dc_warp_sum((double)op.acc);
          z64_forward_last<ROWS, TH>(buf, s_tw_zh, s_tw_z);
          goto forward_y;
        }
        c2r_pre<NZ, ROWS, TH>(buf, s_tw_z, rows);
        __syncthreads();
        // inverse z FFT, real-space step and forward z FFT with the last inverse
        // pass, the step and the first forward pass in one round trip
        using PI = typename Plan<H>::type;
        using PF = typename RLReverse<PI>::type;
        constexpr int RF = RLLast<PI>::value;
        smem_fft_head<H, PI, ROWS, TH, true, true>(buf, NZH, 1, s_tw_zh);
        RealStepOp<T, NZ, RF> op;
        op.wfac = w.wfac_in;
        op.store = w.store;
        op.roff = roff;
        op.rows = rows;
        op.dc_on = (w.dc_in != nullptr);
        fused_pass_pair<H, RF, ROWS, TH, true, false, true>(buf, NZH, 1, s_tw_zh, op);
        if (dc_sum) dc_warp_sum((double)op.acc);
        smem_fft_tail<H, PF, ROWS, TH, false, true>(buf, NZH, 1, s_tw_zh);
        r2c_post<NZ, ROWS, TH>(buf, s_tw_z, rows);
        __syncthreads();
        goto forward_y;
      }
      if constexpr (NZ == 128 && DO_Y && ROWS * 4 == TH) {
        z64_inverse_first<ROWS, TH>(buf, s_tw_z);
        stockham_pass<H, 8, 8, ROWS, TH, true, true>(buf, NZH, 1, s_tw_zh);
      } else {
        c2r_pre<NZ, ROWS, TH>(buf, s_tw_z, rows);
        __syncthreads();
        smem_fft<H, ROWS, TH, true, true>(buf, NZH, 1, s_tw_zh);
      }
    }
  }
  real_space<T, ROWS, NZ, TH>(w, rbuf, roff, rows);
  if (w.mode == MODE_LAST) return;  // uniform over the CTA
  if constexpr (NZ == 1) {
    // one real per row: make it a complex number with zero imaginary part
    for (int r = tid; r < ROWS; r += TH) buf[r].y = T(0);
  }
  __syncthreads();
  if constexpr (NZ > 1) {
    if constexpr (NZ == 128 && DO_Y && ROWS * 4 == TH) {
      stockham_pass<H, 8, 1, ROWS, TH, false, true>(buf, NZH, 1, s_tw_zh);
      z64_forward_last<ROWS, TH>(buf, s_tw_zh, s_tw_z);
    } else {
      smem_fft<H, ROWS, TH, false, true>(buf, NZH, 1, s_tw_zh);
      r2c_post<NZ, ROWS, TH>(buf, s_tw_z, rows);
      __syncthreads();
    }
  }
forward_y:
  if constexpr (DO_Y) plane_y_forward<ROWS, NZH, TH>(buf, s_tw_y);
  if constexpr (BULK) {
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      bulk_s2g(w.spec + soff, buf, SPEC_BYTES);
      bulk_commit();
      bulk_wait_read_all();
    }
  } else {
    if constexpr (LT) {
      const int x = row0 / lt_ny;
      const int y0 = row0 - x * lt_ny;
      for (int i = tid; i < SPEC; i += TH) {
        const int kz = i / ROWS;
        const int yy = i - kz * ROWS;
        if (yy < rows) w.spec[((size_t)kz * lt_nx + x) * lt_ny + y0 + yy] = buf[yy * NZH + kz];
      }
    } else {
      for (int i = tid; i < SPEC; i += TH) {
        if (i / NZH < rows) w.spec[soff + i] = buf[i];
      }
    }
  }
  // the warps' sums were stored before at least one barrier on every path above
  if (dc_sum) dc_cta_store(works + blockIdx.y);
}

// k2 multiply applied inside the fused x pass: exp(-ds b^2 k^2)/N as the
// product of the x table and the (y, kz) table.
template <typename T, int L, int R>
struct KStepOp {
  using T2 = c2_t<T>;
  static constexpr int M = L / R;
  const T* kx;
  const T* kyz;
  int c0;
  int inner;
  bool dc0;  // this tile holds the k = 0 coefficient and the mean mode is carried in FP64
  T fyz;
  __device__ __forceinline__ void prefetch(int b, int j) {
    const int c = c0 + b;
    fyz = (c < inner) ? __ldg(kyz + c) : T(0);
  }
  __device__ __forceinline__ void apply(int b, int j, T2 (&v)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T f = __ldg(kx + j + r * M) * fyz;
      v[r] = T2{v[r].x * f, v[r].y * f};
    }
    if (dc0 && b == 0 && j == 0) v[0] = T2{T(0), T(0)};
  }
  __device__ __forceinline__ void after(int, T2) {}
};

// ---------------------------------------------------------------------------
// Pencil pass along a strided axis.  Tile = TK adjacent columns of `inner`,
// loaded with 16-byte vector loads all issued before use.
// ---------------------------------------------------------------------------
template <typename T, int L, int TK, int TH, int MODE, bool FK>
__global__ void __launch_bounds__(TH)
    pencil_kernel(const PencilWork<T>* __restrict__ works, int inner, int tiles,
                  const c2_t<T>* __restrict__ tw, int nx, int ny, int nz) {
  using C = c2_t<T>;
  using V = typename Vec16<T>::type;
  constexpr int CPV = 16 / sizeof(C);  // complex values per 16-byte vector
  constexpr int VPR = TK / CPV;        // vectors per tile row
  constexpr int NV = L * VPR;          // vectors per tile
  constexpr int UV = (NV + TH - 1) / TH;
  using RL = typename WidePlan<L>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* s_tw = buf + L * TK;
  const PencilWork<T> w = works[blockIdx.y];
  const int tid = threadIdx.x;
  const int o = blockIdx.x / tiles;
  const int c0 = (blockIdx.x - o * tiles) * TK;
  C* base = w.spec + (size_t)o * L * inner;
  const bool full = (c0 + TK <= inner) && (inner % CPV == 0);
  // mean-mode carry: the tile of column 0 drops the FP32 k = 0 coefficient and
  // its first warp turns the plane pass's FP64 partials into the mean
  const bool dc0 = (MODE == PENCIL_KINV) && w.dc_total && o == 0 && c0 == 0;
  for (int i = tid; i < L; i += TH) s_tw[i] = tw[i];
  pdl_wait();  // before any read or write of the spectrum
  DcFinish<T> dcf;
  if (dc0 && tid < 32) dcf.load(w);
  if (full) {
    V v[UV];
#pragma unroll
    for (int u = 0; u < UV; ++u) {
      const int e = tid + u * TH;
      if (NV % TH == 0 || e < NV) {
        const int i = e / VPR;
        const int cv = e - i * VPR;
        v[u] = *reinterpret_cast<const V*>(base + (size_t)i * inner + c0 + cv * CPV);
      }
    }
#pragma unroll
    for (int u = 0; u < UV; ++u) {
      const int e = tid + u * TH;
      if (NV % TH == 0 || e < NV) reinterpret_cast<V*>(buf)[e] = v[u];
    }
  } else {
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      buf[e] = (c < inner) ? base[(size_t)i * inner + c] : C{T(0), T(0)};
    }
  }
  if (dc0 && tid < 32) dcf.finish(w);
  __syncthreads();
  if constexpr (MODE == PENCIL_KINV && L > 1 && FK) {
    // forward FFT, k2 multiply and inverse FFT with the last forward pass, the
    // multiply and the first inverse pass in one round trip
    using RI = typename RLReverse<RL>::type;
    constexpr int RF = RLLast<RL>::value;
    smem_fft_head<L, RL, TK, TH, false, true>(buf, 1, TK, s_tw);
    KStepOp<T, L, RF> op;
    op.kx = w.kx;
    op.kyz = w.kyz;
    op.c0 = c0;
    op.inner = inner;
    op.dc0 = dc0;
    fused_pass_pair<L, RF, TK, TH, false, true, true>(buf, 1, TK, s_tw, op);
    smem_fft_tail<L, RI, TK, TH, true, true>(buf, 1, TK, s_tw);
    goto store_tile;
  }
  if (MODE != PENCIL_INV) smem_fft<L, TK, TH, false, true, C, RL>(buf, 1, TK, s_tw);
  if (MODE == PENCIL_KINV) {
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      if (c < inner) {
        const T f = __ldg(w.kx + i) * __ldg(w.kyz + c);
        const C v = buf[e];
        buf[e] = (dc0 && e == 0) ? C{T(0), T(0)} : C{v.x * f, v.y * f};
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
        const C v = buf[e];
        buf[e] = {v.x * f, v.y * f};
      }
    }
    __syncthreads();
  } else if (MODE == PENCIL_KFULL_IM) {
    // scaledFFTPairIm: Re(IFFT(kdata * FFT(i*data))) is the c2r of
    // i * (kdata(k) - kdata(-k))/2 * X for the Hermitian X = FFT(data); the
    // even part of kdata only produces an imaginary result.
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
        const T f = T(0.5 * (k1 - k2));
        const C v = buf[e];
        buf[e] = {-f * v.y, f * v.x};
      }
    }
    __syncthreads();
  } else if (MODE == PENCIL_KSPEC) {
    // convolveRe: multiply by the second operand's transform, element by
    // element in the same (pencil, column) position.
    const C* kb = w.kspec + (size_t)o * L * inner;
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      if (c < inner) {
        const C b = kb[(size_t)i * inner + c];
        const C v = buf[e];
        buf[e] = {v.x * b.x - v.y * b.y, v.y * b.x + v.x * b.y};
      }
    }
    __syncthreads();
  }
  if (MODE != PENCIL_FWD) smem_fft<L, TK, TH, true, true, C, RL>(buf, 1, TK, s_tw);
store_tile:
  if (full) {
#pragma unroll
    for (int u = 0; u < UV; ++u) {
      const int e = tid + u * TH;
      if (NV % TH == 0 || e < NV) {
        const int i = e / VPR;
        const int cv = e - i * VPR;
        *reinterpret_cast<V*>(base + (size_t)i * inner + c0 + cv * CPV) = reinterpret_cast<const V*>(buf)[e];
      }
    }
  } else {
    for (int e = tid; e < L * TK; e += TH) {
      const int i = e / TK;
      const int cc = e - i * TK;
      const int c = c0 + cc;
      if (c < inner) base[(size_t)i * inner + c] = buf[e];
    }
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

// Sweep kernels are launched with programmatic stream serialisation (they call
// pdl_wait() before touching data another kernel wrote), unless PSB_PDL=0.
static bool pdl_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("PSB_PDL");
    on = (e && e[0] == '0') ? 0 : 1;
  }
  return on != 0;
}

template <typename... K, typename... Args>
static cudaError_t launch_sweep_kernel(void (*kern)(K...), dim3 grid, dim3 block, size_t smem,
                                       cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

static const int kExtents[] = {1, 4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 256};

bool extent_supported(int n) {
  for (int e : kExtents)
    if (e == n) return true;
  return false;
}

template <typename T, int ROWS, int NZ, int TH, bool DO_Y, bool FZ, bool LT = false>
static cudaError_t launch_plane_t(const PlaneWork<T>* d_works, int nworks, int ntiles,
                                  int nrows_total, const c2_t<T>* tw_y, const c2_t<T>* tw_zh,
                                  const c2_t<T>* tw_z, cudaStream_t st, int lt_nx = 0,
                                  int lt_ny = 0) {
  using C = c2_t<T>;
  constexpr int NZH = NZ / 2 + 1;
  constexpr int H = (NZ > 1) ? NZ / 2 : 1;
  const size_t smem =
      sizeof(C) * ((size_t)ROWS * NZH + H + NZ + (DO_Y ? ROWS : 0)) + sizeof(uint64_t);
  auto kern = plane_kernel<T, ROWS, NZ, TH, DO_Y, FZ, LT>;
  static unsigned attr_mask = 0;
  cudaError_t ea = ensure_smem_attr(kern, smem, &attr_mask);
  if (ea != cudaSuccess) return ea;
  dim3 grid(ntiles, nworks);
  return launch_sweep_kernel(kern, grid, dim3(TH), smem, st, d_works, nrows_total, tw_y, tw_zh, tw_z,
                             lt_nx, lt_ny);
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

// ---------------------------------------------------------------------------
// Plane pass of 256 x 256 y-z planes on a cluster of CL CTAs
// (VARIANT_CLUSTER): eight CTAs (PlaneCl).  A 256 x 129 half plane (264 KB in
// FP32, 528 KB in FP64) does not fit one CTA's shared memory; split over the
// cluster it does, and the step needs no y pencil passes (two fewer spectrum
// round trips).  With CH = 128 / CL and RH = 256 / CL, CTA c holds:
//   y phases: kz columns [CH c, CH c + CH) for all y (CTA 0 also kz = 128,
//             which shares the kz = 0 transform), layout Y[y][slot], CH + 1
//             slots a row;
//   z phases: y rows [RH c, RH c + RH) for all kz, layout Z[r][kz], 129 a row.
// Between the phases every thread reads its elements into registers, a cluster
// barrier makes sure every CTA has read its buffer, the elements are written
// to their place in the other layout (this CTA's or a peer's shared memory),
// and a second cluster barrier publishes them.  All CTAs of a cluster work on
// the same plane and mode, so they take the same barriers; no shared memory is
// touched across the cluster after the last one.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Shared-memory address of the same variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_smem(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_peer(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void st_peer(uint32_t addr, double2 v) {
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
}
// Element i of the buffer `buf` in CTA `rank`: here, or a peer's shared memory.
template <typename C>
__device__ __forceinline__ void st_cluster(C* buf, int i, uint32_t rank, uint32_t me, C v) {
  if (rank == me) buf[i] = v;
  else st_peer(peer_smem(buf + i, rank), v);
}

template <typename T> struct PlaneCl;
// Eight 256-thread CTAs per plane in both precisions, so that several CTAs of
// different planes share an SM and hide each other's load latency.  FP32: 64
// registers, 40 KB of shared memory, four CTAs per SM (166 us per 256^3 step,
// against 171 with four 512-thread CTAs and 184 with two 1024-thread CTAs).
// FP64: 126 registers, 80 KB, two CTAs per SM (364 us against 388 with four
// 512-thread CTAs, one per SM).
template <> struct PlaneCl<float> {
  static constexpr int CL = 8, TH = 256, UCMAX = 8, MINB = 4;
};
template <> struct PlaneCl<double> {
  static constexpr int CL = 8, TH = 256, UCMAX = 4, MINB = 2;
};
template <typename T> struct PlaneC256 {
  static constexpr int NY = 256, NZ = 256, NZH = 129, H = 128;
  static constexpr int CL = PlaneCl<T>::CL, TH = PlaneCl<T>::TH;
  static constexpr int CH = (NZ / 2) / CL;  // y-FFT columns per CTA
  static constexpr int YS = CH + 1;         // Y row stride (slot CH: kz = 128 in CTA 0)
  static constexpr int RH = NY / CL;        // z rows per CTA
  static constexpr int YE = NY * YS;
  static constexpr int ZE = RH * NZH;
  static constexpr int BUF = (YE > ZE) ? YE : ZE;
  static constexpr int UY = NY * CH / TH;            // Y elements per thread (+1 slot-CH element)
  static constexpr int UZ = (ZE + TH - 1) / TH;      // Z elements per thread
  static constexpr size_t SMEM = sizeof(c2_t<T>) * ((size_t)BUF + H + NZ + NY);
  // y = e / CH is uniform over each half-warp in the Y -> Z exchange, and the
  // slot-CH column takes one thread per y
  static_assert(CH % 16 == 0 && (NY * CH) % TH == 0 && NY <= TH, "cluster plane layout");
};

template <typename T>
__global__ void __launch_bounds__(PlaneC256<T>::TH, PlaneCl<T>::MINB)
    plane_c256_kernel(const PlaneWork<T>* __restrict__ works, const c2_t<T>* __restrict__ tw_y,
                      const c2_t<T>* __restrict__ tw_zh, const c2_t<T>* __restrict__ tw_z) {
  using P = PlaneC256<T>;
  using C = c2_t<T>;
  constexpr int NY = P::NY, NZ = P::NZ, NZH = P::NZH, H = P::H, TH = P::TH, CH = P::CH, YS = P::YS,
                RH = P::RH, CL = P::CL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* s_tw_zh = buf + P::BUF;
  C* s_tw_z = s_tw_zh + H;
  C* s_tw_y = s_tw_z + NZ;

  const uint32_t me = cluster_ctarank();
  const PlaneWork<T> w = works[blockIdx.y];
  const int x = blockIdx.x / CL;
  const int tid = threadIdx.x;
  const size_t soff = (size_t)x * NY * NZH;
  const int row0 = (int)me * RH;
  const int col0 = (int)me * CH;
  const size_t roff = ((size_t)x * NY + row0) * NZ;
  for (int i = tid; i < H; i += TH) s_tw_zh[i] = tw_zh[i];
  for (int i = tid; i < NZ; i += TH) s_tw_z[i] = tw_z[i];
  for (int i = tid; i < NY; i += TH) s_tw_y[i] = tw_y[i];
  pdl_wait();  // before any read of the spectrum, src or wfac, and any write
  if (w.mode != MODE_FIRST) dc_hilo_store<T>(w.dc_in);  // used after the barriers below

  if (w.mode != MODE_FIRST) {
    // this CTA's columns of the half plane, Y layout; every load issued before
    // the first store
    const C* src = w.spec + soff;
    {
      C t[P::UY];
#pragma unroll
      for (int u = 0; u < P::UY; ++u) {
        const int e = tid + u * TH;
        t[u] = __ldg(src + (size_t)(e / CH) * NZH + col0 + (e % CH));
      }
      C tx = C{T(0), T(0)};
      if (me == 0 && tid < NY) tx = __ldg(src + (size_t)tid * NZH + NZ / 2);
#pragma unroll
      for (int u = 0; u < P::UY; ++u) {
        const int e = tid + u * TH;
        buf[(e / CH) * YS + (e % CH)] = t[u];
      }
      if (me == 0 && tid < NY) buf[tid * YS + CH] = tx;
    }
    __syncthreads();
    // inverse y FFT of the columns (plane_y_inverse on this CTA's part)
    if (me == 0) {
      for (int y = tid; y < NY; y += TH) {
        const C a = buf[y * YS], b = buf[y * YS + CH];
        buf[y * YS] = C{a.x - b.y, a.y + b.x};
      }
    }
    __syncthreads();
    smem_fft<NY, CH, TH, true, true, C, typename PlanY<NY>::type>(buf, 1, YS, s_tw_y);
    if (me == 0) {
      for (int y = tid; y < NY; y += TH) {
        const C c = buf[y * YS];
        buf[y * YS] = C{c.x, T(0)};
        buf[y * YS + CH] = C{c.y, T(0)};
      }
    }
    __syncthreads();
    // Y -> Z: element (y, kz) goes to row y - RH o of CTA o = y / RH
    C v[P::UY];
    C vx = C{T(0), T(0)};
#pragma unroll
    for (int u = 0; u < P::UY; ++u) {
      const int e = tid + u * TH;
      v[u] = buf[(e / CH) * YS + (e % CH)];
    }
    if (me == 0 && tid < NY) vx = buf[tid * YS + CH];
    cluster_sync_all();  // every buffer read
#pragma unroll
    for (int u = 0; u < P::UY; ++u) {
      const int e = tid + u * TH;
      const int y = e / CH, kz = col0 + (e % CH);  // y uniform over a half-warp (CH % 16 == 0)
      const int o = y / RH;
      st_cluster(buf, (y - o * RH) * NZH + kz, (uint32_t)o, me, v[u]);
    }
    if (me == 0 && tid < NY) {
      const int y = tid, o = y / RH;
      st_cluster(buf, (y - o * RH) * NZH + NZ / 2, (uint32_t)o, me, vx);
    }
    cluster_sync_all();  // every Z layout complete
    c2r_pre<NZ, RH, TH>(buf, s_tw_z, RH);
    __syncthreads();
    smem_fft<H, RH, TH, true, true>(buf, NZH, 1, s_tw_zh);
  }
  real_space<T, RH, NZ, TH, PlaneCl<T>::UCMAX>(w, reinterpret_cast<T*>(buf), roff, RH);
  if (w.mode == MODE_LAST) return;  // uniform over the cluster
  __syncthreads();
  smem_fft<H, RH, TH, false, true>(buf, NZH, 1, s_tw_zh);
  r2c_post<NZ, RH, TH>(buf, s_tw_z, RH);
  __syncthreads();
  {
    // Z -> Y: element (r, kz) of row y = row0 + r goes to the CTA owning kz
    C v[P::UZ];
#pragma unroll
    for (int u = 0; u < P::UZ; ++u) {
      const int e = tid + u * TH;
      if (e < P::ZE) v[u] = buf[e];
    }
    cluster_sync_all();  // every buffer read
#pragma unroll
    for (int u = 0; u < P::UZ; ++u) {
      const int e = tid + u * TH;
      if (e < P::ZE) {
        const int r = e / NZH, kz = e - (e / NZH) * NZH;
        const int y = row0 + r;
        const int owner = (kz == NZ / 2) ? 0 : (kz / CH);
        const int slot = (kz == NZ / 2) ? CH : (kz - owner * CH);
        st_cluster(buf, y * YS + slot, (uint32_t)owner, me, v[u]);
      }
    }
    cluster_sync_all();  // every Y layout complete
  }
  // forward y FFT of the columns (plane_y_forward on this CTA's part)
  if (me == 0) {
    for (int y = tid; y < NY; y += TH) buf[y * YS] = C{buf[y * YS].x, buf[y * YS + CH].x};
  }
  __syncthreads();
  smem_fft<NY, CH, TH, false, true, C, typename PlanY<NY>::type>(buf, 1, YS, s_tw_y);
  if (me == 0) {
    for (int k = tid; k <= NY / 2; k += TH) {
      const int km = (NY - k) % NY;
      const C c = buf[k * YS], d = buf[km * YS];
      const C a0 = {T(0.5) * (c.x + d.x), T(0.5) * (c.y - d.y)};
      const C ah = {T(0.5) * (c.y + d.y), T(0.5) * (d.x - c.x)};
      buf[k * YS] = a0;
      buf[k * YS + CH] = ah;
      if (km != k) {
        buf[km * YS] = C{a0.x, -a0.y};
        buf[km * YS + CH] = C{ah.x, -ah.y};
      }
    }
  }
  __syncthreads();
  C* dst = w.spec + soff;
  for (int e = tid; e < NY * CH; e += TH) {
    const int y = e / CH, c = e - (e / CH) * CH;
    dst[(size_t)y * NZH + col0 + c] = buf[y * YS + c];
  }
  if (me == 0)
    for (int y = tid; y < NY; y += TH) dst[(size_t)y * NZH + NZ / 2] = buf[y * YS + CH];
  // mean-mode carry: a partial per CTA (CL per plane), after the barriers above
  if (w.dc_out) dc_cta_store(works + blockIdx.y);
}

template <typename T>
cudaError_t launch_plane_cluster(const PlaneWork<T>* d_works, int nworks, int nx, const c2_t<T>* tw_y,
                                 const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st) {
  using P = PlaneC256<T>;
  auto kern = plane_c256_kernel<T>;
  static unsigned attr_mask = 0;
  cudaError_t e = ensure_smem_attr(kern, P::SMEM, &attr_mask);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P::CL * nx, nworks);
  cfg.blockDim = dim3(P::TH);
  cfg.dynamicSmemBytes = P::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = P::CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, kern, d_works, tw_y, tw_zh, tw_z);
}
template cudaError_t launch_plane_cluster<float>(const PlaneWork<float>*, int, int, const float2*, const float2*,
                                                 const float2*, cudaStream_t);
template cudaError_t launch_plane_cluster<double>(const PlaneWork<double>*, int, int, const double2*,
                                                  const double2*, const double2*, cudaStream_t);

bool cluster_plane_supported(int prec_bytes, int ny, int nz) {
  return (prec_bytes == 4 || prec_bytes == 8) && ny == 256 && nz == 256;
}

#define PSB_PLANE_CASE(T, NY, NZ, TH)                                                      \
  if (ny == NY && nz == NZ)                                                                \
    return (variant & 1) ? launch_plane_t<T, NY, NZ, TH, true, true>(                      \
                               d_works, nworks, nx, nx * ny, tw_y, tw_zh, tw_z, st)        \
                         : launch_plane_t<T, NY, NZ, TH, true, false>(                     \
                               d_works, nworks, nx, nx * ny, tw_y, tw_zh, tw_z, st);

template <typename T>
cudaError_t launch_plane_impl(const PlaneWork<T>* d_works, int nworks, int nx, int ny, int nz,
                              const c2_t<T>* tw_y, const c2_t<T>* tw_zh, const c2_t<T>* tw_z,
                              int variant, cudaStream_t st) {
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
    return launch_plane_t<T, ROWS, NZ, TH, false, false>(                                  \
        d_works, nworks, (nrows + ROWS - 1) / ROWS, nrows, nullptr, tw_zh, tw_z, st);

template <typename T>
cudaError_t launch_rows_impl(const PlaneWork<T>* d_works, int nworks, int nrows, int nz,
                             const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st) {
  PSB_ROW_CASE(T, 1, 256, 256)
  PSB_ROW_CASE(T, 4, 64, 128)
  PSB_ROW_CASE(T, 8, 32, 128)
  PSB_ROW_CASE(T, 12, 32, 128)
  PSB_ROW_CASE(T, 16, 32, 128)
  PSB_ROW_CASE(T, 24, 32, 128)
  PSB_ROW_CASE(T, 32, 32, 256)
  PSB_ROW_CASE(T, 48, 32, 256)
  PSB_ROW_CASE(T, 64, 32, 256)
  PSB_ROW_CASE(T, 96, 16, 256)
  PSB_ROW_CASE(T, 128, 16, 256)
  PSB_ROW_CASE(T, 256, 8, 256)
  return cudaErrorInvalidValue;
}

// Row pass writing the transposed spectrum S[kz][x][y] (tiles of ROWS y of one x).
#define PSB_ROWT_CASE(T, NZ, ROWS, TH)                                                      \
  if (nz == NZ && ny % ROWS == 0)                                                           \
    return launch_plane_t<T, ROWS, NZ, TH, false, false, true>(                             \
        d_works, nworks, nx * ny / ROWS, nx * ny, nullptr, tw_zh, tw_z, st, nx, ny);

template <typename T>
cudaError_t launch_rows_t_impl(const PlaneWork<T>* d_works, int nworks, int nx, int ny, int nz,
                               const c2_t<T>* tw_zh, const c2_t<T>* tw_z, cudaStream_t st) {
  PSB_ROWT_CASE(T, 8, 8, 64)
  PSB_ROWT_CASE(T, 12, 12, 64)
  PSB_ROWT_CASE(T, 16, 16, 128)
  PSB_ROWT_CASE(T, 24, 24, 128)
  PSB_ROWT_CASE(T, 32, 32, 256)
  PSB_ROWT_CASE(T, 48, 16, 256)
  PSB_ROWT_CASE(T, 64, 32, 256)
  PSB_ROWT_CASE(T, 96, 32, 256)
  PSB_ROWT_CASE(T, 128, 32, 256)
  PSB_ROWT_CASE(T, 256, 32, 256)
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// x-y plane pass over the transposed spectrum: one CTA per kz plane, held in
// shared memory with rows padded to NXY + 1 (odd stride: conflict-free along
// both axes).  Forward y FFT, forward x FFT, k2 multiply, inverse x FFT,
// inverse y FFT.
// ---------------------------------------------------------------------------
template <typename T, int NXY, int R>
struct XYKOp {
  using T2 = c2_t<T>;
  static constexpr int M = NXY / R;
  const T* kx;
  const T* kyz;
  int kz;
  int nzh;
  bool dc0;  // kz = 0 plane with the mean mode carried in FP64
  T fyz;
  __device__ __forceinline__ void prefetch(int y, int j) { fyz = __ldg(kyz + (size_t)y * nzh + kz); }
  __device__ __forceinline__ void apply(int y, int j, T2 (&v)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T f = __ldg(kx + j + r * M) * fyz;
      v[r] = T2{v[r].x * f, v[r].y * f};
    }
    if (dc0 && y == 0 && j == 0) v[0] = T2{T(0), T(0)};
  }
  __device__ __forceinline__ void after(int, T2) {}
};

template <typename T, int NXY, int TH, bool FK>
__global__ void __launch_bounds__(TH)
    xy_kernel(const PencilWork<T>* __restrict__ works, int nzh, const c2_t<T>* __restrict__ tw) {
  using C = c2_t<T>;
  using V = typename Vec16<T>::type;
  constexpr int NP = NXY + 1;
  constexpr int NE = NXY * NXY;
  constexpr int CPV = 16 / sizeof(C);
  constexpr int NV = NE / CPV;
  constexpr int UV = (NV + TH - 1) / TH;
  using RL = typename WidePlan<NXY>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* s_tw = buf + NXY * NP;
  const PencilWork<T> w = works[blockIdx.y];
  const int kz = blockIdx.x;
  const int tid = threadIdx.x;
  C* base = w.spec + (size_t)kz * NE;
  const bool dc0 = w.dc_total && kz == 0;  // mean-mode carry (see the pencil pass)
  for (int i = tid; i < NXY; i += TH) s_tw[i] = tw[i];
  pdl_wait();  // before any read or write of the spectrum
  DcFinish<T> dcf;
  if (dc0 && tid < 32) dcf.load(w);
  {
    V v[UV];
#pragma unroll
    for (int u = 0; u < UV; ++u) {
      const int e = tid + u * TH;
      if (NV % TH == 0 || e < NV) v[u] = reinterpret_cast<const V*>(base)[e];
    }
#pragma unroll
    for (int u = 0; u < UV; ++u) {
      const int e = tid + u * TH;
      if (NV % TH == 0 || e < NV) {
#pragma unroll
        for (int c = 0; c < CPV; ++c) {
          const int idx = e * CPV + c;
          const int x = idx / NXY;
          buf[x * NP + (idx - x * NXY)] = reinterpret_cast<const C*>(&v[u])[c];
        }
      }
    }
  }
  if (dc0 && tid < 32) dcf.finish(w);
  __syncthreads();
  smem_fft<NXY, NXY, TH, false, true, C, RL>(buf, NP, 1, s_tw);  // y, rows x
  if constexpr (FK && NXY > 1) {
    using RI = typename RLReverse<RL>::type;
    constexpr int RF = RLLast<RL>::value;
    smem_fft_head<NXY, RL, NXY, TH, false, true>(buf, 1, NP, s_tw);  // x, columns y
    XYKOp<T, NXY, RF> op;
    op.kx = w.kx;
    op.kyz = w.kyz;
    op.kz = kz;
    op.nzh = nzh;
    op.dc0 = dc0;
    fused_pass_pair<NXY, RF, NXY, TH, false, true, true>(buf, 1, NP, s_tw, op);
    smem_fft_tail<NXY, RI, NXY, TH, true, true>(buf, 1, NP, s_tw);
  } else {
    smem_fft<NXY, NXY, TH, false, true, C, RL>(buf, 1, NP, s_tw);
    for (int e = tid; e < NE; e += TH) {
      const int x = e / NXY;
      const int y = e - x * NXY;
      const T f = __ldg(w.kx + x) * __ldg(w.kyz + (size_t)y * nzh + kz);
      const C v = buf[x * NP + y];
      buf[x * NP + y] = (dc0 && e == 0) ? C{T(0), T(0)} : C{v.x * f, v.y * f};
    }
    __syncthreads();
    smem_fft<NXY, NXY, TH, true, true, C, RL>(buf, 1, NP, s_tw);
  }
  smem_fft<NXY, NXY, TH, true, true, C, RL>(buf, NP, 1, s_tw);  // inverse y
#pragma unroll
  for (int u = 0; u < UV; ++u) {
    const int e = tid + u * TH;
    if (NV % TH == 0 || e < NV) {
      V v;
#pragma unroll
      for (int c = 0; c < CPV; ++c) {
        const int idx = e * CPV + c;
        const int x = idx / NXY;
        reinterpret_cast<C*>(&v)[c] = buf[x * NP + (idx - x * NXY)];
      }
      reinterpret_cast<V*>(base)[e] = v;
    }
  }
}

template <typename T, int NXY, int TH, bool FK>
static cudaError_t launch_xy_t(const PencilWork<T>* d_works, int nworks, int nzh,
                               const c2_t<T>* tw, cudaStream_t st) {
  using C = c2_t<T>;
  const size_t smem = sizeof(C) * ((size_t)NXY * (NXY + 1) + NXY);
  auto kern = xy_kernel<T, NXY, TH, FK>;
  static unsigned attr_mask = 0;
  cudaError_t ea = ensure_smem_attr(kern, smem, &attr_mask);
  if (ea != cudaSuccess) return ea;
  dim3 grid(nzh, nworks);
  return launch_sweep_kernel(kern, grid, dim3(TH), smem, st, d_works, nzh, tw);
}

static const int kXYShapes[] = {8, 16, 32, 64, 96, 128};

bool xy_supported(int prec_bytes, int nx, int ny, int nz) {
  if (nx != ny || nz < 4 || !extent_supported(nz)) return false;
  bool listed = false;
  for (int s : kXYShapes) listed |= (s == nx);
  if (!listed) return false;
  const size_t bytes = (size_t)2 * prec_bytes * ((size_t)nx * (nx + 1) + nx);
  return bytes <= 200 * 1024;
}

#define PSB_XY_CASE(T, NXY, TH)                                                             \
  if (nx == NXY)                                                                            \
    return (variant & 2) ? launch_xy_t<T, NXY, TH, true>(d_works, nworks, nzh, tw, st)      \
                         : launch_xy_t<T, NXY, TH, false>(d_works, nworks, nzh, tw, st);

template <typename T>
cudaError_t launch_xy_impl(const PencilWork<T>* d_works, int nworks, int nx, int nzh,
                           const c2_t<T>* tw, int variant, cudaStream_t st) {
  PSB_XY_CASE(T, 8, 64)
  PSB_XY_CASE(T, 16, 128)
  PSB_XY_CASE(T, 32, 256)
  PSB_XY_CASE(T, 64, 512)
  PSB_XY_CASE(T, 96, 512)
  PSB_XY_CASE(T, 128, 1024)
  return cudaErrorInvalidValue;
}

template <typename T, int L, int TK, int TH, int MODE, bool FK>
static cudaError_t launch_pencil_t(const PencilWork<T>* d_works, int nworks, int outer, int inner,
                                   const c2_t<T>* tw, int nx, int ny, int nz, cudaStream_t st) {
  using C = c2_t<T>;
  const size_t smem = sizeof(C) * ((size_t)L * TK + (size_t)L);
  auto kern = pencil_kernel<T, L, TK, TH, MODE, FK>;
  static unsigned attr_mask = 0;
  cudaError_t ea = ensure_smem_attr(kern, smem, &attr_mask);
  if (ea != cudaSuccess) return ea;
  const int tiles = (inner + TK - 1) / TK;
  dim3 grid(outer * tiles, nworks);
  return launch_sweep_kernel(kern, grid, dim3(TH), smem, st, d_works, inner, tiles, tw, nx, ny, nz);
}

template <typename T, int L, int TK, int TH>
static cudaError_t launch_pencil_modes(const PencilWork<T>* d_works, int nworks, int mode, int outer,
                                       int inner, const c2_t<T>* tw, int nx, int ny, int nz,
                                       int variant, cudaStream_t st) {
  switch (mode) {
    case PENCIL_FWD:
      return launch_pencil_t<T, L, TK, TH, PENCIL_FWD, false>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_INV:
      return launch_pencil_t<T, L, TK, TH, PENCIL_INV, false>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_KINV:
      return (variant & 2)
                 ? launch_pencil_t<T, L, TK, TH, PENCIL_KINV, true>(d_works, nworks, outer, inner, tw,
                                                                    nx, ny, nz, st)
                 : launch_pencil_t<T, L, TK, TH, PENCIL_KINV, false>(d_works, nworks, outer, inner, tw,
                                                                     nx, ny, nz, st);
    case PENCIL_KFULL:
      return launch_pencil_t<T, L, TK, TH, PENCIL_KFULL, false>(d_works, nworks, outer, inner, tw, nx, ny, nz, st);
    case PENCIL_KFULL_IM:
      if constexpr (sizeof(T) == 8)
        return launch_pencil_t<T, L, TK, TH, PENCIL_KFULL_IM, false>(d_works, nworks, outer, inner, tw, nx, ny,
                                                                     nz, st);
      break;
    case PENCIL_KSPEC:
      if constexpr (sizeof(T) == 8)
        return launch_pencil_t<T, L, TK, TH, PENCIL_KSPEC, false>(d_works, nworks, outer, inner, tw, nx, ny,
                                                                  nz, st);
      break;
  }
  return cudaErrorInvalidValue;
}

// Tile widths: 256-byte rows (32 float2 or 16 double2 columns).
template <typename T> struct PencilTK { static constexpr int v = 32; };
template <> struct PencilTK<double> { static constexpr int v = 16; };

#define PSB_PENCIL_CASE(T, L, TH)                                                          \
  if (len == L)                                                                             \
    return launch_pencil_modes<T, L, PencilTK<T>::v, TH>(d_works, nworks, mode, outer, inner, tw, \
                                                         nx, ny, nz, variant, st);

template <typename T>
cudaError_t launch_pencil_impl(const PencilWork<T>* d_works, int nworks, int mode, int len,
                               int outer, int inner, const c2_t<T>* tw, int nx, int ny, int nz,
                               int variant, cudaStream_t st) {
  PSB_PENCIL_CASE(T, 1, 64)
  PSB_PENCIL_CASE(T, 4, 64)
  PSB_PENCIL_CASE(T, 8, 64)
  PSB_PENCIL_CASE(T, 12, 128)
  PSB_PENCIL_CASE(T, 16, 128)
  PSB_PENCIL_CASE(T, 24, 128)
  PSB_PENCIL_CASE(T, 32, 128)
  PSB_PENCIL_CASE(T, 48, 256)
  PSB_PENCIL_CASE(T, 64, 256)
  PSB_PENCIL_CASE(T, 96, 256)
  if (len == 128 && sizeof(T) == 4)
    return launch_pencil_modes<T, 128, 16, 128>(d_works, nworks, mode, outer, inner, tw, nx, ny, nz,
                                                variant, st);
  PSB_PENCIL_CASE(T, 128, 256)
  PSB_PENCIL_CASE(T, 256, 256)
  return cudaErrorInvalidValue;
}

// Explicit entry points.
template <>
cudaError_t launch_plane<float>(const PlaneWork<float>* w, int nw, int nx, int ny, int nz,
                                const float2* ty, const float2* tzh, const float2* tz,
                                int variant, cudaStream_t st) {
  return launch_plane_impl<float>(w, nw, nx, ny, nz, ty, tzh, tz, variant, st);
}
template <>
cudaError_t launch_plane<double>(const PlaneWork<double>* w, int nw, int nx, int ny, int nz,
                                 const double2* ty, const double2* tzh, const double2* tz,
                                 int variant, cudaStream_t st) {
  return launch_plane_impl<double>(w, nw, nx, ny, nz, ty, tzh, tz, variant, st);
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
cudaError_t launch_rows_t<float>(const PlaneWork<float>* w, int nw, int nx, int ny, int nz,
                                 const float2* tzh, const float2* tz, cudaStream_t st) {
  return launch_rows_t_impl<float>(w, nw, nx, ny, nz, tzh, tz, st);
}
template <>
cudaError_t launch_rows_t<double>(const PlaneWork<double>* w, int nw, int nx, int ny, int nz,
                                  const double2* tzh, const double2* tz, cudaStream_t st) {
  return launch_rows_t_impl<double>(w, nw, nx, ny, nz, tzh, tz, st);
}
template <>
cudaError_t launch_xy<float>(const PencilWork<float>* w, int nw, int nx, int nzh, const float2* tw,
                             int variant, cudaStream_t st) {
  return launch_xy_impl<float>(w, nw, nx, nzh, tw, variant, st);
}
template <>
cudaError_t launch_xy<double>(const PencilWork<double>* w, int nw, int nx, int nzh,
                              const double2* tw, int variant, cudaStream_t st) {
  return launch_xy_impl<double>(w, nw, nx, nzh, tw, variant, st);
}
template <>
cudaError_t launch_pencil<float>(const PencilWork<float>* w, int nw, int mode, int L, int outer,
                                 int inner, const float2* tw, int nx, int ny, int nz, int variant,
                                 cudaStream_t st) {
  return launch_pencil_impl<float>(w, nw, mode, L, outer, inner, tw, nx, ny, nz, variant, st);
}
template <>
cudaError_t launch_pencil<double>(const PencilWork<double>* w, int nw, int mode, int L, int outer,
                                  int inner, const double2* tw, int nx, int ny, int nz, int variant,
                                  cudaStream_t st) {
  return launch_pencil_impl<double>(w, nw, mode, L, outer, inner, tw, nx, ny, nz, variant, st);
}

}  // namespace psb

extern "C" int ps_gpu_set_bulk_wait_limit(unsigned int polls) {
  const uint32_t v = (polls == 0xFFFFFFFFu) ? psb::kMaxPolls : (uint32_t)polls;
  return cudaMemcpyToSymbol(psb::c_bulk_wait_polls, &v, sizeof(v)) == cudaSuccess ? PS_OK : PS_GPU_ERR;
}
