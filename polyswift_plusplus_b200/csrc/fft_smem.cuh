// Shared-memory Stockham FFT building blocks (radix 2, 3, 4, 8) for sm_100a.
//
// A CTA transforms a batch of B pencils of length L that sit in shared memory,
// element (b, i) at buf[b*bs + i*is].  Every pass keeps a single buffer: each
// thread pulls all of its butterfly inputs into registers, the CTA
// synchronises, then the butterflies are written back in Stockham order.  The
// output is in natural order.  Twiddles come from a table tw[m] =
// exp(-2 pi i m / L) computed on the host in FP64.
#pragma once

#include "common.cuh"

namespace psb {

// ---------------------------------------------------------------------------
// In-register DFTs of radix R (natural-order output).
// ---------------------------------------------------------------------------
template <int R, bool INV, typename C> struct Dft;

template <bool INV, typename C> struct Dft<1, INV, C> {
  static __device__ __forceinline__ void run(C*) {}
};

template <bool INV, typename C> struct Dft<2, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};

template <bool INV, typename C> struct Dft<3, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    using S = decltype(v[0].x);
    const S h = S(0.86602540378443864676);  // sqrt(3)/2
    C s = cadd(v[1], v[2]);
    C d = csub(v[1], v[2]);
    C y0 = cadd(v[0], s);
    C m = {v[0].x - S(0.5) * s.x, v[0].y - S(0.5) * s.y};
    C t = mul_mi<INV>(d);
    t = {h * t.x, h * t.y};
    v[0] = y0;
    v[1] = cadd(m, t);
    v[2] = csub(m, t);
  }
};

template <bool INV, typename C> struct Dft<4, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    C s0 = cadd(v[0], v[2]);
    C d0 = csub(v[0], v[2]);
    C s1 = cadd(v[1], v[3]);
    C d1 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(s0, s1);
    v[2] = csub(s0, s1);
    v[1] = cadd(d0, d1);
    v[3] = csub(d0, d1);
  }
};

template <bool INV, typename C> struct Dft<8, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    using S = decltype(v[0].x);
    const S c = S(0.70710678118654752440);  // sqrt(2)/2
    C a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      a[r] = cadd(v[r], v[r + 4]);
      b[r] = csub(v[r], v[r + 4]);
    }
    // b[r] *= w8^r (conjugated for the inverse)
    {
      C x = b[1];
      if (INV) b[1] = {c * (x.x - x.y), c * (x.x + x.y)};
      else     b[1] = {c * (x.x + x.y), c * (x.y - x.x)};
      b[2] = mul_mi<INV>(b[2]);
      x = b[3];
      if (INV) b[3] = {-c * (x.x + x.y), c * (x.x - x.y)};
      else     b[3] = {c * (x.y - x.x), -c * (x.x + x.y)};
    }
    Dft<4, INV, C>::run(a);
    Dft<4, INV, C>::run(b);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      v[2 * m] = a[m];
      v[2 * m + 1] = b[m];
    }
  }
};

// 16-point DFT as 4 x 4: radix-4 over n1 for each n2, twiddle w16^(n2 k1),
// radix-4 over n2; output index k1 + 4 k2.
template <bool INV, typename C> struct Dft<16, INV, C> {
  template <int M>
  static __device__ __forceinline__ C tw16(C x) {
    using S = decltype(x.x);
    constexpr int m = M % 16;
    if constexpr (m == 0) {
      return x;
    } else if constexpr (m == 4) {
      return mul_mi<INV>(x);
    } else {
      // w = (cos(pi m / 8), -sin(pi m / 8)), conjugated for the inverse
      const S c1 = S(0.92387953251128675613), s1 = S(0.38268343236508977173);
      const S c2 = S(0.70710678118654752440);
      S wr, wi;
      if constexpr (m == 1) { wr = c1; wi = -s1; }
      else if constexpr (m == 2) { wr = c2; wi = -c2; }
      else if constexpr (m == 3) { wr = s1; wi = -c1; }
      else if constexpr (m == 6) { wr = -c2; wi = -c2; }
      else { wr = -c1; wi = s1; }  // m == 9
      if (INV) wi = -wi;
      return C{x.x * wr - x.y * wi, x.x * wi + x.y * wr};
    }
  }
  static __device__ __forceinline__ void run(C* v) {
    C a[4][4];  // a[n2][k1]
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < 4; ++n1) a[n2][n1] = v[4 * n1 + n2];
      Dft<4, INV, C>::run(a[n2]);
    }
    a[1][1] = tw16<1>(a[1][1]);
    a[1][2] = tw16<2>(a[1][2]);
    a[1][3] = tw16<3>(a[1][3]);
    a[2][1] = tw16<2>(a[2][1]);
    a[2][2] = tw16<4>(a[2][2]);
    a[2][3] = tw16<6>(a[2][3]);
    a[3][1] = tw16<3>(a[3][1]);
    a[3][2] = tw16<6>(a[3][2]);
    a[3][3] = tw16<9>(a[3][3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      C b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      Dft<4, INV, C>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
    }
  }
};

// ---------------------------------------------------------------------------
// Radix plans.
// ---------------------------------------------------------------------------
template <int... Rs> struct RadixList {};

template <int L> struct Plan;  // RadixList of the passes, product = L
template <> struct Plan<1> { using type = RadixList<>; };
template <> struct Plan<2> { using type = RadixList<2>; };
template <> struct Plan<3> { using type = RadixList<3>; };
template <> struct Plan<4> { using type = RadixList<4>; };
template <> struct Plan<6> { using type = RadixList<2, 3>; };
template <> struct Plan<8> { using type = RadixList<8>; };
template <> struct Plan<12> { using type = RadixList<4, 3>; };
template <> struct Plan<16> { using type = RadixList<4, 4>; };
template <> struct Plan<24> { using type = RadixList<8, 3>; };
template <> struct Plan<32> { using type = RadixList<8, 4>; };
template <> struct Plan<48> { using type = RadixList<4, 4, 3>; };
template <> struct Plan<64> { using type = RadixList<8, 8>; };
template <> struct Plan<96> { using type = RadixList<8, 4, 3>; };
template <> struct Plan<128> { using type = RadixList<8, 4, 4>; };
template <> struct Plan<192> { using type = RadixList<8, 8, 3>; };
template <> struct Plan<256> { using type = RadixList<8, 8, 4>; };

// One Stockham pass: radix R, NS = product of the radices already applied.
// Thread t handles butterflies g = t + u*T.  BFAST selects the butterfly order:
// batch-fastest (columns, is > 1) or index-fastest (rows, is == 1).
template <int L, int R, int NS, int B, int T, bool INV, bool BFAST, typename C>
__device__ __forceinline__ void stockham_pass(C* buf, int bs, int is, const C* tw) {
  constexpr int M = L / R;       // butterflies per pencil
  constexpr int NB = B * M;      // butterflies in the batch
  constexpr int U = (NB + T - 1) / T;
  constexpr int TS = L / (NS * R);
  C v[U][R];
  const int t = threadIdx.x;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int g = t + u * T;
    if ((NB % T) == 0 || g < NB) {
      const int b = BFAST ? (g % B) : (g / M);
      const int j = BFAST ? (g / B) : (g % M);
      const C* base = buf + b * bs;
#pragma unroll
      for (int r = 0; r < R; ++r) v[u][r] = base[(j + r * M) * is];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int g = t + u * T;
    if ((NB % T) == 0 || g < NB) {
      const int b = BFAST ? (g % B) : (g / M);
      const int j = BFAST ? (g / B) : (g % M);
      const int k = j % NS;
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C w = tw[r * k * TS];
          v[u][r] = INV ? cmulc(v[u][r], w) : cmul(v[u][r], w);
        }
      }
      Dft<R, INV, C>::run(v[u]);
      C* base = buf + b * bs;
      const int d = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(d + r * NS) * is] = v[u][r];
    }
  }
  __syncthreads();
}

template <int L, int NS, typename RL> struct Passes;
template <int L, int NS> struct Passes<L, NS, RadixList<>> {
  template <int B, int T, bool INV, bool BFAST, typename C>
  static __device__ __forceinline__ void run(C*, int, int, const C*) {}
};
template <int L, int NS, int R, int... Rest> struct Passes<L, NS, RadixList<R, Rest...>> {
  template <int B, int T, bool INV, bool BFAST, typename C>
  static __device__ __forceinline__ void run(C* buf, int bs, int is, const C* tw) {
    stockham_pass<L, R, NS, B, T, INV, BFAST>(buf, bs, is, tw);
    Passes<L, NS * R, RadixList<Rest...>>::template run<B, T, INV, BFAST>(buf, bs, is, tw);
  }
};

// Batched FFT of B pencils of length L in shared memory (radix plan RL).
template <int L, int B, int T, bool INV, bool BFAST, typename C, typename RL = typename Plan<L>::type>
__device__ __forceinline__ void smem_fft(C* buf, int bs, int is, const C* tw) {
  Passes<L, 1, RL>::template run<B, T, INV, BFAST>(buf, bs, is, tw);
}

// ---------------------------------------------------------------------------
// Radix-list utilities.
// ---------------------------------------------------------------------------
template <int R, typename RL> struct RLPrepend;
template <int R, int... Rs> struct RLPrepend<R, RadixList<Rs...>> { using type = RadixList<R, Rs...>; };
template <typename RL, int R> struct RLAppend;
template <int... Rs, int R> struct RLAppend<RadixList<Rs...>, R> { using type = RadixList<Rs..., R>; };
template <typename RL> struct RLReverse;
template <> struct RLReverse<RadixList<>> { using type = RadixList<>; };
template <int R, int... Rs> struct RLReverse<RadixList<R, Rs...>> {
  using type = typename RLAppend<typename RLReverse<RadixList<Rs...>>::type, R>::type;
};
template <typename RL> struct RLFirst;
template <int R, int... Rs> struct RLFirst<RadixList<R, Rs...>> {
  static constexpr int value = R;
  using rest = RadixList<Rs...>;
};
template <typename RL> struct RLLast;
template <int R> struct RLLast<RadixList<R>> {
  static constexpr int value = R;
  using init = RadixList<>;
};
template <int R, int R2, int... Rs> struct RLLast<RadixList<R, R2, Rs...>> {
  static constexpr int value = RLLast<RadixList<R2, Rs...>>::value;
  using init = typename RLPrepend<R, typename RLLast<RadixList<R2, Rs...>>::init>::type;
};

// All passes of plan RL except the last (starting at NS = 1).
template <int L, typename RL, int B, int T, bool INV, bool BFAST, typename C>
__device__ __forceinline__ void smem_fft_head(C* buf, int bs, int is, const C* tw) {
  Passes<L, 1, typename RLLast<RL>::init>::template run<B, T, INV, BFAST>(buf, bs, is, tw);
}
// All passes of plan RL except the first (starting at NS = first radix).
template <int L, typename RL, int B, int T, bool INV, bool BFAST, typename C>
__device__ __forceinline__ void smem_fft_tail(C* buf, int bs, int is, const C* tw) {
  Passes<L, RLFirst<RL>::value, typename RLFirst<RL>::rest>::template run<B, T, INV, BFAST>(buf, bs,
                                                                                          is, tw);
}

// The last pass (radix R, NS = L/R) of an FFT in direction INV_A, an
// elementwise operation in registers, and the first pass (radix R, NS = 1) of
// an FFT in direction INV_B, as one shared-memory round trip.  With the same
// radix both passes give a thread's butterfly j the elements j + r*L/R.
// op.apply(b, j, v) receives pencil b's values v[r] at natural positions
// j + r*L/R; op.after(b, s) then receives output 0 of the second DFT (the sum
// of the values apply left).
template <int L, int R, int B, int T, bool INV_A, bool INV_B, bool BFAST, typename C, typename OP>
__device__ __forceinline__ void fused_pass_pair(C* buf, int bs, int is, const C* tw, OP& op) {
  constexpr int M = L / R;
  constexpr int NB = B * M;
  constexpr int U = (NB + T - 1) / T;
  C v[U][R];
  const int t = threadIdx.x;
  // the first butterfly's operand loads (global memory) are issued before the
  // shared-memory reads and the barrier, so their latency overlaps them
  if ((NB % T) == 0 || t < NB) op.prefetch(BFAST ? (t % B) : (t / M), BFAST ? (t / B) : (t % M));
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int g = t + u * T;
    if ((NB % T) == 0 || g < NB) {
      const int b = BFAST ? (g % B) : (g / M);
      const int j = BFAST ? (g / B) : (g % M);
      const C* base = buf + b * bs;
#pragma unroll
      for (int r = 0; r < R; ++r) v[u][r] = base[(j + r * M) * is];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int g = t + u * T;
    if ((NB % T) == 0 || g < NB) {
      const int b = BFAST ? (g % B) : (g / M);
      const int j = BFAST ? (g / B) : (g % M);
      if (u > 0) op.prefetch(b, j);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const C w = tw[r * j];
        v[u][r] = INV_A ? cmulc(v[u][r], w) : cmul(v[u][r], w);
      }
      Dft<R, INV_A, C>::run(v[u]);
      op.apply(b, j, v[u]);
      Dft<R, INV_B, C>::run(v[u]);
      op.after(b, v[u][0]);  // output 0 of the second DFT: the sum of its inputs
      C* base = buf + b * bs;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(j * R + r) * is] = v[u][r];
    }
  }
  __syncthreads();
}

// Fewer, wider passes for the pencil kernel (more values per thread).
template <int L> struct WidePlan { using type = typename Plan<L>::type; };
template <> struct WidePlan<64> { using type = RadixList<16, 4>; };
template <> struct WidePlan<128> { using type = RadixList<16, 8>; };
template <> struct WidePlan<256> { using type = RadixList<16, 16>; };

}  // namespace psb
