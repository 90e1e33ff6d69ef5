// Adjoint of the propagator sweeps of one linear block copolymer (FP64).
//
// Forward:  q_{s+1} = wf_s * G_s(wf_s * q_s) along the chain (sweep 0, from
// block 0's free head) and q+ the same way from the other end (sweep 1);
// phi_f = (1/Q) sum_blocks densfac ds_b sum_n c_n q_n q+_{M-n} with the
// reference's quadrature weights (pspolymer/PsBlock.cpp:256-380) and
// Q = <q_head q+_end> of block 0 (pspolymer/PsBlock.cpp:205-237).  wf_s =
// exp(-ds_b w_f/2) and G_s = IFFT exp(-ds_b b^2 k^2) FFT / N for the block b
// of step s, as in pspolymer/PsFlexPseudoSpec.cpp:158-293.
//
// Backward, for a loss L(phi, ln Q): G is a real symmetric convolution, so the
// transpose of a step is the step itself and the adjoint of each sweep is one
// more sweep run backwards with sources from the quadrature:
//   lam_s = wf_s G_s(wf_s lam_{s+1}) + dL/dq_s (explicit),
//   dL/dw_f      += -ds_b/2 (lam_{s+1} q_{s+1} + q_s mu_s),   mu_s = wf G(wf lam_{s+1}),
//   dL/dL_d      += (2 ds_b b^2 / L_d) R_d,   R_d = (1/N) sum_k conj(U) V K k_d^2,
//   dL/d(ds_b)   += -b^2 sum_d R_d - 1/2 <w_f, lam_{s+1} q_{s+1} + q_s mu_s>,
// with U = FFT(wf lam_{s+1}), V = FFT(wf q_s), plus the explicit ds factor of
// the quadrature weights.  L_d are the box lengths n_d * cell_d.
//
// Storage: the slices of both sweeps are checkpointed every C contour steps
// (C = 1: full storage; C ~ sqrt(M): square-root checkpointing).  Segment j of
// sweep 0 covers n in [jC, min((j+1)C, M)]; the matching part of sweep 1
// (m = M - n) starts at a checkpoint placed at m = M - min((j+1)C, M), so both
// halves of a segment are recomputed from one checkpoint each into two
// (C+1)-slice buffers, and the recomputed slices equal the stored ones bit for
// bit.  The quadrature and each adjoint sweep recompute the segments once.
//
// Branched (tree) chains keep every slice of every sweep (no checkpoints): the
// forward is the engine's own sweeps with junction products, and the adjoint
// sweeps run in reverse dependency order.  A sweep that starts at a junction,
// q_0 = prod_j q^(j)_end, hands its lam_0 back to each arriving sweep's end:
// lam^(j)_end += lam_0 prod_{j' != j} q^(j')_end, before that sweep's adjoint
// starts.
//
// Every launch and descriptor is fixed at creation; reductions use a fixed
// grid and are summed on the host in a fixed order, so results are
// deterministic.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <string>
#include <vector>

#include "engine_state.h"

namespace psb {

constexpr int kAdjRB = 296;
constexpr int kAdjRT = 256;

struct AccumEntry {
  double* dst;
  const double* x;
  const double* y;
  double coef;
};

struct SrcEntry {
  const double* gphi;
  const double* partner;
  double coef;  // without the 1/Q factor
};

struct AdjPoint {
  const double* mu;
  const double* lam_next;
  const double* q_s;
  const double* q_next;
  const double* w;
  double* gwb;
  double* lam_out;   // nullptr: lambda_s is not needed (s = 0)
  double* dsw_part;  // kAdjRB partials
  double half_ds;
  int n_src;
  SrcEntry src[2];
  const double* q_partner;  // Q source partner (nullptr: none at this slice)
  const double* extra;      // adj_init only: junction contributions to lambda (nullptr: none)
  const double* psi;        // charged block: the exponent is w + facz psi (nullptr: w alone)
  double facz;
};

// lam_out[j] += lam0 * prod_{i != j} q_in[i] for the sweeps arriving at a
// junction (the adjoint of the junction product).
struct JunctionAdj {
  const double* lam0;
  int n;
  const double* q_in[PS_MAX_JOINS];
  double* lam_out[PS_MAX_JOINS];
};

struct BlockFieldMap {
  int nb, nf;
  int field[PS_MAX_BLOCKS];
};

__device__ __forceinline__ double adj_block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = kAdjRT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

#define ADJ_LOOP(r, N) \
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < (N); r += (long long)gridDim.x * blockDim.x)

__global__ void adj_accum_kernel(const AccumEntry* __restrict__ e, int ne, long long N) {
  ADJ_LOOP(r, N) {
    for (int i = 0; i < ne; ++i) {
      const AccumEntry a = e[i];
      a.dst[r] += a.coef * a.x[r] * a.y[r];
    }
  }
}

__global__ void adj_normalize_kernel(double* __restrict__ P, double* __restrict__ phi, BlockFieldMap m,
                                     long long N, const DevScalars* __restrict__ sc) {
  const double inv_q = 1.0 / sc->q[0];
  ADJ_LOOP(r, N) {
    double acc[PS_MAX_FIELDS] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < m.nb; ++b) {
      const double v = P[(size_t)b * N + r] * inv_q;
      P[(size_t)b * N + r] = v;
      acc[m.field[b]] += v;
    }
    for (int f = 0; f < m.nf; ++f) phi[(size_t)f * N + r] = acc[f];
  }
}

__global__ void adj_dot_kernel(const double* __restrict__ a, const double* __restrict__ b, long long n,
                               double* __restrict__ part) {
  __shared__ double sh[kAdjRT];
  double acc = 0.0;
  ADJ_LOOP(r, n) acc += a[r] * b[r];
  acc = adj_block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// dL/dQ = g_lnQ / Q - (1/Q) sum_f <g_phi_f, phi_f>  (phi carries 1/Q).
__global__ void adj_gq_kernel(const double* __restrict__ part, double g_lnq, const DevScalars* __restrict__ sc,
                              double* __restrict__ gq) {
  __shared__ double sh[kAdjRT];
  double acc = 0.0;
  for (int i = threadIdx.x; i < kAdjRB; i += blockDim.x) acc += part[i];
  acc = adj_block_sum(acc, sh);
  if (threadIdx.x == 0) {
    const double q = sc->q[0];
    *gq = g_lnq / q - acc / q;
  }
}

__global__ void adj_kmul_kernel(double2* __restrict__ spec, const double* __restrict__ kx,
                                const double* __restrict__ kyz, int nx, int inner) {
  const long long n = (long long)nx * inner;
  ADJ_LOOP(i, n) {
    const int x = (int)(i / inner);
    const int c = (int)(i - (long long)x * inner);
    const double f = kx[x] * kyz[c];
    const double2 v = spec[i];
    spec[i] = make_double2(v.x * f, v.y * f);
  }
}

__device__ __forceinline__ double adj_kcomp(int i, int n, double dx) {
  const double n2 = (double)n / 2.0;
  const double nk = n2 - fabs((double)i - n2);
  return 2.0 * 3.14159265358979323846 * nk / ((double)n * dx);
}

// R_d = sum over the half spectrum (weight 2 off the kz = 0 / nz/2 planes) of
// Re(conj(U) V) * kx*kyz * k_d^2; kx carries 1/N.
__global__ void adj_stress_kernel(const double2* __restrict__ U, const double2* __restrict__ V,
                                  const double* __restrict__ kx, const double* __restrict__ kyz, int nx,
                                  int ny, int nz, double dx, double dy, double dz, double* __restrict__ part) {
  __shared__ double sh[kAdjRT];
  const int nzh = nz / 2 + 1;
  const long long n = (long long)nx * ny * nzh;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  ADJ_LOOP(i, n) {
    const int x = (int)(i / ((long long)ny * nzh));
    const int rem = (int)(i - (long long)x * ny * nzh);
    const int y = rem / nzh;
    const int kz = rem - y * nzh;
    const double mult = (kz == 0 || (2 * kz == nz)) ? 1.0 : 2.0;
    const double2 u = U[i], v = V[i];
    const double t = mult * (u.x * v.x + u.y * v.y) * kx[x] * kyz[rem];
    const double k0 = adj_kcomp(x, nx, dx), k1 = adj_kcomp(y, ny, dy), k2 = adj_kcomp(kz, nz, dz);
    a0 += t * k0 * k0;
    a1 += t * k1 * k1;
    a2 += t * k2 * k2;
  }
  a0 = adj_block_sum(a0, sh);
  a1 = adj_block_sum(a1, sh);
  a2 = adj_block_sum(a2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = a0;
    part[kAdjRB + blockIdx.x] = a1;
    part[2 * kAdjRB + blockIdx.x] = a2;
  }
}

__global__ void adj_init_kernel(const AdjPoint* __restrict__ pp, long long N, const DevScalars* __restrict__ sc,
                                const double* __restrict__ gq) {
  const AdjPoint p = *pp;
  const double inv_q = 1.0 / sc->q[0];
  const double gqn = p.q_partner ? (*gq) / (double)N : 0.0;
  ADJ_LOOP(r, N) {
    double s = 0.0;
    for (int i = 0; i < p.n_src; ++i) s += p.src[i].coef * p.src[i].gphi[r] * p.src[i].partner[r];
    double l = inv_q * s;
    if (p.q_partner) l += gqn * p.q_partner[r];
    if (p.extra) l += p.extra[r];
    p.lam_out[r] = l;
  }
}

__global__ void adj_axpy_kernel(double* __restrict__ dst, const double* __restrict__ x, double coef, long long N) {
  ADJ_LOOP(r, N) dst[r] += coef * x[r];
}

__global__ void adj_junction_kernel(const JunctionAdj* __restrict__ jp, long long N) {
  const JunctionAdj j = *jp;
  ADJ_LOOP(r, N) {
    const double l = j.lam0[r];
    for (int i = 0; i < j.n; ++i) {
      double v = l;
      for (int k = 0; k < j.n; ++k)
        if (k != i) v *= j.q_in[k][r];
      j.lam_out[i][r] += v;
    }
  }
}

__global__ void adj_point_kernel(const AdjPoint* __restrict__ pp, long long N, const DevScalars* __restrict__ sc,
                                 const double* __restrict__ gq) {
  __shared__ double sh[kAdjRT];
  const AdjPoint p = *pp;
  const double inv_q = 1.0 / sc->q[0];
  const double gqn = p.q_partner ? (*gq) / (double)N : 0.0;
  double acc = 0.0;
  ADJ_LOOP(r, N) {
    const double t = p.lam_next[r] * p.q_next[r] + p.q_s[r] * p.mu[r];
    p.gwb[r] += -p.half_ds * t;
    const double x = p.psi ? p.w[r] + p.facz * p.psi[r] : p.w[r];
    acc += x * (-0.5 * t);
    if (p.lam_out) {
      double s = 0.0;
      for (int i = 0; i < p.n_src; ++i) s += p.src[i].coef * p.src[i].gphi[r] * p.src[i].partner[r];
      double l = p.mu[r] + inv_q * s;
      if (p.q_partner) l += gqn * p.q_partner[r];
      p.lam_out[r] = l;
    }
  }
  acc = adj_block_sum(acc, sh);
  if (threadIdx.x == 0) p.dsw_part[blockIdx.x] = acc;
}

__global__ void adj_sum_blocks_kernel(const double* __restrict__ gwb, BlockFieldMap m, long long N,
                                      double* __restrict__ gw) {
  ADJ_LOOP(r, N) {
    double acc[PS_MAX_FIELDS] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < m.nb; ++b) acc[m.field[b]] += gwb[(size_t)b * N + r];
    for (int f = 0; f < m.nf; ++f) gw[(size_t)f * N + r] = acc[f];
  }
}

// Quadrature weight of local slice n of a block with `steps` steps, without ds
// (PsBlock::setCalcQQTIntegral: extended Simpson with 0.33333, trapezoid on the
// last interval when the point count is even).
static std::vector<double> quad_weights(int steps) {
  const int num = steps + 1;
  const int npts = num - 1;
  const bool even = (num % 2) == 0;
  const int numstail = even ? npts - 3 : npts - 2;
  std::vector<double> c(num, 0.0);
  for (int n = 0; n <= numstail; n += 2) {
    c[n] += 0.33333;
    c[n + 1] += 4.0 * 0.33333;
    c[n + 2] += 0.33333;
  }
  if (even) {
    c[num - 2] += 0.5;
    c[num - 1] += 0.5;
  }
  return c;
}

}  // namespace psb

using Op = std::function<cudaError_t(cudaStream_t)>;

struct ps_adj {
  ps_handle* h = nullptr;
  std::string err;
  int ip = 0;  // the polymer of the configuration this adjoint differentiates
  int M = 0, C = 1, J = 0, nb = 0, nf = 0;
  long long N = 0;
  int n0 = 0;  // sweep-0 index of block 0's head slice (Q = <q_n0 q+_{M-n0}>)
  std::vector<int> blk[2];
  std::vector<int> seg_a, seg_b;
  std::vector<std::vector<std::pair<int, double>>> quad;  // per n: (block, densfac ds c)
  double* ck[2] = {nullptr, nullptr};
  double* endq[2] = {nullptr, nullptr};
  double* seg[2] = {nullptr, nullptr};
  double* lam[2] = {nullptr, nullptr};
  double* mu = nullptr;
  double2* spec[2] = {nullptr, nullptr};
  double* P = nullptr;
  double* gwb = nullptr;
  double* gphi = nullptr;
  double* gq = nullptr;
  double* part = nullptr;
  double* h_part = nullptr;
  size_t part_len = 0;
  std::vector<int> slot_block;
  psb::PlaneWork<double>* d_pw = nullptr;
  psb::PencilWork<double>* d_xw = nullptr;
  psb::AccumEntry* d_acc = nullptr;
  psb::AdjPoint* d_pt = nullptr;
  std::vector<psb::PlaneWork<double>> h_pw;
  std::vector<psb::PencilWork<double>> h_xw;
  std::vector<psb::AccumEntry> h_acc;
  std::vector<psb::AdjPoint> h_pt;
  std::vector<Op> fwd, bwd;
  // branched chains: the polymer's executed sweeps (h->sweeps indices, in
  // dependency order), the steps' blocks, junction accumulators, descriptors
  bool tree = false;
  std::vector<int> tsw;
  std::vector<std::vector<int>> tblk;
  std::vector<double*> jacc;
  std::vector<psb::JunctionAdj> h_jn;
  psb::JunctionAdj* d_jn = nullptr;
  size_t storage_bytes = 0;
  size_t E_off = 0, gq_off = 0;  // offsets (in doubles) into part
  bool have_forward = false;
  bool have_backward = false;
};

namespace psb {

#define PA_CUDA(a, call)                                                 \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      (a)->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
      return PS_GPU_ERR;                                                 \
    }                                                                    \
  } while (0)

static thread_local std::string g_adj_err;

// Program builder: descriptors go to host tables (uploaded once), ops refer to
// them by offset.
struct Builder {
  ps_adj* a;
  ps_handle* h;
  int nx, ny, nz, nzh;
  bool fused;

  const double* wf(int b) const {
    const BlockMap& bm = h->blocks[a->ip][b];
    for (size_t i = 0; i < h->wfac_keys.size(); ++i) {
      const WfacKey& k = h->wfac_keys[i];
      if (k.field == bm.field && k.ds == bm.ds && k.charge_field == bm.charge_field &&
          (bm.charge_field < 0 || k.facz == bm.facz))
        return h->bd.wfac[i];
    }
    return nullptr;
  }
  int ktab(int b) const {
    const BlockMap& bm = h->blocks[a->ip][b];
    for (size_t i = 0; i < h->ktab_keys.size(); ++i)
      if (h->ktab_keys[i].first == bm.ds && h->ktab_keys[i].second == bm.bseg) return (int)i;
    return 0;
  }
  size_t plane(const PlaneWork<double>& w) {
    a->h_pw.push_back(w);
    return a->h_pw.size() - 1;
  }
  size_t pencil(const PencilWork<double>& w) {
    a->h_xw.push_back(w);
    return a->h_xw.size() - 1;
  }
  PlaneWork<double> pw(int mode, const double* src, double2* spec, const double* win, const double* wout,
                       double* store) {
    PlaneWork<double> w;
    memset(&w, 0, sizeof(w));
    w.mode = mode;
    w.src = src;
    w.spec = spec;
    w.wfac_in = win;
    w.wfac_out = wout;
    w.store = store;
    w.status = &h->d_sc->error_flags;
    return w;
  }
  PencilWork<double> xw(double2* spec, int b) {
    PencilWork<double> x;
    memset(&x, 0, sizeof(x));
    x.spec = spec;
    if (b >= 0) {
      x.kx = h->bd.kx[ktab(b)];
      x.kyz = h->bd.kyz[ktab(b)];
    }
    return x;
  }
  // Real-space plane pass (rows + y pencils on grids without the fused design):
  // MODE_FIRST / MID end with the forward y-z transform; MID / LAST start with
  // the inverse one.
  void real_pass(std::vector<Op>& ops, size_t pw0, int n, size_t yx0, int mode) {
    ps_adj* A = a;
    const int nx_ = nx, ny_ = ny, nz_ = nz, nzh_ = nzh;
    ps_handle* H = h;
    if (fused) {
      ops.push_back([=](cudaStream_t st) {
        return launch_plane<double>(A->d_pw + pw0, n, nx_, ny_, nz_, H->bd.tw_y, H->bd.tw_zh, H->bd.tw_z, 0, st);
      });
      return;
    }
    if (mode != MODE_FIRST && ny > 1)
      ops.push_back([=](cudaStream_t st) {
        return launch_pencil<double>(A->d_xw + yx0, n, PENCIL_INV, ny_, nx_, nzh_, H->bd.tw_y, nx_, ny_, nz_, 0, st);
      });
    ops.push_back([=](cudaStream_t st) {
      return launch_rows<double>(A->d_pw + pw0, n, nx_ * ny_, nz_, H->bd.tw_zh, H->bd.tw_z, st);
    });
    if (mode != MODE_LAST && ny > 1)
      ops.push_back([=](cudaStream_t st) {
        return launch_pencil<double>(A->d_xw + yx0, n, PENCIL_FWD, ny_, nx_, nzh_, H->bd.tw_y, nx_, ny_, nz_, 0, st);
      });
  }
  void x_pass(std::vector<Op>& ops, size_t x0, int n, int mode) {
    ps_adj* A = a;
    const int nx_ = nx, ny_ = ny, nz_ = nz, inner = ny * nzh;
    ps_handle* H = h;
    ops.push_back([=](cudaStream_t st) {
      return launch_pencil<double>(A->d_xw + x0, n, mode, nx_, 1, inner, H->bd.tw_x, nx_, ny_, nz_, 0, st);
    });
  }
  // Lockstep sweeps over `len` steps.  Sweep i runs steps s0[i] .. s0[i]+len-1
  // of sweep sig[i] from slice src[i] (nullptr: ones); store(i, k) gives the
  // destination of its slice k (nullptr: not stored).
  void sweeps(std::vector<Op>& ops, int nsw, const int* sig, const int* s0, const double* const* src, int len,
              const std::function<double*(int, int)>& store) {
    for (int k = 0; k <= len; ++k) {
      const int mode = (k == 0) ? MODE_FIRST : (k == len ? MODE_LAST : MODE_MID);
      size_t p0 = 0, y0 = 0;
      for (int i = 0; i < nsw; ++i) {
        const std::vector<int>& bl = a->blk[sig[i]];
        const double* win = (k > 0) ? wf(bl[s0[i] + k - 1]) : nullptr;
        const double* wout = (k < len) ? wf(bl[s0[i] + k]) : nullptr;
        const size_t p = plane(pw(mode, k == 0 ? src[i] : nullptr, a->spec[i], win, wout, store(i, k)));
        const size_t y = pencil(xw(a->spec[i], -1));
        if (i == 0) {
          p0 = p;
          y0 = y;
        }
      }
      real_pass(ops, p0, nsw, y0, mode);
      if (k < len) {
        size_t x0 = 0;
        for (int i = 0; i < nsw; ++i) {
          const size_t x = pencil(xw(a->spec[i], a->blk[sig[i]][s0[i] + k]));
          if (i == 0) x0 = x;
        }
        x_pass(ops, x0, nsw, PENCIL_KINV);
      }
    }
  }
};

// Slice idx of sweep sig while segment j is resident.
static double* slice_ptr(ps_adj* a, int sig, int idx, int j) {
  const long long N = a->N;
  if (a->C == 1) {
    if (sig == 0) return (idx == a->M) ? a->endq[0] : a->ck[0] + (size_t)idx * N;
    return (idx == a->M) ? a->endq[1] : a->ck[1] + (size_t)(a->M - 1 - idx) * N;
  }
  if (sig == 0) return a->seg[0] + (size_t)(idx - a->seg_a[j]) * N;
  return a->seg[1] + (size_t)(idx - (a->M - a->seg_b[j])) * N;
}

static void recompute(Builder& B, std::vector<Op>& ops, int j) {
  ps_adj* a = B.a;
  if (a->C == 1) return;
  const int sig[2] = {0, 1};
  const int s0[2] = {a->seg_a[j], a->M - a->seg_b[j]};
  const double* src[2] = {a->ck[0] + (size_t)j * a->N, a->ck[1] + (size_t)j * a->N};
  const int len = a->seg_b[j] - a->seg_a[j];
  B.sweeps(ops, 2, sig, s0, src, len, [a](int i, int k) { return a->seg[i] + (size_t)k * a->N; });
}

// Sources of slice idx of sweep sig: every quadrature pair it belongs to, and Q.
static void fill_sources(ps_adj* a, AdjPoint& p, int sig, int idx, int j) {
  const int n = (sig == 0) ? idx : a->M - idx;
  p.n_src = 0;
  for (auto& e : a->quad[n]) {
    const int f = a->h->blocks[a->ip][e.first].field;
    SrcEntry s;
    s.gphi = a->gphi + (size_t)f * a->N;
    s.partner = slice_ptr(a, 1 - sig, a->M - idx, j);
    s.coef = e.second;
    p.src[p.n_src++] = s;
  }
  const int qslice = (sig == 0) ? a->n0 : a->M - a->n0;
  p.q_partner = (idx == qslice) ? slice_ptr(a, 1 - sig, a->M - idx, j) : nullptr;
}

// One adjoint step through block b: mu = wf G(wf lam_next), the stress
// partials of (U, V) = (FFT(wf lam_next), FFT(wf q_s)), dL/dw of the step and,
// when lam_out is set, lam_s = mu + the explicit sources of slice s (in `src`).
static void adjoint_step_p(Builder& B, std::vector<Op>& ops, int b, const double* q_s, const double* q_next,
                           const double* lam_next, double* lam_out, const AdjPoint& src) {
  ps_adj* a = B.a;
  ps_handle* h = B.h;
  const double* wfb = B.wf(b);
  const BlockMap& bm = h->blocks[a->ip][b];
  const int slot = (int)a->slot_block.size();
  a->slot_block.push_back(b);
  // U = FFT(wf lam_{s+1}) in spec[0], V = FFT(wf q_s) in spec[1]
  const size_t p0 = B.plane(B.pw(MODE_FIRST, lam_next, a->spec[0], nullptr, wfb, nullptr));
  B.plane(B.pw(MODE_FIRST, q_s, a->spec[1], nullptr, wfb, nullptr));
  const size_t y0 = B.pencil(B.xw(a->spec[0], -1));
  B.pencil(B.xw(a->spec[1], -1));
  B.real_pass(ops, p0, 2, y0, MODE_FIRST);
  const size_t x0 = B.pencil(B.xw(a->spec[0], -1));
  B.pencil(B.xw(a->spec[1], -1));
  B.x_pass(ops, x0, 2, PENCIL_FWD);
  const int kt = B.ktab(b);
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const double dx = h->cfg.cell[0], dy = h->cfg.cell[1], dz = h->cfg.cell[2];
  const size_t poff = (size_t)slot * 4 * kAdjRB;
  ops.push_back([=](cudaStream_t st) {
    adj_stress_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->spec[0], a->spec[1], h->bd.kx[kt], h->bd.kyz[kt], nx, ny,
                                                   nz, dx, dy, dz, a->part + poff);
    return cudaGetLastError();
  });
  const int inner = ny * B.nzh;
  ops.push_back([=](cudaStream_t st) {
    adj_kmul_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->spec[0], h->bd.kx[kt], h->bd.kyz[kt], nx, inner);
    return cudaGetLastError();
  });
  const size_t x1 = B.pencil(B.xw(a->spec[0], -1));
  B.x_pass(ops, x1, 1, PENCIL_INV);
  const size_t p1 = B.plane(B.pw(MODE_LAST, nullptr, a->spec[0], wfb, nullptr, a->mu));
  const size_t y1 = B.pencil(B.xw(a->spec[0], -1));
  B.real_pass(ops, p1, 1, y1, MODE_LAST);
  AdjPoint p = src;
  p.mu = a->mu;
  p.lam_next = lam_next;
  p.q_s = q_s;
  p.q_next = q_next;
  p.w = h->d_w + (size_t)bm.field * a->N;
  p.gwb = a->gwb + (size_t)b * a->N;
  p.lam_out = lam_out;
  p.dsw_part = a->part + poff + 3 * kAdjRB;
  p.half_ds = 0.5 * bm.ds;
  p.extra = nullptr;
  p.psi = (bm.charge_field >= 0) ? h->d_psi + (size_t)bm.charge_field * a->N : nullptr;
  p.facz = bm.facz;
  a->h_pt.push_back(p);
  const size_t pi = a->h_pt.size() - 1;
  const long long N = a->N;
  ops.push_back([=](cudaStream_t st) {
    adj_point_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_pt + pi, N, h->d_sc, a->gq);
    return cudaGetLastError();
  });
}

static void adjoint_step(Builder& B, std::vector<Op>& ops, int sig, int s, int j, int cur) {
  ps_adj* a = B.a;
  AdjPoint src;
  memset(&src, 0, sizeof(src));
  if (s >= 1) fill_sources(a, src, sig, s, j);
  adjoint_step_p(B, ops, a->blk[sig][s], slice_ptr(a, sig, s, j), slice_ptr(a, sig, s + 1, j), a->lam[cur],
                 (s >= 1) ? a->lam[1 - cur] : nullptr, src);
}

static void adjoint_init(ps_adj* a, std::vector<Op>& ops, int sig, int j, int cur) {
  AdjPoint p;
  memset(&p, 0, sizeof(p));
  p.lam_out = a->lam[cur];
  fill_sources(a, p, sig, a->M, j);
  a->h_pt.push_back(p);
  const size_t pi = a->h_pt.size() - 1;
  const long long N = a->N;
  ps_handle* h = a->h;
  ops.push_back([=](cudaStream_t st) {
    adj_init_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_pt + pi, N, h->d_sc, a->gq);
    return cudaGetLastError();
  });
}

template <typename T>
static int adj_upload(ps_adj* a, T** dst, const std::vector<T>& v) {
  PA_CUDA(a, cudaMalloc((void**)dst, sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty()) PA_CUDA(a, cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return PS_OK;
}

static BlockFieldMap field_map(ps_adj* a) {
  BlockFieldMap fm;
  memset(&fm, 0, sizeof(fm));
  fm.nb = a->nb;
  fm.nf = a->nf;
  for (int b = 0; b < a->nb; ++b) fm.field[b] = a->h->blocks[a->ip][b].field;
  return fm;
}


// Branched chain (see the header): every slice stored by the engine's sweeps.
static int tree_build(ps_adj* a, int ec) {
  ps_handle* h = a->h;
  const int ip = ec;  // the engine's (expanded) polymer index
  a->tree = true;
  a->C = 1;
  a->J = 0;
  a->N = h->N;
  a->nf = h->nf;
  a->nb = (int)h->blocks[ip].size();
  const long long N = a->N;
  std::vector<int> pos(h->sweeps.size(), -1);  // h->sweeps index -> position in tsw
  for (int e : h->exec)
    if (h->sweeps[e].polymer == ip) {
      pos[e] = (int)a->tsw.size();
      a->tsw.push_back(e);
    }
  const int ns = (int)a->tsw.size();
  auto S = [h](int sweep, int idx) -> double* {
    return h->bd.slices[h->sweeps[sweep].storage] + (size_t)idx * h->N;
  };
  int steps_total = 0;
  size_t slice_count = 0;
  a->tblk.resize(ns);
  for (int t = 0; t < ns; ++t) {
    const Sweep& sw = h->sweeps[a->tsw[t]];
    a->tblk[t].assign(sw.total, 0);
    for (const Seg& g : sw.segs)
      for (int k = 0; k < g.steps; ++k) a->tblk[t][g.off + k] = g.block;
    steps_total += sw.total;
    slice_count += (size_t)sw.total + 1;
  }
  a->M = 0;
  for (int b = 0; b < a->nb; ++b) a->M += h->blocks[ip][b].steps;
  // explicit sources per (sweep position, slice): quadrature pairs and Q
  struct Src {
    int block;
    double coef;
    int psweep, pidx;
  };
  std::vector<std::vector<std::vector<Src>>> src(ns);
  for (int t = 0; t < ns; ++t) src[t].resize(h->sweeps[a->tsw[t]].total + 1);
  const double densfac = h->chain_dwt[ip] * h->chain_vf[ip] / h->alpha[ip];
  for (int b = 0; b < a->nb; ++b) {
    const BlockMap& bm = h->blocks[ip][b];
    const std::vector<double> c = quad_weights(bm.steps);
    for (int n = 0; n <= bm.steps; ++n) {
      const double coef = densfac * bm.ds * c[n];
      const int hi = bm.off_head + n, ti = bm.off_tail + bm.steps - n;
      src[pos[bm.sweep_head]][hi].push_back({b, coef, bm.sweep_tail, ti});
      src[pos[bm.sweep_tail]][ti].push_back({b, coef, bm.sweep_head, hi});
      AccumEntry ae;
      ae.dst = a->P + (size_t)b * N;
      ae.x = S(bm.sweep_head, hi);
      ae.y = S(bm.sweep_tail, ti);
      ae.coef = coef;
      a->h_acc.push_back(ae);
    }
  }
  for (auto& v : src)
    for (auto& e : v)
      if (e.size() > 2) {
        a->err = "more than two quadrature pairs on one contour slice";
        return PS_INPUT_ERR;
      }
  const BlockMap& b0 = h->blocks[ip][0];
  const int qh_sw = b0.sweep_head, qh_i = b0.off_head;
  const int qt_sw = b0.sweep_tail, qt_i = b0.off_tail + b0.steps;
  auto fill = [&](AdjPoint& p, int t, int i) {
    p.n_src = 0;
    for (const Src& e : src[t][i]) {
      SrcEntry se;
      se.gphi = a->gphi + (size_t)h->blocks[ip][e.block].field * N;
      se.partner = S(e.psweep, e.pidx);
      se.coef = e.coef;
      p.src[p.n_src++] = se;
    }
    const int sw = a->tsw[t];
    p.q_partner = (sw == qh_sw && i == qh_i) ? S(qt_sw, qt_i) : (sw == qt_sw && i == qt_i) ? S(qh_sw, qh_i) : nullptr;
  };
  // junction accumulators: one per sweep whose end feeds a junction
  a->jacc.assign(ns, nullptr);
  const size_t NB = sizeof(double) * (size_t)N;
  PA_CUDA(a, cudaSetDevice(h->dev));
  for (int t = 0; t < ns; ++t)
    for (auto& in : h->sweeps[a->tsw[t]].jin) {
      const int u = pos[in.first];
      if (u < 0 || in.second != h->sweeps[in.first].total) {
        a->err = "junction input is not the end of one of this polymer's sweeps";
        return PS_INPUT_ERR;
      }
      if (!a->jacc[u]) PA_CUDA(a, cudaMalloc((void**)&a->jacc[u], NB));
    }
  for (int sg = 0; sg < 2; ++sg) {
    PA_CUDA(a, cudaMalloc((void**)&a->lam[sg], NB));
    PA_CUDA(a, cudaMalloc((void**)&a->spec[sg], sizeof(double2) * (size_t)h->n[0] * h->n[1] * h->nzh));
  }
  a->storage_bytes = NB * slice_count;
  PA_CUDA(a, cudaMalloc((void**)&a->mu, NB));
  PA_CUDA(a, cudaMalloc((void**)&a->gwb, NB * a->nb));
  PA_CUDA(a, cudaMalloc((void**)&a->gphi, NB * a->nf));
  PA_CUDA(a, cudaMemset(a->gphi, 0, NB * a->nf));
  PA_CUDA(a, cudaMalloc((void**)&a->gq, sizeof(double)));
  a->E_off = (size_t)steps_total * 4 * kAdjRB;
  a->gq_off = a->E_off + (size_t)a->nb * kAdjRB;
  a->part_len = a->gq_off + kAdjRB;
  PA_CUDA(a, cudaMalloc((void**)&a->part, sizeof(double) * a->part_len));
  PA_CUDA(a, cudaMemset(a->part, 0, sizeof(double) * a->part_len));
  PA_CUDA(a, cudaMallocHost((void**)&a->h_part, sizeof(double) * a->part_len));
  // a->P was sized before the accumulation entries pointed at it
  Builder B;
  B.a = a;
  B.h = h;
  B.nx = h->n[0];
  B.ny = h->n[1];
  B.nz = h->n[2];
  B.nzh = h->nzh;
  B.fused = plane_fused_supported(8, h->n[1], h->n[2]);
  const BlockFieldMap fm = field_map(a);

  // ---- forward: the engine's sweeps (every slice stored), Q, quadrature
  a->fwd.push_back([h](cudaStream_t) {
    long long nl = 0;
    return engine_sweeps(h, &nl, 0) == PS_OK ? cudaSuccess : cudaErrorLaunchFailure;
  });
  {
    const double* qx = S(qh_sw, qh_i);
    const double* qy = S(qt_sw, qt_i);
    a->fwd.push_back([=](cudaStream_t st) {
      cudaError_t e = launch_dot_partials<double>(qx, qy, N, h->d_qpart, st);
      if (e == cudaSuccess) e = launch_finalize_q(h->d_qpart, (double)N, 0, h->d_sc, st);
      return e;
    });
    a->fwd.push_back([=](cudaStream_t st) { return cudaMemsetAsync(a->P, 0, sizeof(double) * N * a->nb, st); });
    const int ne = (int)a->h_acc.size();
    a->fwd.push_back([=](cudaStream_t st) {
      adj_accum_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_acc, ne, N);
      return cudaGetLastError();
    });
    a->fwd.push_back([=](cudaStream_t st) {
      adj_normalize_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->P, h->d_phi, fm, N, h->d_sc);
      return cudaGetLastError();
    });
  }
  // ---- backward (bwd[0]: the <g_phi, phi> reduction, as for linear chains)
  {
    const long long nfN = (long long)a->nf * N;
    a->bwd.push_back([=](cudaStream_t st) {
      adj_dot_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->gphi, h->d_phi, nfN, a->part + a->gq_off);
      return cudaGetLastError();
    });
    for (int b = 0; b < a->nb; ++b) {
      const int f = h->blocks[ip][b].field;
      a->bwd.push_back([=](cudaStream_t st) {
        adj_dot_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->gphi + (size_t)f * N, a->P + (size_t)b * N, N,
                                                  a->part + a->E_off + (size_t)b * kAdjRB);
        return cudaGetLastError();
      });
    }
    a->bwd.push_back([=](cudaStream_t st) { return cudaMemsetAsync(a->gwb, 0, sizeof(double) * N * a->nb, st); });
    for (int t = 0; t < ns; ++t)
      if (a->jacc[t]) {
        double* jb = a->jacc[t];
        a->bwd.push_back([=](cudaStream_t st) { return cudaMemsetAsync(jb, 0, NB, st); });
      }
    for (int t = ns - 1; t >= 0; --t) {
      const int sw = a->tsw[t];
      const Sweep& swp = h->sweeps[sw];
      const int T = swp.total;
      const bool junction = !swp.jin.empty();
      int cur = 0;
      {
        AdjPoint p;
        memset(&p, 0, sizeof(p));
        p.lam_out = a->lam[cur];
        fill(p, t, T);
        p.extra = a->jacc[t];
        a->h_pt.push_back(p);
        const size_t pi = a->h_pt.size() - 1;
        a->bwd.push_back([=](cudaStream_t st) {
          adj_init_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_pt + pi, N, h->d_sc, a->gq);
          return cudaGetLastError();
        });
      }
      for (int st_ = T - 1; st_ >= 0; --st_) {
        AdjPoint p;
        memset(&p, 0, sizeof(p));
        const bool out = (st_ >= 1) || junction;
        if (out) fill(p, t, st_);
        adjoint_step_p(B, a->bwd, a->tblk[t][st_], S(sw, st_), S(sw, st_ + 1), a->lam[cur],
                       out ? a->lam[1 - cur] : nullptr, p);
        if (out) cur = 1 - cur;
      }
      if (junction) {
        JunctionAdj jn;
        memset(&jn, 0, sizeof(jn));
        jn.lam0 = a->lam[cur];
        jn.n = (int)swp.jin.size();
        for (int i = 0; i < jn.n; ++i) {
          jn.q_in[i] = S(swp.jin[i].first, swp.jin[i].second);
          jn.lam_out[i] = a->jacc[pos[swp.jin[i].first]];
        }
        a->h_jn.push_back(jn);
        const size_t ji = a->h_jn.size() - 1;
        a->bwd.push_back([=](cudaStream_t st) {
          adj_junction_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_jn + ji, N);
          return cudaGetLastError();
        });
      }
    }
  }
  int r2 = adj_upload(a, &a->d_pw, a->h_pw);
  if (!r2) r2 = adj_upload(a, &a->d_xw, a->h_xw);
  if (!r2) r2 = adj_upload(a, &a->d_acc, a->h_acc);
  if (!r2) r2 = adj_upload(a, &a->d_pt, a->h_pt);
  if (!r2) r2 = adj_upload(a, &a->d_jn, a->h_jn);
  return r2;
}

// polymer: the caller's polymer of cfg to differentiate (its phi contribution
// and ln Q), chain: its quadrature chain (0 unless polyDisperseBCP); single:
// the configuration must be a one-polymer melt (ps_adj_create).
static int adj_build(ps_adj* a, const ps_config* cfg, int polymer, int chain, bool single, int checkpoint) {
  if (cfg->precision != PS_PREC_FP64) {
    a->err = "the adjoint runs in FP64 (precision must be PS_PREC_FP64)";
    return PS_ATTRIB_ERR;
  }
  if (polymer < 0 || polymer >= cfg->n_polymers) {
    a->err = "polymer index out of range";
    return PS_ATTRIB_ERR;
  }
  if (single && (cfg->n_polymers != 1 || cfg->n_solvents != 0)) {
    a->err = "ps_adj_create takes one polymer and no solvent (ps_adj_create_polymer takes a blend)";
    return PS_INPUT_ERR;
  }
  a->h = new ps_handle();
  a->h->no_slices = true;
  a->h->no_alias = true;  // mirror-symmetric chains: both sweeps run and are differentiated
  int rc = engine_create(a->h, cfg);
  if (rc) {
    a->err = a->h->err;
    return rc;
  }
  ps_handle* h = a->h;
  if (chain < 0 || chain >= h->user_ng[polymer]) {
    a->err = "chain index out of range (a polyDisperseBCP polymer has n_g chains, any other one)";
    return PS_ATTRIB_ERR;
  }
  const int ec = h->user_first[polymer] + chain;  // the engine's (expanded) polymer index
  a->ip = ec;
  std::vector<int> own;  // this chain's sweeps
  for (int k = 0; k < (int)h->sweeps.size(); ++k)
    if (h->sweeps[k].polymer == ec) own.push_back(k);
  bool linear = (own.size() == 2);
  for (int k : own) linear = linear && h->sweeps[k].jin.empty();
  if (!linear) {
    // a branched chain: rebuild the engine with slice storage
    engine_free(a->h);
    delete a->h;
    a->h = new ps_handle();
    a->h->no_slices = false;
    rc = engine_create(a->h, cfg);
    if (rc) {
      a->err = a->h->err;
      return rc;
    }
    PA_CUDA(a, cudaMalloc((void**)&a->P, sizeof(double) * (size_t)a->h->N * a->h->blocks[ec].size()));
    return tree_build(a, ec);
  }
  const Sweep& s0 = h->sweeps[own[0]];
  const Sweep& s1 = h->sweeps[own[1]];
  if (s0.storage < 0 || s1.storage < 0 || s0.storage == s1.storage) {
    a->err = "the adjoint needs two executed sweeps";
    return PS_INPUT_ERR;
  }
  a->M = s0.total;
  a->N = h->N;
  a->nf = h->nf;
  a->nb = (int)h->blocks[a->ip].size();
  const int M = a->M;
  for (int sg = 0; sg < 2; ++sg) {
    const Sweep& sw = sg ? s1 : s0;
    a->blk[sg].assign(M, 0);
    for (const Seg& g : sw.segs)
      for (int k = 0; k < g.steps; ++k) a->blk[sg][g.off + k] = g.block;
  }
  // quadrature pairs in sweep-0 indexing: (q_n, q+_{M-n})
  a->quad.assign(M + 1, {});
  const double densfac = h->chain_dwt[ec] * h->chain_vf[ec] / h->alpha[ec];
  for (int b = 0; b < a->nb; ++b) {
    const BlockMap& bm = h->blocks[a->ip][b];
    const std::vector<double> c = quad_weights(bm.steps);
    const bool head0 = (h->sweeps[bm.sweep_head].storage == s0.storage);
    const int o = head0 ? bm.off_head : M - bm.off_head - bm.steps;  // block start in sweep 0
    for (int n = o; n <= o + bm.steps; ++n) {
      const int loc = head0 ? n - o : o + bm.steps - n;
      a->quad[n].push_back({b, densfac * bm.ds * c[loc]});
    }
  }
  for (auto& v : a->quad)
    if (v.size() > 2) {
      a->err = "more than two quadrature pairs on one contour slice";
      return PS_INPUT_ERR;
    }
  {
    const BlockMap& b0 = h->blocks[a->ip][0];
    const bool head0 = (h->sweeps[b0.sweep_head].storage == s0.storage);
    a->n0 = head0 ? b0.off_head : M - b0.off_head;
    if (a->n0 != 0 && a->n0 != M) {
      a->err = "the adjoint needs block 0 to start at a free chain end";
      return PS_INPUT_ERR;
    }
  }
  // checkpoints
  int C = checkpoint;
  if (C <= 0) C = std::max(1, (int)ceil(sqrt((double)M)));
  if (C > M) C = M;
  a->C = C;
  for (int s = 0; s < M; s += C) {
    a->seg_a.push_back(s);
    a->seg_b.push_back(std::min(s + C, M));
  }
  a->J = (int)a->seg_a.size();
  const size_t NB = sizeof(double) * (size_t)a->N;
  const size_t nspec = (size_t)h->n[0] * h->n[1] * h->nzh;
  PA_CUDA(a, cudaSetDevice(h->dev));
  for (int sg = 0; sg < 2; ++sg) {
    PA_CUDA(a, cudaMalloc((void**)&a->ck[sg], NB * a->J));
    PA_CUDA(a, cudaMalloc((void**)&a->endq[sg], NB));
    if (C > 1) PA_CUDA(a, cudaMalloc((void**)&a->seg[sg], NB * (C + 1)));
    PA_CUDA(a, cudaMalloc((void**)&a->lam[sg], NB));
    PA_CUDA(a, cudaMalloc((void**)&a->spec[sg], sizeof(double2) * nspec));
  }
  a->storage_bytes = NB * (2 * (size_t)a->J + 2 + (C > 1 ? 2 * (size_t)(C + 1) : 0));
  PA_CUDA(a, cudaMalloc((void**)&a->mu, NB));
  PA_CUDA(a, cudaMalloc((void**)&a->P, NB * a->nb));
  PA_CUDA(a, cudaMalloc((void**)&a->gwb, NB * a->nb));
  PA_CUDA(a, cudaMalloc((void**)&a->gphi, NB * a->nf));
  PA_CUDA(a, cudaMemset(a->gphi, 0, NB * a->nf));
  PA_CUDA(a, cudaMalloc((void**)&a->gq, sizeof(double)));
  a->E_off = (size_t)2 * M * 4 * kAdjRB;
  a->gq_off = a->E_off + (size_t)a->nb * kAdjRB;
  a->part_len = a->gq_off + kAdjRB;
  PA_CUDA(a, cudaMalloc((void**)&a->part, sizeof(double) * a->part_len));
  PA_CUDA(a, cudaMemset(a->part, 0, sizeof(double) * a->part_len));
  PA_CUDA(a, cudaMallocHost((void**)&a->h_part, sizeof(double) * a->part_len));

  Builder B;
  B.a = a;
  B.h = h;
  B.nx = h->n[0];
  B.ny = h->n[1];
  B.nz = h->n[2];
  B.nzh = h->nzh;
  B.fused = plane_fused_supported(8, h->n[1], h->n[2]);
  const BlockFieldMap fm = field_map(a);
  const long long N = a->N;

  // ---- forward: both sweeps in lockstep, checkpoints and end slices stored
  {
    const int sig[2] = {0, 1};
    const int st0[2] = {0, 0};
    const double* src[2] = {nullptr, nullptr};
    B.sweeps(a->fwd, 2, sig, st0, src, M, [a, M](int i, int k) -> double* {
      if (k == M) return a->endq[i];
      for (int j = 0; j < a->J; ++j) {
        const int pos = (i == 0) ? a->seg_a[j] : M - a->seg_b[j];
        if (pos == k) return a->ck[i] + (size_t)j * a->N;
      }
      return nullptr;
    });
    // Q = <q_n0 q+_{M-n0}>
    const double* qx = (a->n0 == 0) ? a->ck[0] : a->endq[0];
    const double* qy = (a->n0 == 0) ? a->endq[1] : a->ck[1] + (size_t)(a->J - 1) * N;
    a->fwd.push_back([=](cudaStream_t st) {
      cudaError_t e = launch_dot_partials<double>(qx, qy, N, h->d_qpart, st);
      if (e == cudaSuccess) e = launch_finalize_q(h->d_qpart, (double)N, 0, h->d_sc, st);
      return e;
    });
    // quadrature, segment by segment
    a->fwd.push_back([=](cudaStream_t st) { return cudaMemsetAsync(a->P, 0, sizeof(double) * N * a->nb, st); });
    for (int j = 0; j < a->J; ++j) {
      recompute(B, a->fwd, j);
      const size_t e0 = a->h_acc.size();
      const int nend = (j == a->J - 1) ? a->seg_b[j] : a->seg_b[j] - 1;
      for (int n = a->seg_a[j]; n <= nend; ++n)
        for (auto& e : a->quad[n]) {
          AccumEntry ae;
          ae.dst = a->P + (size_t)e.first * N;
          ae.x = slice_ptr(a, 0, n, j);
          ae.y = slice_ptr(a, 1, M - n, j);
          ae.coef = e.second;
          a->h_acc.push_back(ae);
        }
      const int ne = (int)(a->h_acc.size() - e0);
      a->fwd.push_back([=](cudaStream_t st) {
        adj_accum_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->d_acc + e0, ne, N);
        return cudaGetLastError();
      });
    }
    a->fwd.push_back([=](cudaStream_t st) {
      adj_normalize_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->P, h->d_phi, fm, N, h->d_sc);
      return cudaGetLastError();
    });
  }
  // ---- backward.  bwd[0] is the <g_phi, phi> reduction; ps_adj_backward
  // launches the dL/dQ kernel right after it, before any source is read.
  {
    const long long nfN = (long long)a->nf * N;
    a->bwd.push_back([=](cudaStream_t st) {
      adj_dot_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->gphi, h->d_phi, nfN, a->part + a->gq_off);
      return cudaGetLastError();
    });
    for (int b = 0; b < a->nb; ++b) {
      const int f = h->blocks[a->ip][b].field;
      a->bwd.push_back([=](cudaStream_t st) {
        adj_dot_kernel<<<kAdjRB, kAdjRT, 0, st>>>(a->gphi + (size_t)f * N, a->P + (size_t)b * N, N,
                                                  a->part + a->E_off + (size_t)b * kAdjRB);
        return cudaGetLastError();
      });
    }
    a->bwd.push_back([=](cudaStream_t st) { return cudaMemsetAsync(a->gwb, 0, sizeof(double) * N * a->nb, st); });
    // sweep 0: lambda from n = M down, segments last to first
    int cur = 0;
    for (int j = a->J - 1; j >= 0; --j) {
      recompute(B, a->bwd, j);
      if (j == a->J - 1) adjoint_init(a, a->bwd, 0, j, cur);
      for (int s = a->seg_b[j] - 1; s >= a->seg_a[j]; --s) {
        adjoint_step(B, a->bwd, 0, s, j, cur);
        cur = 1 - cur;
      }
    }
    // sweep 1: lambda+ from m = M down, i.e. segments first to last
    cur = 0;
    for (int j = 0; j < a->J; ++j) {
      recompute(B, a->bwd, j);
      if (j == 0) adjoint_init(a, a->bwd, 1, j, cur);
      for (int m = M - a->seg_a[j] - 1; m >= M - a->seg_b[j]; --m) {
        adjoint_step(B, a->bwd, 1, m, j, cur);
        cur = 1 - cur;
      }
    }
  }
  int r2 = adj_upload(a, &a->d_pw, a->h_pw);
  if (!r2) r2 = adj_upload(a, &a->d_xw, a->h_xw);
  if (!r2) r2 = adj_upload(a, &a->d_acc, a->h_acc);
  if (!r2) r2 = adj_upload(a, &a->d_pt, a->h_pt);
  return r2;
}

static void adj_free(ps_adj* a) {
  if (a->h) {
    cudaSetDevice(a->h->dev);
    if (a->h->st) cudaStreamSynchronize(a->h->st);
  }
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (int sg = 0; sg < 2; ++sg) {
    f(a->ck[sg]);
    f(a->endq[sg]);
    f(a->seg[sg]);
    f(a->lam[sg]);
    f(a->spec[sg]);
  }
  f(a->mu);
  f(a->P);
  f(a->gwb);
  f(a->gphi);
  f(a->gq);
  f(a->part);
  if (a->h_part) cudaFreeHost(a->h_part);
  f(a->d_pw);
  f(a->d_xw);
  f(a->d_acc);
  f(a->d_pt);
  f(a->d_jn);
  for (auto p : a->jacc) f(p);
  if (a->h) {
    engine_free(a->h);
    delete a->h;
  }
}

static int run_ops(ps_adj* a, const std::vector<Op>& ops, size_t from) {
  for (size_t i = from; i < ops.size(); ++i) PA_CUDA(a, ops[i](a->h->st));
  return PS_OK;
}

}  // namespace psb

using namespace psb;

extern "C" {

static int adj_create(const ps_config* cfg, int polymer, int chain, bool single, int checkpoint_interval,
                      ps_adj** out) {
  if (!cfg || !out) {
    g_adj_err = "null argument";
    return PS_ATTRIB_ERR;
  }
  *out = nullptr;
  ps_adj* a = new ps_adj();
  int rc = adj_build(a, cfg, polymer, chain, single, checkpoint_interval);
  if (rc) {
    g_adj_err = a->err;
    adj_free(a);
    delete a;
    cudaGetLastError();  // clear a failed allocation's last-error state
    return rc;
  }
  *out = a;
  return PS_OK;
}

int ps_adj_create(const ps_config* cfg, int checkpoint_interval, ps_adj** out) {
  return adj_create(cfg, 0, 0, true, checkpoint_interval, out);
}

int ps_adj_create_polymer(const ps_config* cfg, int polymer, int chain, int checkpoint_interval,
                          ps_adj** out) {
  return adj_create(cfg, polymer, chain, false, checkpoint_interval, out);
}

int ps_adj_set_potential(ps_adj* a, const double* psi) {
  if (!a || !a->h || !psi) return PS_ATTRIB_ERR;
  ps_handle* h = a->h;
  if (h->nq == 0) {
    a->err = "the configuration has no chargeDens field";
    return PS_ATTRIB_ERR;
  }
  PA_CUDA(a, cudaSetDevice(h->dev));
  PA_CUDA(a, cudaMemcpyAsync(h->d_psi, psi, sizeof(double) * (size_t)h->nq * a->N, cudaMemcpyDeviceToDevice,
                             h->st));
  a->have_forward = false;
  return PS_OK;
}

int ps_adj_potential_grad(ps_adj* a, double* g_psi) {
  if (!a || !a->h || !g_psi) return PS_ATTRIB_ERR;
  ps_handle* h = a->h;
  if (h->nq == 0) {
    a->err = "the configuration has no chargeDens field";
    return PS_ATTRIB_ERR;
  }
  if (!a->have_backward) {
    a->err = "ps_adj_potential_grad needs a ps_adj_backward first";
    return PS_ATTRIB_ERR;
  }
  const long long N = a->N;
  PA_CUDA(a, cudaSetDevice(h->dev));
  PA_CUDA(a, cudaMemsetAsync(g_psi, 0, sizeof(double) * (size_t)h->nq * N, h->st));
  // psi enters a charged block's exponent as facz psi next to w: dL/dpsi = facz dL/dw of the block
  for (int b = 0; b < a->nb; ++b) {
    const BlockMap& bm = h->blocks[a->ip][b];
    if (bm.charge_field < 0) continue;
    adj_axpy_kernel<<<kAdjRB, kAdjRT, 0, h->st>>>(g_psi + (size_t)bm.charge_field * N, a->gwb + (size_t)b * N,
                                                  bm.facz, N);
    PA_CUDA(a, cudaGetLastError());
  }
  PA_CUDA(a, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int ps_adj_species(const ps_adj* a, double* f_weight, double* length_ratio, double* dens_avg) {
  if (!a || !a->h) return PS_ATTRIB_ERR;
  const ps_handle* h = a->h;
  if (f_weight) *f_weight = h->chain_dwt[a->ip] * h->chain_vf[a->ip];
  if (length_ratio) *length_ratio = h->alpha[a->ip];
  if (dens_avg)
    for (int i = 0; i < h->nf; ++i) dens_avg[i] = h->fm.dens_avg[i];
  return PS_OK;
}

int ps_adj_destroy(ps_adj* a) {
  if (!a) return PS_OK;
  adj_free(a);
  delete a;
  return PS_OK;
}

const char* ps_adj_last_error(const ps_adj* a) { return a ? a->err.c_str() : g_adj_err.c_str(); }

int ps_adj_info(const ps_adj* a, int* contour_steps, int* checkpoint_interval, size_t* slice_bytes) {
  if (!a) return PS_ATTRIB_ERR;
  if (contour_steps) *contour_steps = a->M;
  if (checkpoint_interval) *checkpoint_interval = a->C;
  if (slice_bytes) *slice_bytes = a->storage_bytes;
  return PS_OK;
}

int ps_adj_forward(ps_adj* a, const double* w, double* phi, double* log_q) {
  if (!a || !w) return PS_ATTRIB_ERR;
  ps_handle* h = a->h;
  const size_t nfN = (size_t)a->nf * a->N;
  PA_CUDA(a, cudaSetDevice(h->dev));
  PA_CUDA(a, cudaMemcpyAsync(h->d_w, w, sizeof(double) * nfN, cudaMemcpyDeviceToDevice, h->st));
  PA_CUDA(a, cudaMemsetAsync(&h->d_sc->error_flags, 0, sizeof(int), h->st));
  long long nl = 0;
  int rc = engine_pre(h, &nl);
  if (rc) {
    a->err = h->err;
    return rc;
  }
  rc = run_ops(a, a->fwd, 0);
  if (rc) return rc;
  if (phi) PA_CUDA(a, cudaMemcpyAsync(phi, h->d_phi, sizeof(double) * nfN, cudaMemcpyDeviceToDevice, h->st));
  rc = engine_check_scalars(h);
  if (rc) {
    a->err = h->err;
    return rc;
  }
  if (log_q) *log_q = h->h_sc->log_q[0];
  a->have_forward = true;
  a->have_backward = false;
  return PS_OK;
}

int ps_adj_backward(ps_adj* a, const double* g_phi, double g_log_q, double* g_w, double* g_box,
                    double* g_ds) {
  if (!a || !g_phi || !g_w) return PS_ATTRIB_ERR;
  if (!a->have_forward) {
    a->err = "ps_adj_backward needs a ps_adj_forward first";
    return PS_ATTRIB_ERR;
  }
  ps_handle* h = a->h;
  const long long N = a->N;
  PA_CUDA(a, cudaSetDevice(h->dev));
  PA_CUDA(a, cudaMemcpyAsync(a->gphi, g_phi, sizeof(double) * (size_t)a->nf * N, cudaMemcpyDeviceToDevice,
                             h->st));
  PA_CUDA(a, a->bwd[0](h->st));
  adj_gq_kernel<<<1, kAdjRT, 0, h->st>>>(a->part + a->gq_off, g_log_q, h->d_sc, a->gq);
  PA_CUDA(a, cudaGetLastError());
  int rc = run_ops(a, a->bwd, 1);
  if (rc) return rc;
  adj_sum_blocks_kernel<<<kAdjRB, kAdjRT, 0, h->st>>>(a->gwb, field_map(a), N, g_w);
  PA_CUDA(a, cudaGetLastError());
  PA_CUDA(a, cudaMemcpyAsync(a->h_part, a->part, sizeof(double) * a->part_len, cudaMemcpyDeviceToHost, h->st));
  PA_CUDA(a, cudaStreamSynchronize(h->st));
  // host sums in a fixed order
  double gbox[3] = {0.0, 0.0, 0.0};
  std::vector<double> gds(a->nb, 0.0);
  const double L[3] = {h->n[0] * h->cfg.cell[0], h->n[1] * h->cfg.cell[1], h->n[2] * h->cfg.cell[2]};
  for (size_t slot = 0; slot < a->slot_block.size(); ++slot) {
    const int b = a->slot_block[slot];
    const BlockMap& bm = h->blocks[a->ip][b];
    const double* p = a->h_part + slot * 4 * kAdjRB;
    double R[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < kAdjRB; ++i) R[q] += p[q * kAdjRB + i];
    const double b2 = bm.bseg * bm.bseg;
    for (int d = 0; d < 3; ++d) gbox[d] += 2.0 * bm.ds * b2 / L[d] * R[d];
    gds[b] += -b2 * (R[0] + R[1] + R[2]) + R[3];
  }
  for (int b = 0; b < a->nb; ++b) {
    double E = 0.0;
    for (int i = 0; i < kAdjRB; ++i) E += a->h_part[a->E_off + (size_t)b * kAdjRB + i];
    gds[b] += E / h->blocks[a->ip][b].ds;
  }
  if (g_box)
    for (int d = 0; d < 3; ++d) g_box[d] = gbox[d];
  if (g_ds)
    for (int b = 0; b < a->nb; ++b) g_ds[b] = gds[b];
  a->have_backward = true;
  return PS_OK;
}

void* ps_adj_stream(const ps_adj* a) { return (a && a->h) ? (void*)a->h->st : nullptr; }

}  // extern "C"
