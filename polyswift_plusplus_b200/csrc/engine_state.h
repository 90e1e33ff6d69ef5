// State of one SCFT instance on the device (ps_handle) and the engine
// functions that the batch driver (batch.cu) composes into its own graph.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "../../include/pswift.h"
#include "field_kernels.cuh"
#include "kernels.h"
#include "mt19937.h"
#include "sweeps.cuh"

namespace psb {

enum { HEAD = 0, TAIL = 1 };

struct Seg {
  int block;
  int from;   // HEAD: this sweep produces the block's qs; TAIL: its qts
  int off;    // slice offset of the segment inside the sweep
  int steps;
  int wfac_id;
  int ktab_id;
};

struct Sweep {
  int polymer;
  std::vector<Seg> segs;
  int total = 0;
  int storage = -1;  // index of the executed sweep holding its slices
  // Branched polymers: a sweep that starts at a junction of three or more block
  // ends starts from the product of the final slices (sweep, slice) of the
  // sweeps arriving there, written into junction buffer jbuf before it runs.
  std::vector<std::pair<int, int>> jin;
  int jbuf = -1;
};

// Boltzmann-factor table key: one wfac array per distinct (field, ds, charge)
// (charge_field -1: flexPseudoSpec; else chargeFlexPseudoSpec with facz = za alpha L).
struct WfacKey {
  int field;
  double ds;
  int charge_field;
  double facz;
  bool operator==(const WfacKey& o) const {
    return field == o.field && ds == o.ds && charge_field == o.charge_field && facz == o.facz;
  }
};

struct BlockMap {
  int steps;
  int field;
  double ds, bseg;
  int charge_field;  // -1: not charged
  double za, qalpha, facz;
  int sweep_head, off_head;  // qs[n]  = slices(sweep_head)[off_head + n]
  int sweep_tail, off_tail;  // qts[n] = slices(sweep_tail)[off_tail + n]
};

template <typename T> struct Buffers {
  std::vector<T*> slices;        // per executed sweep: (total+1)*N
  std::vector<c2_t<T>*> spec;    // per executed sweep
  std::vector<T*> wfac;          // per (field, ds) key
  std::vector<T*> jbuf;          // junction start buffers of branched polymers (N each)
  std::vector<double*> dcbuf;    // per executed sweep, FP32 sweeps: mean-mode carry (partials
                                 // [0, dc_cap), the mean at dc_cap, the count at dc_cap + 1, the
                                 // fed-back rounding at dc_cap + 2)
  int dc_cap = 0;
  std::vector<T*> kx, kyz;       // per (ds, bseg) key
  c2_t<T>* tw_x = nullptr;
  c2_t<T>* tw_y = nullptr;
  c2_t<T>* tw_z = nullptr;
  c2_t<T>* tw_zh = nullptr;
  PlaneWork<T>* d_plane = nullptr;
  PencilWork<T>* d_pencil = nullptr;
  std::vector<PlaneWork<T>> h_plane;    // host copies of the work tables
  std::vector<PencilWork<T>> h_pencil;
  std::vector<JunctionLaunch<T>> junc;  // junction starts, by global step (junc_off/junc_cnt)
};

}  // namespace psb

struct ps_handle {
  ps_config cfg;   // with every polyDisperseBCP expanded into its quadrature chains
  ps_config ucfg;  // as the caller gave it
  // polymer ("chain") index of cfg -> the caller's polymer, its quadrature index,
  // density weight (1, or w_k / Gamma(alpha)) and the caller's volfrac
  std::vector<int> chain_user, chain_k;
  std::vector<double> chain_dwt, chain_vf;
  // caller's polymer -> first chain and number of chains (1 unless polydisperse)
  std::vector<int> user_first, user_ng;
  int n[3];
  long long N = 0;
  int nzh = 0;
  int nf = 0;
  int prec = PS_PREC_FP64;
  int dev = 0;
  bool fused_plane = true;
  cudaStream_t st = nullptr;
  std::string err;

  double* d_w = nullptr;    // nf*N
  double* d_phi = nullptr;  // nf*N
  double* d_p = nullptr;
  double* d_noise = nullptr;  // nf*N scaled Gaussians of the current iteration
  void* noise_gen = nullptr;   // device generator of d_noise (noise.cu), or nullptr
  int nq = 0;                 // chargeDens PhysFields
  double* d_rho = nullptr;    // nq*N charge densities
  double* d_psi = nullptr;    // nq*N electric potentials

  std::vector<std::vector<psb::BlockMap>> blocks;
  std::vector<double> alpha;  // length ratios
  std::vector<psb::Sweep> sweeps;
  std::vector<int> exec;  // sweep indices that are executed (own storage)
  std::vector<psb::WfacKey> wfac_keys;
  std::vector<std::pair<double, double>> ktab_keys;
  int kmax = 0;
  std::vector<int> plane_off, plane_cnt, pencil_off, pencil_cnt;
  // Lockstep schedule: executed sweep e runs its local step k - sw_start[e] at
  // global step k; a sweep leaving a junction starts one step after the last
  // arriving sweep's final step, and its junction kernel runs in between.
  std::vector<int> sw_start;
  std::vector<int> junc_off, junc_cnt;  // per global step, into Buffers<T>::junc
  // the same tables restricted to one executed sweep (VARIANT_SPLIT), and the
  // streams and events of its launch chain
  std::vector<std::vector<int>> sw_plane_off, sw_plane_cnt, sw_pencil_off, sw_pencil_cnt;
  std::vector<cudaStream_t> sw_st;
  std::vector<cudaEvent_t> sw_ev;
  cudaEvent_t ev_split = nullptr;

  psb::Buffers<float> bf;
  psb::Buffers<double> bd;

  double* d_qpart = nullptr;
  double* d_upart = nullptr;
  psb::DevScalars* d_sc = nullptr;
  psb::DevScalars* h_sc = nullptr;  // pinned
  psb::FieldModel fm;

  // Anderson history
  int am_slots = 0;
  double* d_hw = nullptr;
  double* d_hd = nullptr;
  double* d_gram = nullptr;
  double* d_gpart = nullptr;

  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int eager_iters = 0;
  long long launches_per_iter = 0;
  int variant = -1;  // kernel variant (VARIANT_* bits); -1: autotune before the graph is built
  float tune_ms[psb::VARIANT_COUNT] = {};
  bool xy_ok = false;  // the row + x-y plane design exists for this grid
  bool cluster_ok = false;  // the two-CTA cluster plane pass exists for this grid and precision
  bool in_batch = false;  // owned by a ps_batch, whose merged work tables point into it
  bool branched = false;  // a branched polymer: its sweeps run as dependent launch chains only
  int n_jbuf = 0;
  bool no_slices = false; // tables only, no slice storage (the adjoint keeps its own)
  bool no_alias = false;  // mirror-symmetric chains keep both sweeps (the adjoint differentiates each)
  void* filter = nullptr;  // spectral filter updater (filter.cu), or nullptr
  void* poisson = nullptr; // Poisson updater (poisson.cu), or nullptr
  std::vector<int> post_order;  // updaters after the field update, in run order (POST_*)

  psb::Mt19937 rng;
  long long pending_gauss = 0;  // Gaussian draws owed to the stream (noise = 0)
  long long iterations = 0;

  // Sweep timing: CUDA events around the propagator sweeps of each iteration.
  int timing_cap = 0;
  int timing_count = 0;
  cudaEvent_t ev_cap_start = nullptr, ev_cap_end = nullptr;  // recorded during capture
  std::vector<cudaEvent_t> ev_start, ev_end;                 // one pair per sample
  cudaGraphNode_t node_start = nullptr, node_end = nullptr;  // event-record nodes in the graph
  bool graph_has_timing = false;
  std::vector<float> eager_ms;  // samples taken on eager iterations

  // Asynchronous field read-back (ps_gpu_get_fields_async): per (which, index) a
  // device snapshot taken on st and copied to the host on io_st.
  struct ReadSlot {
    double* d = nullptr;
    cudaEvent_t snap = nullptr;  // snapshot complete (st)
    cudaEvent_t done = nullptr;  // host copy complete (io_st)
  };
  std::map<std::pair<int, int>, ReadSlot> read_slots;
  cudaStream_t io_st = nullptr;
  // Asynchronous upload (ps_gpu_set_fields_async): the pressure field goes up
  // on up_st after the work enqueued on st so far (up_ev), and every field
  // update waits for p_ready (recorded at creation, then after each upload; an
  // event-wait node of the captured graph).
  cudaStream_t up_st = nullptr;
  cudaEvent_t up_ev = nullptr;
  cudaEvent_t p_ready = nullptr;
  double sweep_bytes = 0.0;  // algorithmic bytes of the sweeps of one iteration
  long long sweep_steps = 0; // propagator steps (all sweeps) of one iteration
};

namespace psb {

#define PS_CUDA(h, call)                                                               \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return PS_GPU_ERR;                                                               \
    }                                                                                  \
  } while (0)

// Pieces of one iteration, all on h->st (engine.cu):
//   engine_pre:  reset phi, Boltzmann factors of every (field, ds);
//   the sweeps:  handle_sweep_set(h) under launch_sweep_set;
//   engine_post: Q, contour quadrature into phi, field update, pressure shift.
// Build an instance from a configuration (ps_gpu_create without the wrapper);
// with h->no_slices set beforehand no propagator slice storage is allocated.
int engine_create(ps_handle* h, const ps_config* cfg);
void engine_free(ps_handle* h);
// Spectral filter updater (filter.cu): applied after iteration `step` (0-based)
// when its schedule says so; freed with the handle.
int filter_after_iteration(ps_handle* h, long long step);
void filter_free(ps_handle* h);
// polyDisperseBCP (polydisperse.cu): `out` = `in` with each polydisperse polymer
// replaced by its n_g quadrature chains; fills the chain tables of h.
int expand_polydisperse(ps_handle* h, const ps_config& in, ps_config* out);
// Poisson updater (poisson.cu), the same way.
int poisson_after_iteration(ps_handle* h, long long step);
void poisson_free(ps_handle* h);
// Updaters that run after the field update, in h->post_order.
enum { POST_FILTER = 1, POST_POISSON = 2 };
void post_order_set(ps_handle* h, int code, bool on);
int engine_pre(ps_handle* h, long long* nlaunch);
int engine_post(ps_handle* h, long long* nlaunch);
// The instance's propagator sweeps alone, on h->st (variant bit 3: as concurrent
// launch chains forked from and joined back into h->st).
int engine_sweeps(ps_handle* h, long long* nlaunch, int variant);
// Host-side random-number bookkeeping owed before each iteration.
int engine_prepare_noise(ps_handle* h);
// Updater noise drawn on the device (noise.cu).  noise_launch forks the draws of
// one iteration off h->st and noise_join joins them back (both legal in stream
// capture); noise_upload / noise_download move the MT19937 state between the
// host generator and the device.
int noise_setup(ps_handle* h);
void noise_free(ps_handle* h);
int noise_upload(ps_handle* h);
int noise_download(ps_handle* h);
int noise_launch(ps_handle* h, long long* nlaunch);
int noise_join(ps_handle* h);
int noise_check(ps_handle* h);
// Copy the device scalars back and turn error flags into status codes.
int engine_check_scalars(ps_handle* h);

template <typename T> Buffers<T>& bufs(ps_handle* h);
template <> inline Buffers<float>& bufs<float>(ps_handle* h) { return h->bf; }
template <> inline Buffers<double>& bufs<double>(ps_handle* h) { return h->bd; }

template <typename T> SweepSet<T> handle_sweep_set(ps_handle* h) {
  Buffers<T>& B = bufs<T>(h);
  SweepSet<T> s;
  for (int d = 0; d < 3; ++d) s.n[d] = h->n[d];
  s.nzh = h->nzh;
  s.fused_plane = h->fused_plane;
  s.xy_ok = h->xy_ok;
  s.kmax = h->kmax;
  s.tw_x = B.tw_x;
  s.tw_y = B.tw_y;
  s.tw_z = B.tw_z;
  s.tw_zh = B.tw_zh;
  s.d_plane = B.d_plane;
  s.d_pencil = B.d_pencil;
  s.plane_off = h->plane_off.data();
  s.plane_cnt = h->plane_cnt.data();
  s.pencil_off = h->pencil_off.data();
  s.pencil_cnt = h->pencil_cnt.data();
  if (!B.junc.empty()) {
    s.junc = B.junc.data();
    s.junc_off = h->junc_off.data();
    s.junc_cnt = h->junc_cnt.data();
  }
  return s;
}

}  // namespace psb
