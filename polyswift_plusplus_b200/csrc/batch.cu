// Batched SCFT: many independent instances, one captured CUDA graph.
//
// Instances are grouped into size classes (same grid and precision).  Every
// class runs its propagator sweeps as one merged sweep set: at global contour
// step k a single plane/row launch and a single spectral launch cover the
// works of every member that has a step k, so small grids fill the GPU
// together instead of one after another.  The per-instance field work (phi
// reset, Boltzmann factors, Q, contour quadrature, the steepest-descent or
// Anderson update, the pressure shift) runs on each instance's own stream, as
// parallel branches of the same graph:
//
//   fork -> [pre(i) on stream i] -> [class sweeps on class stream c] ->
//   [post(i) on stream i] -> join
//
// The per-instance semantics are exactly those of ps_gpu_iterate on the
// instance alone (PsDomain::update, pstrol/PsDomain.cpp:332-372); a merged
// launch does the same arithmetic per work as a single-instance launch of the
// same kernel variant.
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "engine_state.h"

namespace psb {

struct BatchClass {
  int n[3] = {0, 0, 0};
  int prec = PS_PREC_FP64;
  std::vector<int> members;
  int kmax = -1;
  std::vector<int> plane_off, plane_cnt, pencil_off, pencil_cnt;
  // members' junction starts (branched polymers), by global step
  std::vector<JunctionLaunch<float>> junc_f;
  std::vector<JunctionLaunch<double>> junc_d;
  std::vector<int> junc_off, junc_cnt;
  void* d_plane = nullptr;   // PlaneWork<T>[]
  void* d_pencil = nullptr;  // PencilWork<T>[]
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  int variant = -1;
  float tune_ms[VARIANT_COUNT] = {};
  // Chains mode: each member runs its sweeps as its own concurrent launch chains
  // (the single-instance split variants) instead of all members' sweeps merged
  // into one launch per step; chosen by timing, or by a forced variant with bit 3.
  bool chains = false;
  float chains_ms = -1.f;
};

static thread_local std::string g_batch_err;

}  // namespace psb

struct ps_batch {
  std::vector<ps_handle*> inst;
  std::vector<int> class_of;
  std::vector<psb::BatchClass> classes;
  int dev = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_inst;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int eager_iters = 0;
  int forced_variant = -1;
  long long launches_per_iter = 0;
  std::string err;
};

namespace psb {

#define PB_CUDA(b, call)                                                 \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      (b)->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
      return PS_GPU_ERR;                                                 \
    }                                                                    \
  } while (0)

template <typename T> static std::vector<JunctionLaunch<T>>& class_junc(BatchClass& c);
template <> std::vector<JunctionLaunch<float>>& class_junc<float>(BatchClass& c) { return c.junc_f; }
template <> std::vector<JunctionLaunch<double>>& class_junc<double>(BatchClass& c) { return c.junc_d; }

template <typename T>
static SweepSet<T> class_sweep_set(ps_batch* b, BatchClass& c) {
  ps_handle* h0 = b->inst[c.members[0]];
  SweepSet<T> s = handle_sweep_set<T>(h0);  // grid, design flags, twiddles
  s.kmax = c.kmax;
  s.d_plane = static_cast<const PlaneWork<T>*>(c.d_plane);
  s.d_pencil = static_cast<const PencilWork<T>*>(c.d_pencil);
  s.plane_off = c.plane_off.data();
  s.plane_cnt = c.plane_cnt.data();
  s.pencil_off = c.pencil_off.data();
  s.pencil_cnt = c.pencil_cnt.data();
  std::vector<JunctionLaunch<T>>& jv = class_junc<T>(c);
  s.junc = jv.empty() ? nullptr : jv.data();
  s.junc_off = c.junc_off.data();
  s.junc_cnt = c.junc_cnt.data();
  return s;
}

// Concatenate the members' per-step work tables.
template <typename T>
static int build_class_tables(ps_batch* b, BatchClass& c) {
  c.kmax = 0;
  for (int i : c.members) c.kmax = std::max(c.kmax, b->inst[i]->kmax);
  std::vector<PlaneWork<T>> pw;
  std::vector<PencilWork<T>> xw;
  c.plane_off.assign(c.kmax + 1, 0);
  c.plane_cnt.assign(c.kmax + 1, 0);
  c.pencil_off.assign(c.kmax + 1, 0);
  c.pencil_cnt.assign(c.kmax + 1, 0);
  std::vector<JunctionLaunch<T>>& jv = class_junc<T>(c);
  jv.clear();
  c.junc_off.assign(c.kmax + 1, 0);
  c.junc_cnt.assign(c.kmax + 1, 0);
  for (int k = 0; k <= c.kmax; ++k) {
    c.plane_off[k] = (int)pw.size();
    c.pencil_off[k] = (int)xw.size();
    c.junc_off[k] = (int)jv.size();
    for (int i : c.members) {
      ps_handle* h = b->inst[i];
      if (k > h->kmax) continue;
      const Buffers<T>& B = bufs<T>(h);
      for (int j = 0; j < h->junc_cnt[k]; ++j) jv.push_back(B.junc[h->junc_off[k] + j]);
    }
    c.junc_cnt[k] = (int)jv.size() - c.junc_off[k];
    for (int i : c.members) {
      ps_handle* h = b->inst[i];
      if (k > h->kmax) continue;
      const Buffers<T>& B = bufs<T>(h);
      for (int j = 0; j < h->plane_cnt[k]; ++j) pw.push_back(B.h_plane[h->plane_off[k] + j]);
      for (int j = 0; j < h->pencil_cnt[k]; ++j) xw.push_back(B.h_pencil[h->pencil_off[k] + j]);
    }
    c.plane_cnt[k] = (int)pw.size() - c.plane_off[k];
    c.pencil_cnt[k] = (int)xw.size() - c.pencil_off[k];
  }
  PB_CUDA(b, cudaMalloc(&c.d_plane, sizeof(PlaneWork<T>) * std::max<size_t>(pw.size(), 1)));
  PB_CUDA(b, cudaMemcpy(c.d_plane, pw.data(), sizeof(PlaneWork<T>) * pw.size(), cudaMemcpyHostToDevice));
  PB_CUDA(b, cudaMalloc(&c.d_pencil, sizeof(PencilWork<T>) * std::max<size_t>(xw.size(), 1)));
  PB_CUDA(b, cudaMemcpy(c.d_pencil, xw.data(), sizeof(PencilWork<T>) * xw.size(), cudaMemcpyHostToDevice));
  return PS_OK;
}

static int class_variant(ps_batch* b, const BatchClass& c) {
  int v = (b->forced_variant >= 0) ? b->forced_variant : (c.variant < 0 ? 0 : c.variant);
  if ((v & VARIANT_XY) && !b->inst[c.members[0]]->xy_ok) v &= ~VARIANT_XY;
  return v & ~VARIANT_SPLIT;  // the kernels; bit 3 is the class's chains mode
}

static bool class_chains(const ps_batch* b, const BatchClass& c) {
  return (b->forced_variant >= 0) ? ((b->forced_variant & VARIANT_SPLIT) != 0) : c.chains;
}

// Chains mode: every member's sweeps on its own stream (after its pre work).
static int launch_class_chains(ps_batch* b, BatchClass& c, long long* nl) {
  const int v = class_variant(b, c) | VARIANT_SPLIT;
  for (int i : c.members) {
    int rc = engine_sweeps(b->inst[i], nl, v);
    if (rc) {
      b->err = "instance " + std::to_string(i) + ": " + b->inst[i]->err;
      return rc;
    }
  }
  return PS_OK;
}

static int launch_class(ps_batch* b, BatchClass& c, long long* nl) {
  const int v = class_variant(b, c);
  cudaError_t e = (c.prec == PS_PREC_MIXED)
                      ? launch_sweep_set<float>(class_sweep_set<float>(b, c), v, c.st, nl)
                      : launch_sweep_set<double>(class_sweep_set<double>(b, c), v, c.st, nl);
  PB_CUDA(b, e);
  return PS_OK;
}

static int instance_error(ps_batch* b, int i, int rc) {
  b->err = "instance " + std::to_string(i) + ": " + b->inst[i]->err;
  return rc;
}

// One batch iteration on b->st and its forked streams (eager or under capture).
static int launch_batch_iteration(ps_batch* b, long long* nl) {
  PB_CUDA(b, cudaEventRecord(b->ev_fork, b->st));
  for (size_t i = 0; i < b->inst.size(); ++i) {
    ps_handle* h = b->inst[i];
    PB_CUDA(b, cudaStreamWaitEvent(h->st, b->ev_fork, 0));
    int rc = noise_launch(h, nl);  // the instance's updater noise, if any
    if (rc) return instance_error(b, (int)i, rc);
    rc = engine_pre(h, nl);
    if (rc) return instance_error(b, (int)i, rc);
    PB_CUDA(b, cudaEventRecord(b->ev_inst[i], h->st));
  }
  for (BatchClass& c : b->classes) {
    if (class_chains(b, c)) {
      int rc = launch_class_chains(b, c, nl);  // on the members' own streams
      if (rc) return rc;
      continue;
    }
    for (int i : c.members) PB_CUDA(b, cudaStreamWaitEvent(c.st, b->ev_inst[i], 0));
    int rc = launch_class(b, c, nl);
    if (rc) return rc;
    PB_CUDA(b, cudaEventRecord(c.ev, c.st));
    PB_CUDA(b, cudaStreamWaitEvent(b->st, c.ev, 0));
  }
  for (size_t i = 0; i < b->inst.size(); ++i) {
    ps_handle* h = b->inst[i];
    if (!class_chains(b, b->classes[b->class_of[i]]))
      PB_CUDA(b, cudaStreamWaitEvent(h->st, b->classes[b->class_of[i]].ev, 0));
    int rc = engine_post(h, nl);
    if (rc) return instance_error(b, (int)i, rc);
    PB_CUDA(b, cudaEventRecord(b->ev_inst[i], h->st));
    PB_CUDA(b, cudaStreamWaitEvent(b->st, b->ev_inst[i], 0));
  }
  return PS_OK;
}

// Updaters that run after the field update (spectral filters, Poisson), per
// instance in its updaterSequence order, on the instance's stream between this
// batch iteration and the next (they sit outside the captured graph because
// their schedule depends on the step, as for a single handle).
static int run_post_updaters(ps_batch* b) {
  bool any = false;
  for (ps_handle* h : b->inst) any |= !h->post_order.empty();
  if (!any) return PS_OK;
  PB_CUDA(b, cudaEventRecord(b->ev_fork, b->st));
  for (size_t i = 0; i < b->inst.size(); ++i) {
    ps_handle* h = b->inst[i];
    if (h->post_order.empty()) continue;
    PB_CUDA(b, cudaStreamWaitEvent(h->st, b->ev_fork, 0));
    for (int code : h->post_order) {
      int rc = (code == POST_FILTER) ? filter_after_iteration(h, h->iterations)
                                     : poisson_after_iteration(h, h->iterations);
      if (rc) return instance_error(b, (int)i, rc);
    }
    PB_CUDA(b, cudaEventRecord(b->ev_inst[i], h->st));
    PB_CUDA(b, cudaStreamWaitEvent(b->st, b->ev_inst[i], 0));
  }
  return PS_OK;
}

static int batch_autotune(ps_batch* b) {
  PB_CUDA(b, cudaStreamSynchronize(b->st));
  for (BatchClass& c : b->classes) {
    if (c.variant >= 0) continue;
    int best = 0;
    cudaError_t e = (c.prec == PS_PREC_MIXED)
                        ? autotune_sweep_set<float>(class_sweep_set<float>(b, c), c.st, c.tune_ms, &best)
                        : autotune_sweep_set<double>(class_sweep_set<double>(b, c), c.st, c.tune_ms, &best);
    PB_CUDA(b, e);
    c.variant = best;
    // the same kernels as the members' own concurrent chains: one warm-up and
    // one timed pass, forked from and joined back into c.st
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PB_CUDA(b, cudaEventCreate(&e0));
    PB_CUDA(b, cudaEventCreate(&e1));
    float ms = -1.f;
    int rc = PS_OK;
    for (int pass = 0; pass < 2 && rc == PS_OK; ++pass) {
      if (pass == 1) PB_CUDA(b, cudaEventRecord(e0, c.st));
      PB_CUDA(b, cudaEventRecord(b->ev_fork, c.st));
      for (int i : c.members) PB_CUDA(b, cudaStreamWaitEvent(b->inst[i]->st, b->ev_fork, 0));
      long long nl = 0;
      rc = launch_class_chains(b, c, &nl);
      for (int i : c.members) {
        PB_CUDA(b, cudaEventRecord(b->ev_inst[i], b->inst[i]->st));
        PB_CUDA(b, cudaStreamWaitEvent(c.st, b->ev_inst[i], 0));
      }
    }
    if (rc == PS_OK) {
      PB_CUDA(b, cudaEventRecord(e1, c.st));
      PB_CUDA(b, cudaEventSynchronize(e1));
      PB_CUDA(b, cudaEventElapsedTime(&ms, e0, e1));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    c.chains_ms = ms;
    c.chains = (ms >= 0.f && ms < c.tune_ms[best]);
  }
  return PS_OK;
}

static void drop_graph(ps_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
}

static int batch_iterate(ps_batch* b, int n) {
  PB_CUDA(b, cudaSetDevice(b->dev));
  for (int it = 0; it < n; ++it) {
    for (size_t i = 0; i < b->inst.size(); ++i) {
      int rc = engine_prepare_noise(b->inst[i]);
      if (rc) return instance_error(b, (int)i, rc);
    }
    if (b->eager_iters < 1) {
      long long nl = 0;
      int rc = launch_batch_iteration(b, &nl);
      if (rc) return rc;
      b->launches_per_iter = nl;
      b->eager_iters++;
    } else {
      if (!b->gexec) {
        if (b->forced_variant < 0) {
          int rc = batch_autotune(b);
          if (rc) return rc;
        }
        long long nl = 0;
        PB_CUDA(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int rc = launch_batch_iteration(b, &nl);
        cudaGraph_t g = nullptr;
        cudaError_t ec = cudaStreamEndCapture(b->st, &g);
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (ec != cudaSuccess) {
          b->err = std::string("graph capture: ") + cudaGetErrorString(ec);
          return PS_GPU_ERR;
        }
        b->graph = g;
        PB_CUDA(b, cudaGraphInstantiate(&b->gexec, b->graph, 0));
        b->launches_per_iter = nl;
      }
      PB_CUDA(b, cudaGraphLaunch(b->gexec, b->st));
    }
    int rc = run_post_updaters(b);
    if (rc) return rc;
    for (ps_handle* h : b->inst) h->iterations++;
  }
  PB_CUDA(b, cudaStreamSynchronize(b->st));
  for (size_t i = 0; i < b->inst.size(); ++i) {
    int rc = engine_check_scalars(b->inst[i]);
    if (rc) return instance_error(b, (int)i, rc);
  }
  return PS_OK;
}

static void batch_free(ps_batch* b) {
  cudaSetDevice(b->dev);
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graph(b);
  for (BatchClass& c : b->classes) {
    if (c.d_plane) cudaFree(c.d_plane);
    if (c.d_pencil) cudaFree(c.d_pencil);
    if (c.ev) cudaEventDestroy(c.ev);
    if (c.st) cudaStreamDestroy(c.st);
  }
  for (cudaEvent_t e : b->ev_inst)
    if (e) cudaEventDestroy(e);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  for (ps_handle* h : b->inst) ps_gpu_destroy(h);
  if (b->st) cudaStreamDestroy(b->st);
}

static int batch_create(ps_batch* b, const ps_config* cfgs, int count) {
  for (int i = 0; i < count; ++i) {
    if (cfgs[i].device != cfgs[0].device) {
      b->err = "all instances of a batch must be on the same device";
      return PS_ATTRIB_ERR;
    }
  }
  b->dev = cfgs[0].device;
  std::map<std::tuple<int, int, int, int>, int> cls;
  for (int i = 0; i < count; ++i) {
    ps_handle* h = nullptr;
    int rc = ps_gpu_create(&cfgs[i], &h);
    if (rc) {
      b->err = "instance " + std::to_string(i) + ": " + ps_gpu_last_error(nullptr);
      return rc;
    }
    h->in_batch = true;
    b->inst.push_back(h);
    auto key = std::make_tuple(h->n[0], h->n[1], h->n[2], h->prec);
    auto it = cls.find(key);
    int ci;
    if (it == cls.end()) {
      ci = (int)b->classes.size();
      cls[key] = ci;
      BatchClass c;
      for (int d = 0; d < 3; ++d) c.n[d] = h->n[d];
      c.prec = h->prec;
      for (int v = 0; v < VARIANT_COUNT; ++v) c.tune_ms[v] = -1.f;
      b->classes.push_back(c);
    } else {
      ci = it->second;
    }
    b->classes[ci].members.push_back(i);
    b->class_of.push_back(ci);
  }
  PB_CUDA(b, cudaSetDevice(b->dev));
  PB_CUDA(b, cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  PB_CUDA(b, cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  b->ev_inst.assign(count, nullptr);
  for (int i = 0; i < count; ++i) PB_CUDA(b, cudaEventCreateWithFlags(&b->ev_inst[i], cudaEventDisableTiming));
  for (BatchClass& c : b->classes) {
    PB_CUDA(b, cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
    PB_CUDA(b, cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming));
    int rc = (c.prec == PS_PREC_MIXED) ? build_class_tables<float>(b, c) : build_class_tables<double>(b, c);
    if (rc) return rc;
  }
  return PS_OK;
}

}  // namespace psb

using namespace psb;

extern "C" {

int ps_gpu_batch_create(const ps_config* cfgs, int count, ps_batch** out) {
  if (!cfgs || !out || count < 1) {
    g_batch_err = "null argument or empty batch";
    return PS_ATTRIB_ERR;
  }
  *out = nullptr;
  ps_batch* b = new ps_batch();
  int rc = batch_create(b, cfgs, count);
  if (rc != PS_OK) {
    g_batch_err = b->err;
    batch_free(b);
    delete b;
    cudaGetLastError();  // clear a failed allocation's last-error state
    return rc;
  }
  *out = b;
  return PS_OK;
}

int ps_gpu_batch_destroy(ps_batch* b) {
  if (!b) return PS_OK;
  batch_free(b);
  delete b;
  return PS_OK;
}

const char* ps_gpu_batch_last_error(const ps_batch* b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

int ps_gpu_batch_size(const ps_batch* b) { return b ? (int)b->inst.size() : 0; }

ps_handle* ps_gpu_batch_instance(ps_batch* b, int i) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return nullptr;
  return b->inst[i];
}

int ps_gpu_batch_iterate(ps_batch* b, int n_iter) {
  if (!b) return PS_ATTRIB_ERR;
  if (n_iter < 0) {
    b->err = "n_iter must be >= 0";
    return PS_ATTRIB_ERR;
  }
  return batch_iterate(b, n_iter);
}

int ps_gpu_batch_set_variant(ps_batch* b, int variant) {
  if (!b || variant < -1 || variant >= VARIANT_COUNT) return PS_ATTRIB_ERR;
  PB_CUDA(b, cudaSetDevice(b->dev));
  PB_CUDA(b, cudaStreamSynchronize(b->st));
  drop_graph(b);
  b->forced_variant = variant;
  for (BatchClass& c : b->classes) c.variant = -1;
  return PS_OK;
}

int ps_gpu_batch_classes(const ps_batch* b, int* n_classes, int* class_of, int max_inst, int* variants,
                         int max_classes) {
  if (!b || !n_classes) return PS_ATTRIB_ERR;
  *n_classes = (int)b->classes.size();
  for (int i = 0; class_of && i < max_inst && i < (int)b->class_of.size(); ++i) class_of[i] = b->class_of[i];
  for (int c = 0; variants && c < max_classes && c < (int)b->classes.size(); ++c)
    variants[c] = (b->forced_variant >= 0)
                      ? b->forced_variant
                      : (b->classes[c].variant < 0 ? -1
                                                   : (b->classes[c].variant | (b->classes[c].chains ? VARIANT_SPLIT : 0)));
  return PS_OK;
}

long long ps_gpu_batch_launches_per_iteration(const ps_batch* b) { return b ? b->launches_per_iter : 0; }

void* ps_gpu_batch_stream(const ps_batch* b) { return b ? (void*)b->st : nullptr; }

}  // extern "C"
