// Host engine and C-ABI of the B200 SCFT inner loop.
//
// ps_handle owns every device buffer of one SCFT instance: w, phi, p (FP64),
// the propagator slices of each sweep (FP64 or FP32), the half spectra, the
// Boltzmann factors, the k^2 tables, reduction scratch and the Anderson
// history.  One CUDA stream per handle; an iteration is captured once into a
// CUDA graph and replayed.
//
// Semantics follow PsDomain::update (pstrol/PsDomain.cpp:332-372): densities
// reset, PsBlockCopolymer::update for each polymer, then the updater with F
// evaluated on the updated w (pseffhamil/PsSteepDUpdater.cpp:200-201).
#include <math.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "engine_state.h"

namespace psb {

static thread_local std::string g_thread_err;

// PsBlockBase::setBlockSteps (psbase/PsBlockBase.cpp:252-326).
static int set_block_steps(double bs, int force, int* out, std::string& err) {
  long bsint;
  const double intpart = (double)((long)bs);
  const double dx = bs - intpart;
  if (force) {
    bsint = (long)floor(bs + 0.5);
  } else {
    if ((dx > 0.0001) && (dx < 0.9999)) {
      char b[160];
      snprintf(b, sizeof(b), "non-integer # of block steps: blockSteps = %.17g", bs);
      err = b;
      return PS_INPUT_ERR;
    }
    const long c = (long)ceil(bs), f = (long)floor(bs);
    if (c == f) bsint = c;
    else if (fabs(bs - (double)c) < fabs(bs - (double)f)) bsint = c;
    else bsint = f;
  }
  if (bsint < 4) {
    err = "# of block steps too small (< 4)";
    return PS_INPUT_ERR;
  }
  *out = (int)bsint;
  return PS_OK;
}

// Connection end of block `to` that block `from` attaches to
// (PsBlockCopolymer::buildCntBlockType, pspolymer/PsBlockCopolymer.cpp:157-182).
static int joined_end(const ps_polymer_config& P, int from, int to) {
  const ps_block_config& B = P.blocks[to];
  for (int t = 0; t < B.n_tail; ++t)
    if (B.tail_joined[t] == from) return TAIL;
  return HEAD;
}

// Linear-chain sweeps of one polymer.  Returns false for branched or
// inconsistent architectures.
static bool chain_sweeps(const ps_polymer_config& P, std::vector<std::pair<int, int>>& order) {
  const int nb = P.n_blocks;
  auto conns = [&](int b, int e) -> std::vector<int> {
    const ps_block_config& B = P.blocks[b];
    std::vector<int> v;
    if (e == HEAD) v.assign(B.head_joined, B.head_joined + B.n_head);
    else v.assign(B.tail_joined, B.tail_joined + B.n_tail);
    return v;
  };
  for (int b = 0; b < nb; ++b)
    for (int e = 0; e < 2; ++e) {
      auto c = conns(b, e);
      if (c.size() > 1) return false;
      if (c.size() == 1) {
        const int to = c[0];
        if (to < 0 || to >= nb || to == b) return false;
        const int te = joined_end(P, b, to);
        auto back = conns(to, te);
        if (back.size() != 1 || back[0] != b) return false;
      }
    }
  int sb = -1, se = -1;
  for (int b = 0; b < nb && sb < 0; ++b) {
    if (P.blocks[b].n_head == 0) { sb = b; se = HEAD; }
    else if (P.blocks[b].n_tail == 0) { sb = b; se = TAIL; }
  }
  if (sb < 0) return false;
  std::vector<int> seen(nb, 0);
  int b = sb, e = se;
  while (true) {
    if (seen[b]) return false;
    seen[b] = 1;
    order.push_back({b, e});
    const int o = (e == HEAD) ? TAIL : HEAD;
    auto c = conns(b, o);
    if (c.empty()) break;
    const int to = c[0];
    e = joined_end(P, b, to);
    b = to;
  }
  for (int i = 0; i < nb; ++i)
    if (!seen[i]) return false;
  return true;
}

// Sweeps of a branched (tree-shaped) polymer, following the reference's
// dependency-driven solve order (pspolymer/PsBlockCopolymer.cpp:189-313,
// pspolymer/PsBlock.cpp:387-472).  Each directed propagation "block b solved
// from end e" appears in exactly one sweep.  A sweep starts at a free end (q = 1)
// or at a junction of three or more block ends (q = product of the final q of
// the other blocks there), runs through simple block-to-block joins, and stops
// at the next free end or junction.  Sweeps are appended in dependency order.
// Returns an empty string, or why the architecture is not supported.
static std::string tree_sweeps(ps_handle* h, int ip, const ps_polymer_config& P) {
  const int nb = P.n_blocks;
  auto conns = [&](int b, int e) -> std::vector<int> {
    const ps_block_config& B = P.blocks[b];
    std::vector<int> v;
    if (e == HEAD) v.assign(B.head_joined, B.head_joined + B.n_head);
    else v.assign(B.tail_joined, B.tail_joined + B.n_tail);
    std::sort(v.begin(), v.end());  // junction products in ascending block order
    return v;
  };
  for (int b = 0; b < nb; ++b)
    for (int e = 0; e < 2; ++e)
      for (int c : conns(b, e)) {
        if (c < 0 || c >= nb || c == b) return "joined block index out of range";
        const auto back = conns(c, joined_end(P, b, c));
        if (std::find(back.begin(), back.end(), b) == back.end()) return "inconsistent head/tail joins";
      }
  // a simple join: the end meets exactly one other block end, which meets only it
  auto simple = [&](int b, int e) -> bool {
    const auto c = conns(b, e);
    return c.size() == 1 && conns(c[0], joined_end(P, b, c[0])).size() == 1;
  };
  // sweep_of[b][e]: sweep holding "b solved from e"
  std::vector<std::array<int, 2>> sweep_of(nb, {-1, -1});
  std::vector<Sweep> made;
  std::vector<std::vector<std::pair<int, int>>> need;  // (block, end) of each input: solved from that end's far side
  for (int b = 0; b < nb; ++b)
    for (int e = 0; e < 2; ++e) {
      const auto c0 = conns(b, e);
      if (simple(b, e)) continue;  // reached by continuing another sweep
      Sweep sw;
      sw.polymer = ip;
      std::vector<std::pair<int, int>> in;
      for (int c : c0) in.push_back({c, joined_end(P, b, c)});
      int cb = b, ce = e;
      for (int guard = 0; guard <= 2 * nb; ++guard) {
        if (sweep_of[cb][ce] >= 0) return "a block graph with a cycle";
        sweep_of[cb][ce] = (int)made.size();
        Seg g;
        g.block = cb;
        g.from = ce;
        g.off = sw.total;
        g.steps = h->blocks[ip][cb].steps;
        g.wfac_id = g.ktab_id = -1;
        sw.segs.push_back(g);
        sw.total += g.steps;
        const int o = (ce == HEAD) ? TAIL : HEAD;
        if (!simple(cb, o)) break;
        const int nbk = conns(cb, o)[0];
        ce = joined_end(P, cb, nbk);
        cb = nbk;
      }
      made.push_back(sw);
      need.push_back(in);
    }
  for (int b = 0; b < nb; ++b)
    if (sweep_of[b][0] < 0 || sweep_of[b][1] < 0) return "a block graph with a cycle";
  // inputs: the sweep arriving at each joined end (it ends there: a junction stops a sweep)
  std::vector<std::vector<int>> in_sweeps(made.size());
  for (size_t i = 0; i < made.size(); ++i)
    for (auto& ce : need[i]) {
      const int far = (ce.second == HEAD) ? TAIL : HEAD;
      in_sweeps[i].push_back(sweep_of[ce.first][far]);
    }
  // dependency order
  std::vector<int> order, placed(made.size(), 0);
  for (size_t round = 0; round < made.size() && order.size() < made.size(); ++round)
    for (size_t i = 0; i < made.size(); ++i) {
      if (placed[i]) continue;
      bool ready = true;
      for (int j : in_sweeps[i]) ready = ready && placed[j];
      if (ready) {
        placed[i] = 1;
        order.push_back((int)i);
      }
    }
  if (order.size() != made.size()) return "a block graph with a cycle";
  std::vector<int> index_of(made.size());
  const int base = (int)h->sweeps.size();
  for (size_t r = 0; r < order.size(); ++r) index_of[order[r]] = base + (int)r;
  for (int i : order) {
    Sweep sw = made[i];
    for (int j : in_sweeps[i]) sw.jin.push_back({index_of[j], made[j].total});
    if (!sw.jin.empty()) {
      if ((int)sw.jin.size() > PS_MAX_JOINS) return "too many blocks at one junction";
      sw.jbuf = h->n_jbuf++;
      h->branched = true;
    }
    sw.storage = (int)h->exec.size();
    h->exec.push_back((int)h->sweeps.size());
    for (const Seg& g : sw.segs) {
      BlockMap& bm = h->blocks[ip][g.block];
      if (g.from == HEAD) { bm.sweep_head = (int)h->sweeps.size(); bm.off_head = g.off; }
      else { bm.sweep_tail = (int)h->sweeps.size(); bm.off_tail = g.off; }
    }
    h->sweeps.push_back(sw);
  }
  return "";
}

template <typename T>
static int alloc_copy(ps_handle* h, T** dst, const std::vector<T>& src) {
  PS_CUDA(h, cudaMalloc((void**)dst, sizeof(T) * std::max<size_t>(src.size(), 1)));
  PS_CUDA(h, cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  return PS_OK;
}

template <typename T>
static int make_twiddles(ps_handle* h, c2_t<T>** dst, int L) {
  std::vector<c2_t<T>> tw(std::max(L, 1));
  const double twopi = 2.0 * acos(-1.0);
  for (int m = 0; m < L; ++m) {
    const double a = twopi * (double)m / (double)L;
    tw[m].x = (T)cos(a);
    tw[m].y = (T)(-sin(a));
  }
  return alloc_copy(h, dst, tw);
}

// Separable exp(-ds b^2 k^2): kx carries the 1/N of the unnormalised pair
// (pspolymer/PsFlexPseudoSpec.cpp:152, :188-206; psbase/PsGridField.cpp:66-104).
static double kcomp(int i, int n, double dx) {
  const double twopi = 2.0 * acos(-1.0);
  const double n2 = (double)n / 2.0;
  const double nk = n2 - fabs((double)i - n2);
  double k = twopi * nk / (double)n;
  return k / dx;
}

// The FP32 sweeps carry their mean mode in FP64 (PlaneWork in kernels.h) unless
// the environment sets PSB_DC_CARRY=0 (kept to measure what the carry buys).
static bool dc_carry_enabled() {
  const char* e = getenv("PSB_DC_CARRY");
  return !(e && e[0] == '0');
}

template <typename T>
static int build_device_tables(ps_handle* h) {
  Buffers<T>& B = bufs<T>(h);
  const long long N = h->N;
  // slices + spectra
  for (int s : h->exec) {
    const Sweep& sw = h->sweeps[s];
    T* sl = nullptr;
    if (!h->no_slices) PS_CUDA(h, cudaMalloc((void**)&sl, sizeof(T) * (size_t)(sw.total + 1) * N));
    B.slices.push_back(sl);
    c2_t<T>* sp = nullptr;
    PS_CUDA(h, cudaMalloc((void**)&sp, sizeof(c2_t<T>) * (size_t)h->n[0] * h->n[1] * h->nzh));
    B.spec.push_back(sp);
  }
  for (size_t i = 0; i < h->wfac_keys.size(); ++i) {
    T* wf = nullptr;
    PS_CUDA(h, cudaMalloc((void**)&wf, sizeof(T) * (size_t)N));
    B.wfac.push_back(wf);
  }
  for (int i = 0; i < h->n_jbuf; ++i) {
    T* jb = nullptr;
    PS_CUDA(h, cudaMalloc((void**)&jb, sizeof(T) * (size_t)N));
    B.jbuf.push_back(jb);
  }
  // Mean-mode carry of the FP32 sweeps: one buffer per executed sweep, room for
  // a partial per CTA of any plane/row pass variant (fused plane: nx, cluster:
  // 8 nx, row passes: at least 8 rows per CTA).
  if (sizeof(T) == 4 && dc_carry_enabled()) {
    B.dc_cap = std::max(kDcMinSlots, std::max(8 * h->n[0], (h->n[0] * h->n[1] + 7) / 8));
    for (size_t e = 0; e < h->exec.size(); ++e) {
      double* d = nullptr;
      PS_CUDA(h, cudaMalloc((void**)&d, sizeof(double) * (size_t)(B.dc_cap + 3)));
      B.dcbuf.push_back(d);
      PS_CUDA(h, cudaMemset(d, 0, sizeof(double) * (size_t)(B.dc_cap + 3)));
    }
  }
  for (auto& kk : h->ktab_keys) {
    const double ds = kk.first, b = kk.second;
    std::vector<T> kx(h->n[0]), kyz((size_t)h->n[1] * h->nzh);
    for (int i = 0; i < h->n[0]; ++i) {
      const double k = kcomp(i, h->n[0], h->cfg.cell[0]);
      kx[i] = (T)(exp(-1.0 * ds * (k * k) * b * b) / (double)N);
    }
    for (int j = 0; j < h->n[1]; ++j) {
      const double ky = kcomp(j, h->n[1], h->cfg.cell[1]);
      for (int kz = 0; kz < h->nzh; ++kz) {
        const double kzv = kcomp(kz, h->n[2], h->cfg.cell[2]);
        kyz[(size_t)j * h->nzh + kz] =
            (T)(exp(-1.0 * ds * (ky * ky) * b * b) * exp(-1.0 * ds * (kzv * kzv) * b * b));
      }
    }
    T* dkx = nullptr;
    T* dkyz = nullptr;
    int rc = alloc_copy(h, &dkx, kx);
    if (rc) return rc;
    rc = alloc_copy(h, &dkyz, kyz);
    if (rc) return rc;
    B.kx.push_back(dkx);
    B.kyz.push_back(dkyz);
  }
  int rc = make_twiddles<T>(h, &B.tw_x, h->n[0]);
  if (!rc) rc = make_twiddles<T>(h, &B.tw_y, h->n[1]);
  if (!rc) rc = make_twiddles<T>(h, &B.tw_z, h->n[2]);
  if (!rc) rc = make_twiddles<T>(h, &B.tw_zh, std::max(h->n[2] / 2, 1));
  if (rc) return rc;

  // Work tables for every global step.
  std::vector<PlaneWork<T>> pw;
  std::vector<PencilWork<T>> xw;
  h->plane_off.assign(h->kmax + 1, 0);
  h->plane_cnt.assign(h->kmax + 1, 0);
  h->pencil_off.assign(h->kmax + 1, 0);
  h->pencil_cnt.assign(h->kmax + 1, 0);
  auto seg_of = [&](const Sweep& sw, int step) -> const Seg& {
    for (const Seg& g : sw.segs)
      if (step >= g.off && step < g.off + g.steps) return g;
    return sw.segs.back();
  };
  const size_t ne = h->exec.size();
  h->sw_plane_off.assign(ne, std::vector<int>(h->kmax + 1, 0));
  h->sw_plane_cnt.assign(ne, std::vector<int>(h->kmax + 1, 0));
  h->sw_pencil_off.assign(ne, std::vector<int>(h->kmax + 1, 0));
  h->sw_pencil_cnt.assign(ne, std::vector<int>(h->kmax + 1, 0));
  for (int k = 0; k <= h->kmax; ++k) {
    h->plane_off[k] = (int)pw.size();
    h->pencil_off[k] = (int)xw.size();
    for (size_t e = 0; e < h->exec.size(); ++e) {
      const Sweep& sw = h->sweeps[h->exec[e]];
      const int kg = k;                    // global step
      const int kl = kg - h->sw_start[e];  // this sweep's own step
      if (kl < 0 || kl > sw.total) continue;
      h->sw_plane_off[e][kg] = (int)pw.size();
      h->sw_plane_cnt[e][kg] = 1;
      if (kl < sw.total) {
        h->sw_pencil_off[e][kg] = (int)xw.size();
        h->sw_pencil_cnt[e][kg] = 1;
      }
      PlaneWork<T> w;
      memset(&w, 0, sizeof(w));
      w.mode = (kl == 0) ? MODE_FIRST : (kl == sw.total ? MODE_LAST : MODE_MID);
      w.src = (kl == 0 && sw.jbuf >= 0) ? B.jbuf[sw.jbuf] : nullptr;
      w.spec = B.spec[e];
      w.wfac_in = (kl > 0) ? B.wfac[seg_of(sw, kl - 1).wfac_id] : nullptr;
      w.wfac_out = (kl < sw.total) ? B.wfac[seg_of(sw, kl).wfac_id] : nullptr;
      w.store = B.slices[e] ? B.slices[e] + (size_t)kl * N : nullptr;
      w.status = &h->d_sc->error_flags;
      double* dc = B.dcbuf.empty() ? nullptr : B.dcbuf[e];
      if (dc) {
        if (w.mode != MODE_FIRST) w.dc_in = dc + B.dc_cap;
        if (w.mode != MODE_LAST) {
          w.dc_out = dc;
          w.dc_count = dc + B.dc_cap + 1;
        }
      }
      pw.push_back(w);
      if (kl < sw.total) {
        PencilWork<T> x;
        memset(&x, 0, sizeof(x));
        x.spec = B.spec[e];
        x.kx = B.kx[seg_of(sw, kl).ktab_id];
        x.kyz = B.kyz[seg_of(sw, kl).ktab_id];
        if (dc) {
          x.dc_parts = dc;
          x.dc_count = dc + B.dc_cap + 1;
          x.dc_total = dc + B.dc_cap;
          x.dc_err = dc + B.dc_cap + 2;
          x.dc_scale = 1.0 / (double)N;
          x.dc_first = (kl == 0) ? 1 : 0;
        }
        xw.push_back(x);
      }
    }
    h->plane_cnt[k] = (int)pw.size() - h->plane_off[k];
    h->pencil_cnt[k] = (int)xw.size() - h->pencil_off[k];
  }
  rc = alloc_copy(h, &B.d_plane, pw);
  if (!rc) rc = alloc_copy(h, &B.d_pencil, xw);
  B.h_plane = pw;
  B.h_pencil = xw;
  // junction starts for lockstep launches, before the leaving sweep's first step
  B.junc.clear();
  h->junc_off.assign(h->kmax + 1, 0);
  h->junc_cnt.assign(h->kmax + 1, 0);
  for (int k = 0; k <= h->kmax; ++k) {
    h->junc_off[k] = (int)B.junc.size();
    for (size_t e = 0; e < h->exec.size(); ++e) {
      const Sweep& sw = h->sweeps[h->exec[e]];
      if (sw.jbuf < 0 || h->sw_start[e] != k) continue;
      JunctionLaunch<T> jl;
      memset(&jl, 0, sizeof(jl));
      jl.in.n = (int)sw.jin.size();
      for (int i = 0; i < jl.in.n; ++i)
        jl.in.q[i] = B.slices[h->sweeps[sw.jin[i].first].storage] + (size_t)sw.jin[i].second * N;
      jl.out = B.jbuf[sw.jbuf];
      jl.n = N;
      B.junc.push_back(jl);
    }
    h->junc_cnt[k] = (int)B.junc.size() - h->junc_off[k];
  }
  return rc;
}

// Launch the propagator sweeps of one iteration.
template <typename T>
static int launch_sweeps(ps_handle* h, long long* nlaunch, int variant) {
  if (!(variant & VARIANT_SPLIT) || h->sw_st.empty()) {
    // lockstep: every sweep's step in shared launches, junction starts between steps
    PS_CUDA(h, launch_sweep_set<T>(handle_sweep_set<T>(h), variant, h->st, nlaunch));
    return PS_OK;
  }
  // one launch chain per executed sweep, forked from and joined back into h->st
  PS_CUDA(h, cudaEventRecord(h->ev_split, h->st));
  for (size_t e = 0; e < h->sw_st.size(); ++e) {
    SweepSet<T> s = handle_sweep_set<T>(h);
    s.plane_off = h->sw_plane_off[e].data();
    s.plane_cnt = h->sw_plane_cnt[e].data();
    s.pencil_off = h->sw_pencil_off[e].data();
    s.pencil_cnt = h->sw_pencil_cnt[e].data();
    s.junc = nullptr;  // this chain launches its own junction start below
    PS_CUDA(h, cudaStreamWaitEvent(h->sw_st[e], h->ev_split, 0));
    const Sweep& sw = h->sweeps[h->exec[e]];
    if (sw.jbuf >= 0) {
      // junction start (PsBlock::combineSetJnt): after the arriving sweeps
      Buffers<T>& B = bufs<T>(h);
      JunctionIn<T> in;
      memset(&in, 0, sizeof(in));
      in.n = (int)sw.jin.size();
      for (int i = 0; i < in.n; ++i) {
        const int es = h->sweeps[sw.jin[i].first].storage;
        PS_CUDA(h, cudaStreamWaitEvent(h->sw_st[e], h->sw_ev[es], 0));
        in.q[i] = B.slices[es] + (size_t)sw.jin[i].second * h->N;
      }
      PS_CUDA(h, launch_junction<T>(in, h->N, B.jbuf[sw.jbuf], h->sw_st[e]));
      ++*nlaunch;
    }
    PS_CUDA(h, launch_sweep_set<T>(s, variant & ~VARIANT_SPLIT, h->sw_st[e], nlaunch));
    PS_CUDA(h, cudaEventRecord(h->sw_ev[e], h->sw_st[e]));
    PS_CUDA(h, cudaStreamWaitEvent(h->st, h->sw_ev[e], 0));
  }
  return PS_OK;
}

template <typename T>
static int launch_pre(ps_handle* h, long long* nlaunch) {
  Buffers<T>& B = bufs<T>(h);
  const long long N = h->N;
  PS_CUDA(h, launch_zero(h->d_phi, (long long)h->nf * N, h->st));
  ++*nlaunch;
  if (h->nq > 0) {
    // PsChargeDens::update: resetDensField (psphysf/PsChargeDens.cpp:180-190)
    PS_CUDA(h, launch_zero(h->d_rho, (long long)h->nq * N, h->st));
    ++*nlaunch;
  }
  for (size_t i = 0; i < h->wfac_keys.size(); ++i) {
    const WfacKey& k = h->wfac_keys[i];
    if (k.charge_field < 0)
      PS_CUDA(h, launch_wfac<T>(h->d_w + (size_t)k.field * N, B.wfac[i], -0.5 * k.ds, N, h->st));
    else
      PS_CUDA(h, launch_wfac_charged<T>(h->d_w + (size_t)k.field * N, h->d_psi + (size_t)k.charge_field * N,
                                        B.wfac[i], -0.5 * k.ds, k.facz, N, h->st));
    ++*nlaunch;
  }
  return PS_OK;
}

template <typename T> static int launch_post(ps_handle* h, long long* nlaunch);

template <typename T>
static int launch_iteration(ps_handle* h, long long* nlaunch) {
  // this iteration's updater noise, drawn beside the sweeps
  int rc = noise_launch(h, nlaunch);
  if (rc) return rc;
  rc = launch_pre<T>(h, nlaunch);
  if (rc) return rc;
  // cudaEventRecordExternal: inside stream capture this becomes an event-record
  // node of the graph (a plain record would only order the capture).
  if (h->timing_cap > 0)
    PS_CUDA(h, cudaEventRecordWithFlags(h->ev_cap_start, h->st, cudaEventRecordExternal));
  rc = launch_sweeps<T>(h, nlaunch, h->variant < 0 ? (h->branched ? VARIANT_SPLIT : 0) : h->variant);
  if (rc) return rc;
  if (h->timing_cap > 0)
    PS_CUDA(h, cudaEventRecordWithFlags(h->ev_cap_end, h->st, cudaEventRecordExternal));
  return launch_post<T>(h, nlaunch);
}

template <typename T>
static int launch_post(ps_handle* h, long long* nlaunch) {
  Buffers<T>& B = bufs<T>(h);
  const long long N = h->N;
  auto slice = [&](int sweep, int idx) -> const T* {
    return B.slices[h->sweeps[sweep].storage] + (size_t)idx * N;
  };
  // solvents before polymers (PsDomain::update, pstrol/PsDomain.cpp:359-362)
  for (int is = 0; is < h->cfg.n_solvents; ++is) {
    const ps_solvent_config& S = h->cfg.solvents[is];
    if (S.kind == PS_SOLV_IONS)
      PS_CUDA(h, launch_ions(h->d_psi + (size_t)S.charge_field * N, S.zc, S.neutral_factor, N, is,
                             h->d_qpart, h->d_sc, h->d_rho + (size_t)S.charge_field * N,
                             S.has_block_field ? h->d_rho + (size_t)S.block_field * N : nullptr, h->st));
    else
      PS_CUDA(h, launch_solvent(h->d_w + (size_t)S.field * N, -1.0 / h->fm.scale_len, S.volfrac, N, is,
                                h->d_qpart, h->d_sc, h->d_phi + (size_t)S.field * N, h->st));
    *nlaunch += 3;
  }
  for (int ip = 0; ip < h->cfg.n_polymers; ++ip) {
    const BlockMap& b0 = h->blocks[ip][0];
    PS_CUDA(h, launch_dot_partials<T>(slice(b0.sweep_head, b0.off_head),
                                      slice(b0.sweep_tail, b0.off_tail + b0.steps), N, h->d_qpart,
                                      h->st));
    PS_CUDA(h, launch_finalize_q(h->d_qpart, (double)N, ip, h->d_sc, h->st));
    *nlaunch += 2;
  }
  for (int ip = 0; ip < h->cfg.n_polymers; ++ip) {
    // densWt vf / lengthRatio (pspolymer/PsBlock.cpp:164-172); densWt = 1 or w_k / Gamma(alpha)
    const double densfac = h->chain_dwt[ip] * h->chain_vf[ip] / h->alpha[ip];
    for (size_t ib = 0; ib < h->blocks[ip].size(); ++ib) {
      const BlockMap& b = h->blocks[ip][ib];
      PS_CUDA(h, launch_quadrature<T>(slice(b.sweep_head, b.off_head), slice(b.sweep_tail, b.off_tail),
                                      b.steps, N, b.ds, densfac, h->d_sc, ip,
                                      h->d_phi + (size_t)b.field * N, h->st));
      ++*nlaunch;
      if (b.charge_field >= 0) {
        // the charged block is the only density source of its field, so phi_f here
        // is what PsChargeFlexPseudoSpec::setPhysFields reads
        PS_CUDA(h, launch_charge_accum(h->d_phi + (size_t)b.field * N, b.qalpha, b.za, N,
                                       h->d_rho + (size_t)b.charge_field * N, h->st));
        ++*nlaunch;
      }
    }
  }
  // the field update is the first reader of p: wait for an asynchronous upload
  // of it (an external event-wait node when this is being captured)
  if (h->p_ready) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PS_CUDA(h, cudaStreamIsCapturing(h->st, &cs));
    PS_CUDA(h, cudaStreamWaitEvent(h->st, h->p_ready,
                                   cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0));
  }
  FieldPtrs fp;
  memset(&fp, 0, sizeof(fp));
  for (int i = 0; i < h->nf; ++i) {
    fp.w[i] = h->d_w + (size_t)i * N;
    fp.phi[i] = h->d_phi + (size_t)i * N;
  }
  fp.p = h->d_p;
  fp.noise = (h->cfg.updater.noise != 0.0) ? h->d_noise : nullptr;
  if (fp.noise) {
    int rc = noise_join(h);
    if (rc) return rc;
  }
  if (h->cfg.updater.kind == PS_UPD_ANDERSON) {
    const int m = h->cfg.updater.anderson_depth;
    PS_CUDA(h, launch_am_residual(h->fm, fp, h->d_hw, h->d_hd, h->am_slots, h->d_sc, h->d_upart, h->st));
    PS_CUDA(h, launch_am_gram((long long)h->nf * N, h->d_hd, h->am_slots, m, h->d_sc, h->d_gpart, h->st));
    PS_CUDA(h, launch_am_solve(h->d_gpart, h->d_gram, h->am_slots, m, h->cfg.updater.anderson_start,
                               h->cfg.updater.anderson_mix, h->cfg.updater.lambda0, h->d_sc, h->st));
    PS_CUDA(h, launch_am_mix(h->fm, fp, h->d_hw, h->d_hd, h->am_slots, h->d_sc, h->d_upart, h->st));
    PS_CUDA(h, launch_update_finalize_am(h->fm, h->d_upart, h->d_sc, h->st));
    *nlaunch += 5;
  } else {
    PS_CUDA(h, launch_sd_update(h->fm, fp, h->d_upart, h->st));
    PS_CUDA(h, launch_update_finalize(h->fm, h->d_upart, h->d_sc, h->st));
    *nlaunch += 2;
  }
  PS_CUDA(h, launch_pressure_shift(h->d_p, N, h->d_sc, h->st));
  ++*nlaunch;
  return PS_OK;
}

// Time every kernel variant on this instance's own sweeps (same inputs, one
// warm-up and one timed sweep each) and keep the fastest.
template <typename T>
static int autotune_t(ps_handle* h) {
  cudaEvent_t a = nullptr, b = nullptr;
  PS_CUDA(h, cudaEventCreate(&a));
  cudaError_t e = cudaEventCreate(&b);
  float best = 1e30f;
  int best_v = 0;
  int rc = PS_OK;
  for (int v = 0; v < VARIANT_COUNT && e == cudaSuccess && rc == PS_OK; ++v) {
    h->tune_ms[v] = -1.f;
    if ((v & VARIANT_XY) && (!h->xy_ok || (v & VARIANT_FUSE_Z))) continue;  // absent / same
    if ((v & VARIANT_CLUSTER) && (!h->cluster_ok || (v & VARIANT_XY))) continue;
    if ((v & VARIANT_SPLIT) && h->sw_st.empty()) continue;                 // one sweep only
    long long nl = 0;
    rc = launch_sweeps<T>(h, &nl, v);  // warm-up
    if (rc == PS_OK) e = cudaEventRecord(a, h->st);
    if (rc == PS_OK && e == cudaSuccess) rc = launch_sweeps<T>(h, &nl, v);
    if (rc == PS_OK && e == cudaSuccess) e = cudaEventRecord(b, h->st);
    if (rc == PS_OK && e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (rc == PS_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (rc != PS_OK || e != cudaSuccess) break;
    h->tune_ms[v] = ms;
    if (ms < best) {
      best = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (rc) return rc;
  PS_CUDA(h, e);
  h->variant = best_v;
  return PS_OK;
}

static int autotune(ps_handle* h) {
  return (h->prec == PS_PREC_MIXED) ? autotune_t<float>(h) : autotune_t<double>(h);
}

static int run_iteration(ps_handle* h, long long* nlaunch) {
  return (h->prec == PS_PREC_MIXED) ? launch_iteration<float>(h, nlaunch)
                                    : launch_iteration<double>(h, nlaunch);
}

int engine_pre(ps_handle* h, long long* nlaunch) {
  return (h->prec == PS_PREC_MIXED) ? launch_pre<float>(h, nlaunch) : launch_pre<double>(h, nlaunch);
}

int engine_sweeps(ps_handle* h, long long* nlaunch, int variant) {
  return (h->prec == PS_PREC_MIXED) ? launch_sweeps<float>(h, nlaunch, variant)
                                    : launch_sweeps<double>(h, nlaunch, variant);
}

int engine_post(ps_handle* h, long long* nlaunch) {
  return (h->prec == PS_PREC_MIXED) ? launch_post<float>(h, nlaunch) : launch_post<double>(h, nlaunch);
}

// Bring the host generator up to date before the host reads it: take back the
// state of device draws, then make the Gaussian draws the reference makes every
// iteration even at noise = 0 (pseffhamil/PsPolymerUpdater.cpp:263-295), which
// are owed to the stream and drawn lazily.
static int settle_rng(ps_handle* h) {
  int rc = noise_download(h);
  if (rc) return rc;
  while (h->pending_gauss > 0) {
    (void)h->rng.gauss();
    --h->pending_gauss;
  }
  return PS_OK;
}

int engine_prepare_noise(ps_handle* h) {
  if (h->cfg.updater.noise == 0.0) {
    h->pending_gauss += (long long)h->nf * h->N;
    return PS_OK;
  }
  // The draws themselves are kernels of the iteration (noise_launch).  The
  // generator moves to the device once and stays there until the host draws
  // again, so no iteration waits on the host.
  if (h->pending_gauss > 0) {
    int rc = settle_rng(h);
    if (rc) return rc;
  }
  return noise_upload(h);
}

template <typename T> static void free_buffers(Buffers<T>& B) {
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (auto p : B.slices) f(p);
  for (auto p : B.spec) f(p);
  for (auto p : B.wfac) f(p);
  for (auto p : B.jbuf) f(p);
  for (auto p : B.dcbuf) f(p);
  for (auto p : B.kx) f(p);
  for (auto p : B.kyz) f(p);
  f(B.tw_x); f(B.tw_y); f(B.tw_z); f(B.tw_zh); f(B.d_plane); f(B.d_pencil);
  B = Buffers<T>();
}

static void free_all(ps_handle* h) {
  noise_free(h);
  filter_free(h);
  poisson_free(h);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(h->d_w); f(h->d_phi); f(h->d_p); f(h->d_noise); f(h->d_rho); f(h->d_psi);
  free_buffers(h->bf);
  free_buffers(h->bd);
  f(h->d_qpart); f(h->d_upart); f(h->d_sc);
  if (h->h_sc) cudaFreeHost(h->h_sc);
  f(h->d_hw); f(h->d_hd); f(h->d_gram); f(h->d_gpart);
  if (h->ev_cap_start) cudaEventDestroy(h->ev_cap_start);
  if (h->ev_cap_end) cudaEventDestroy(h->ev_cap_end);
  for (auto e : h->ev_start) cudaEventDestroy(e);
  for (auto e : h->ev_end) cudaEventDestroy(e);
  for (auto s : h->sw_st) cudaStreamDestroy(s);
  for (auto e : h->sw_ev) cudaEventDestroy(e);
  if (h->ev_split) cudaEventDestroy(h->ev_split);
  if (h->io_st) cudaStreamSynchronize(h->io_st);
  for (auto& kv : h->read_slots) {
    f(kv.second.d);
    if (kv.second.snap) cudaEventDestroy(kv.second.snap);
    if (kv.second.done) cudaEventDestroy(kv.second.done);
  }
  h->read_slots.clear();
  if (h->io_st) cudaStreamDestroy(h->io_st);
  if (h->up_st) cudaStreamSynchronize(h->up_st);
  if (h->up_st) cudaStreamDestroy(h->up_st);
  if (h->up_ev) cudaEventDestroy(h->up_ev);
  if (h->p_ready) cudaEventDestroy(h->p_ready);
  if (h->st) cudaStreamDestroy(h->st);
}

static int create_impl(ps_handle* h, const ps_config* ucfg) {
  h->ucfg = *ucfg;
  {
    int rc = expand_polydisperse(h, *ucfg, &h->cfg);
    if (rc) return rc;
  }
  const ps_config& c = h->cfg;
  for (int d = 0; d < 3; ++d) {
    h->n[d] = c.n[d];
    if (!extent_supported(c.n[d])) {
      h->err = "unsupported grid extent " + std::to_string(c.n[d]) +
               " (supported: 1,4,8,12,16,24,32,48,64,96,128,256)";
      return PS_INPUT_ERR;
    }
    if (!(c.cell[d] > 0.0)) {
      h->err = "cellSizes must be positive";
      return PS_ATTRIB_ERR;
    }
  }
  h->N = (long long)c.n[0] * c.n[1] * c.n[2];
  h->nzh = c.n[2] / 2 + 1;
  h->nf = c.n_fields;
  h->prec = c.precision;
  if (h->prec != PS_PREC_FP64 && h->prec != PS_PREC_MIXED) {
    h->err = "precision must be PS_PREC_FP64 or PS_PREC_MIXED";
    return PS_ATTRIB_ERR;
  }
  if (h->nf < 2 || h->nf > 3) {
    h->err = "n_fields must be 2 or 3 (the steepest-descent updater supports 2 or 3)";
    return PS_ATTRIB_ERR;
  }
  if (c.n_polymers < 1 || c.n_polymers > PS_MAX_POLYMERS) {
    h->err = "n_polymers out of range";
    return PS_ATTRIB_ERR;
  }
  if (c.n_interactions < 0 || c.n_interactions > PS_MAX_INTERACTIONS) {
    h->err = "n_interactions out of range";
    return PS_ATTRIB_ERR;
  }
  if (c.updater.kind == PS_UPD_ANDERSON &&
      (c.updater.anderson_depth < 1 || c.updater.anderson_depth > 32)) {
    h->err = "anderson_depth must be in 1..32";
    return PS_ATTRIB_ERR;
  }
  // Polymers, blocks, steps, density averages (psbase/PsBlockBase.cpp:163-204,
  // pspolymer/PsPolymerHldr.cpp:67-83, pspolymer/PsBlockCopolymer.cpp:113-127).
  const double scale_len = (double)c.polymers[0].length;
  double dens_avg[PS_MAX_FIELDS] = {0, 0, 0, 0};
  double vtot = 0.0;
  h->blocks.resize(c.n_polymers);
  for (int ip = 0; ip < c.n_polymers; ++ip) {
    const ps_polymer_config& P = c.polymers[ip];
    if (P.n_blocks < 1 || P.n_blocks > PS_MAX_BLOCKS) {
      h->err = "polymer " + std::to_string(ip) + ": n_blocks out of range";
      return PS_ATTRIB_ERR;
    }
    if (P.length <= 0) {
      h->err = "polymer " + std::to_string(ip) + ": length must be positive";
      return PS_ATTRIB_ERR;
    }
    const double alpha = (double)P.length / scale_len;
    h->alpha.push_back(alpha);
    const ps_polydisperse_config& D = c.polydisperse[ip];
    if (h->chain_k[ip] == 0) vtot += h->chain_vf[ip];
    double ftot = 0.0;
    for (int ib = 0; ib < P.n_blocks; ++ib) ftot = ftot + P.blocks[ib].lengthfrac;
    if (!D.enabled && fabs(ftot - 1.0) > 0.00001) {
      h->err = "polymer " + std::to_string(ip) + ": |totalFrac - 1.0| > tolerance";
      return PS_INPUT_ERR;
    }
    for (int ib = 0; ib < P.n_blocks; ++ib) {
      const ps_block_config& B = P.blocks[ib];
      if (B.field < 0 || B.field >= h->nf) {
        h->err = "block field index out of range";
        return PS_ATTRIB_ERR;
      }
      if (!(B.ds > 0.0)) {
        h->err = "ds not set";
        return PS_ATTRIB_ERR;
      }
      // lengthWeight: 1; for a polydisperse chain w_k / Gamma(alpha) on the polydisperse
      // block and 1 / n_g on the other (pspolymer/PsPolyDisperseBCP.cpp:458-480)
      const double lwt = !D.enabled ? 1.0 : (ib == D.poly_block ? h->chain_dwt[ip] : 1.0 / (double)D.n_g);
      dens_avg[B.field] = dens_avg[B.field] + lwt * B.lengthfrac * h->chain_vf[ip];
      BlockMap bm;
      memset(&bm, 0, sizeof(bm));
      std::string e2;
      int rc = set_block_steps(alpha * B.lengthfrac / B.ds, B.force_block_steps, &bm.steps, e2);
      if (rc) {
        h->err = "polymer " + std::to_string(ip) + " block " + std::to_string(ib) + ": " + e2;
        return rc;
      }
      bm.field = B.field;
      bm.ds = B.ds;
      bm.bseg = (B.bseg_ratio > 0.0) ? B.bseg_ratio : 1.0;
      const ps_block_charge& Z = c.block_charge[ip][ib];
      bm.charge_field = -1;
      if (Z.charged) {
        if (c.n_charges < 1 || c.n_charges > PS_MAX_CHARGES || Z.charge_field < 0 ||
            Z.charge_field >= c.n_charges) {
          h->err = "polymer " + std::to_string(ip) + " block " + std::to_string(ib) +
                   ": chargefield out of range";
          return PS_ATTRIB_ERR;
        }
        bm.charge_field = Z.charge_field;
        bm.za = Z.za;
        bm.qalpha = Z.alpha;
        // facZ = za alpha N (pspolymer/PsChargeFlexPseudoSpec.cpp:104-106)
        bm.facz = Z.za * Z.alpha * scale_len;
      }
      h->blocks[ip].push_back(bm);
    }
  }
  // polyDisperseBCP length-fraction check over all quadrature blocks
  // (pspolymer/PsPolyDisperseBCP.cpp:246-274)
  for (int up = 0; up < h->ucfg.n_polymers; ++up) {
    const ps_polydisperse_config& D = h->ucfg.polydisperse[up];
    if (!D.enabled) continue;
    double tot = 0.0;
    for (int ib = 0; ib < h->ucfg.polymers[up].n_blocks; ++ib)
      for (int k = 0; k < D.n_g; ++k) {
        const int ch = h->user_first[up] + k;
        const double lwt = (ib == D.poly_block) ? h->chain_dwt[ch] : 1.0 / (double)D.n_g;
        tot = tot + c.polymers[ch].blocks[ib].lengthfrac * lwt;
      }
    if (fabs(tot - 1.0) > 0.00001) {
      h->err = "PsPolyDisperseBCP::buildData: |totalFrac - 1.0| > tolerance";
      return PS_INPUT_ERR;
    }
  }
  // simpleSolvent: density average and volume fraction (pssolvent/PsSimpleSolvent.cpp:56-80,
  // psphysf/PsPhysFieldHldr.cpp:190-257)
  if (c.n_solvents < 0 || c.n_solvents > PS_MAX_SOLVENTS) {
    h->err = "n_solvents out of range";
    return PS_ATTRIB_ERR;
  }
  if (c.n_charges < 0 || c.n_charges > PS_MAX_CHARGES) {
    h->err = "n_charges out of range";
    return PS_ATTRIB_ERR;
  }
  h->nq = c.n_charges;
  for (int is = 0; is < c.n_solvents; ++is) {
    const ps_solvent_config& S = c.solvents[is];
    if (S.field < 0 || S.field >= h->nf) {
      h->err = "solvent " + std::to_string(is) + ": scfield out of range";
      return PS_ATTRIB_ERR;
    }
    if (S.kind == PS_SOLV_IONS) {
      if (S.charge_field < 0 || S.charge_field >= h->nq ||
          (S.has_block_field && (S.block_field < 0 || S.block_field >= h->nq)) || S.zc == 0.0) {
        h->err = "solvent " + std::to_string(is) +
                 ": simpleIons needs chargefield (and blockfield) and zc != 0";
        return PS_ATTRIB_ERR;
      }
    } else if (S.kind == PS_SOLV_SIMPLE) {
      dens_avg[S.field] = dens_avg[S.field] + S.volfrac;
    } else {
      h->err = "solvent " + std::to_string(is) + ": unknown kind";
      return PS_ATTRIB_ERR;
    }
  }
  // A charged block must be the only density source of its scfield: its
  // rho += za alpha phi_f then sees its own density, as the reference's does.
  for (int ip = 0; ip < c.n_polymers; ++ip)
    for (size_t ib = 0; ib < h->blocks[ip].size(); ++ib) {
      const BlockMap& b = h->blocks[ip][ib];
      if (b.charge_field < 0) continue;
      int others = 0;
      for (int jp = 0; jp < c.n_polymers; ++jp)
        for (size_t jb = 0; jb < h->blocks[jp].size(); ++jb)
          if ((jp != ip || jb != ib) && h->blocks[jp][jb].field == b.field) ++others;
      for (int is = 0; is < c.n_solvents; ++is)
        if (c.solvents[is].kind == PS_SOLV_SIMPLE && c.solvents[is].field == b.field) ++others;
      if (others) {
        h->err = "polymer " + std::to_string(ip) + " block " + std::to_string(ib) +
                 ": a charged block must be the only density source of its scfield";
        return PS_INPUT_ERR;
      }
    }
  double vsolv = 0.0;
  for (int is = 0; is < c.n_solvents; ++is) vsolv += c.solvents[is].volfrac;
  vtot = vsolv + vtot;
  if (fabs(vtot - 1.0) > 0.00001) {
    h->err = "sum of polymer and solvent volume fractions != 1";
    return PS_INPUT_ERR;
  }
  // Sweeps
  for (int ip = 0; ip < c.n_polymers; ++ip) {
    const ps_polymer_config& P = c.polymers[ip];
    std::vector<std::pair<int, int>> order;
    if (!chain_sweeps(P, order)) {
      const std::string why = tree_sweeps(h, ip, P);
      if (!why.empty()) {
        h->err = "polymer " + std::to_string(ip) + ": " + why;
        return PS_INPUT_ERR;
      }
      continue;
    }
    Sweep a, b;
    a.polymer = b.polymer = ip;
    for (auto& be : order) {
      Seg g;
      g.block = be.first;
      g.from = be.second;
      g.off = a.total;
      g.steps = h->blocks[ip][g.block].steps;
      g.wfac_id = g.ktab_id = -1;
      a.segs.push_back(g);
      a.total += g.steps;
    }
    for (int i = (int)order.size() - 1; i >= 0; --i) {
      Seg g;
      g.block = order[i].first;
      g.from = (order[i].second == HEAD) ? TAIL : HEAD;
      g.off = b.total;
      g.steps = h->blocks[ip][g.block].steps;
      g.wfac_id = g.ktab_id = -1;
      b.segs.push_back(g);
      b.total += g.steps;
    }
    // Mirror-symmetric chains (homopolymers, ABA) give identical sweeps.
    bool same = (a.segs.size() == b.segs.size());
    for (size_t i = 0; same && i < a.segs.size(); ++i) {
      const BlockMap& x = h->blocks[ip][a.segs[i].block];
      const BlockMap& y = h->blocks[ip][b.segs[i].block];
      same = (x.field == y.field && x.steps == y.steps && x.ds == y.ds && x.bseg == y.bseg &&
              x.charge_field == y.charge_field && x.facz == y.facz);
    }
    const int ia = (int)h->sweeps.size();
    a.storage = (int)h->exec.size();
    h->exec.push_back(ia);
    h->sweeps.push_back(a);
    if (same && !h->no_alias) {
      b.storage = a.storage;
    } else {
      b.storage = (int)h->exec.size();
      h->exec.push_back(ia + 1);
    }
    h->sweeps.push_back(b);
    for (int which = 0; which < 2; ++which) {
      const Sweep& sw = h->sweeps[ia + which];
      for (const Seg& g : sw.segs) {
        BlockMap& bm = h->blocks[ip][g.block];
        if (g.from == HEAD) { bm.sweep_head = ia + which; bm.off_head = g.off; }
        else { bm.sweep_tail = ia + which; bm.off_tail = g.off; }
      }
    }
  }
  // wfac / k-table keys
  for (Sweep& sw : h->sweeps)
    for (Seg& g : sw.segs) {
      const BlockMap& bm = h->blocks[sw.polymer][g.block];
      WfacKey wk{bm.field, bm.ds, bm.charge_field, bm.charge_field >= 0 ? bm.facz : 0.0};
      auto it = std::find(h->wfac_keys.begin(), h->wfac_keys.end(), wk);
      if (it == h->wfac_keys.end()) {
        g.wfac_id = (int)h->wfac_keys.size();
        h->wfac_keys.push_back(wk);
      } else {
        g.wfac_id = (int)(it - h->wfac_keys.begin());
      }
      std::pair<double, double> kk(bm.ds, bm.bseg);
      auto it2 = std::find(h->ktab_keys.begin(), h->ktab_keys.end(), kk);
      if (it2 == h->ktab_keys.end()) {
        g.ktab_id = (int)h->ktab_keys.size();
        h->ktab_keys.push_back(kk);
      } else {
        g.ktab_id = (int)(it2 - h->ktab_keys.begin());
      }
    }
  // Lockstep schedule (engine_state.h): junction-leaving sweeps start one step
  // after the last sweep arriving at their junction ends.
  h->sw_start.assign(h->exec.size(), 0);
  h->kmax = 0;
  for (size_t e = 0; e < h->exec.size(); ++e) {
    const Sweep& sw = h->sweeps[h->exec[e]];
    for (const auto& in : sw.jin) {
      const Sweep& src = h->sweeps[in.first];
      h->sw_start[e] = std::max(h->sw_start[e], h->sw_start[src.storage] + src.total + 1);
    }
    h->kmax = std::max(h->kmax, h->sw_start[e] + sw.total);
  }
  // Field model
  FieldModel& fm = h->fm;
  memset(&fm, 0, sizeof(fm));
  fm.nf = h->nf;
  fm.n_int = c.n_interactions;
  for (int it = 0; it < c.n_interactions; ++it) {
    const ps_interaction_config& I = c.interactions[it];
    if (I.field_a < 0 || I.field_a >= h->nf || I.field_b < 0 || I.field_b >= h->nf ||
        I.field_a == I.field_b) {
      h->err = "interaction scfields out of range";
      return PS_ATTRIB_ERR;
    }
    fm.int_a[it] = I.field_a;
    fm.int_b[it] = I.field_b;
    fm.chin[it] = I.chi * scale_len;
  }
  for (int i = 0; i < h->nf; ++i) fm.dens_avg[i] = dens_avg[i];
  fm.lambda0 = c.updater.lambda0;
  fm.lambda1 = c.updater.lambda1;
  fm.npol = c.n_polymers;
  for (int ip = 0; ip < c.n_polymers; ++ip) {
    // -vf ln Q / alpha; a polydisperse chain carries its weight: -vf (w_k / Gamma) ln Q_k / alpha
    fm.vf[ip] = h->chain_dwt[ip] * h->chain_vf[ip];
    fm.alpha[ip] = h->alpha[ip];
  }
  fm.nsolv = c.n_solvents;
  for (int is = 0; is < c.n_solvents; ++is) fm.solv_vf[is] = c.solvents[is].volfrac;
  fm.scale_len = scale_len;
  fm.N = h->N;

  // Device
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    h->err = "no CUDA device available";
    return PS_GPU_ERR;
  }
  h->dev = c.device;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  if (h->exec.size() > 1) {
    PS_CUDA(h, cudaEventCreateWithFlags(&h->ev_split, cudaEventDisableTiming));
    for (size_t e = 0; e < h->exec.size(); ++e) {
      cudaStream_t s = nullptr;
      cudaEvent_t ev = nullptr;
      PS_CUDA(h, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      h->sw_st.push_back(s);
      PS_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      h->sw_ev.push_back(ev);
    }
  }
  const int pb = (h->prec == PS_PREC_MIXED) ? 4 : 8;
  h->fused_plane = plane_fused_supported(pb, c.n[1], c.n[2]);
  h->xy_ok = xy_supported(pb, c.n[0], c.n[1], c.n[2]);
  h->cluster_ok = !h->fused_plane && cluster_plane_supported(pb, c.n[1], c.n[2]);
  const size_t nfN = (size_t)h->nf * h->N;
  PS_CUDA(h, cudaMalloc((void**)&h->d_w, sizeof(double) * nfN));
  PS_CUDA(h, cudaMalloc((void**)&h->d_phi, sizeof(double) * nfN));
  PS_CUDA(h, cudaMalloc((void**)&h->d_p, sizeof(double) * (size_t)h->N));
  PS_CUDA(h, cudaMemset(h->d_w, 0, sizeof(double) * nfN));
  PS_CUDA(h, cudaMemset(h->d_phi, 0, sizeof(double) * nfN));
  PS_CUDA(h, cudaMemset(h->d_p, 0, sizeof(double) * (size_t)h->N));
  PS_CUDA(h, cudaEventCreateWithFlags(&h->p_ready, cudaEventDisableTiming));
  PS_CUDA(h, cudaEventRecord(h->p_ready, h->st));
  if (h->nq > 0) {
    const size_t qN = (size_t)h->nq * h->N;
    PS_CUDA(h, cudaMalloc((void**)&h->d_rho, sizeof(double) * qN));
    PS_CUDA(h, cudaMalloc((void**)&h->d_psi, sizeof(double) * qN));
    PS_CUDA(h, cudaMemset(h->d_rho, 0, sizeof(double) * qN));
    PS_CUDA(h, cudaMemset(h->d_psi, 0, sizeof(double) * qN));
  }
  if (c.updater.noise != 0.0) {
    PS_CUDA(h, cudaMalloc((void**)&h->d_noise, sizeof(double) * nfN));
    int rn = noise_setup(h);
    if (rn) return rn;
  }
  PS_CUDA(h, cudaMalloc((void**)&h->d_qpart, sizeof(double) * kRedBlocks));
  PS_CUDA(h, cudaMalloc((void**)&h->d_upart, sizeof(double) * kRedBlocks * kUpdQ));
  PS_CUDA(h, cudaMemset(h->d_upart, 0, sizeof(double) * kRedBlocks * kUpdQ));
  PS_CUDA(h, cudaMalloc((void**)&h->d_sc, sizeof(DevScalars)));
  PS_CUDA(h, cudaMemset(h->d_sc, 0, sizeof(DevScalars)));
  PS_CUDA(h, cudaMallocHost((void**)&h->h_sc, sizeof(DevScalars)));
  if (c.updater.kind == PS_UPD_ANDERSON) {
    const int m = c.updater.anderson_depth;
    h->am_slots = m + 1;
    PS_CUDA(h, cudaMalloc((void**)&h->d_hw, sizeof(double) * nfN * h->am_slots));
    PS_CUDA(h, cudaMalloc((void**)&h->d_hd, sizeof(double) * nfN * h->am_slots));
    PS_CUDA(h, cudaMalloc((void**)&h->d_gram, sizeof(double) * h->am_slots * h->am_slots));
    PS_CUDA(h, cudaMemset(h->d_gram, 0, sizeof(double) * h->am_slots * h->am_slots));
    PS_CUDA(h, cudaMalloc((void**)&h->d_gpart, sizeof(double) * kRedBlocks * 33));
  }
  int rc = (h->prec == PS_PREC_MIXED) ? build_device_tables<float>(h) : build_device_tables<double>(h);
  if (rc) return rc;
  h->rng.seed_((uint32_t)(c.seed & 0xffffffffULL));
  // Algorithmic bytes of one propagator step: read q(s), read wfac, write q(s+ds).
  h->sweep_steps = 0;
  for (int s : h->exec) h->sweep_steps += h->sweeps[s].total;
  h->sweep_bytes = 3.0 * (double)h->N * (double)pb * (double)h->sweep_steps;
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int engine_check_scalars(ps_handle* h) {
  PS_CUDA(h, cudaMemcpyAsync(h->h_sc, h->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  int rn = noise_check(h);
  if (rn) return rn;
  // a timed-out bulk copy first: the pass it stopped leaves stale data that
  // may also make Q or F non-finite
  if (h->h_sc->error_flags & 4) {
    h->err = "a bulk shared-memory copy did not complete within the wait limit";
    return PS_GPU_ERR;
  }
  if (h->h_sc->error_flags & 1) {
    h->err = "PsBlock::calcBigQ() found nan/inf?";
    return PS_RUN_ERR;
  }
  if (h->h_sc->error_flags & 2) {
    h->err = "non-finite free energy";
    return PS_RUN_ERR;
  }
  return PS_OK;
}

static int iterate_impl(ps_handle* h, int n) {
  PS_CUDA(h, cudaSetDevice(h->dev));
  for (int it = 0; it < n; ++it) {
    int rc = engine_prepare_noise(h);
    if (rc) return rc;
    const bool sample = h->timing_cap > 0 && h->timing_count < h->timing_cap;
    if (h->eager_iters < 1) {
      long long nl = 0;
      rc = run_iteration(h, &nl);
      if (rc) return rc;
      if (sample) {
        // eager iteration: the capture events hold this iteration's interval
        PS_CUDA(h, cudaEventSynchronize(h->ev_cap_end));
        float ms = 0.f;
        PS_CUDA(h, cudaEventElapsedTime(&ms, h->ev_cap_start, h->ev_cap_end));
        h->eager_ms.push_back(ms);
      }
      h->launches_per_iter = nl;
      h->eager_iters++;
    } else {
      if (!h->gexec) {
        if (h->variant < 0) {
          rc = autotune(h);
          if (rc) return rc;
        }
        long long nl = 0;
        PS_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        rc = run_iteration(h, &nl);
        cudaGraph_t g = nullptr;
        cudaError_t ec = cudaStreamEndCapture(h->st, &g);
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (ec != cudaSuccess) {
          h->err = std::string("graph capture: ") + cudaGetErrorString(ec);
          return PS_GPU_ERR;
        }
        h->graph = g;
        PS_CUDA(h, cudaGraphInstantiate(&h->gexec, h->graph, 0));
        h->launches_per_iter = nl;
        h->graph_has_timing = false;
        if (h->timing_cap > 0) {
          size_t nn = 0;
          PS_CUDA(h, cudaGraphGetNodes(h->graph, nullptr, &nn));
          std::vector<cudaGraphNode_t> nodes(nn);
          PS_CUDA(h, cudaGraphGetNodes(h->graph, nodes.data(), &nn));
          for (auto nd : nodes) {
            cudaGraphNodeType ty;
            PS_CUDA(h, cudaGraphNodeGetType(nd, &ty));
            if (ty != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev;
            PS_CUDA(h, cudaGraphEventRecordNodeGetEvent(nd, &ev));
            if (ev == h->ev_cap_start) h->node_start = nd;
            if (ev == h->ev_cap_end) h->node_end = nd;
          }
          h->graph_has_timing = (h->node_start && h->node_end);
        }
      }
      if (sample && h->graph_has_timing) {
        PS_CUDA(h, cudaGraphExecEventRecordNodeSetEvent(h->gexec, h->node_start, h->ev_start[h->timing_count]));
        PS_CUDA(h, cudaGraphExecEventRecordNodeSetEvent(h->gexec, h->node_end, h->ev_end[h->timing_count]));
        h->timing_count++;
      }
      PS_CUDA(h, cudaGraphLaunch(h->gexec, h->st));
    }
    // updaterSequence order: these run after the field updater of the same step
    for (int code : h->post_order) {
      int rc = (code == POST_FILTER) ? filter_after_iteration(h, h->iterations)
                                     : poisson_after_iteration(h, h->iterations);
      if (rc) return rc;
    }
    h->iterations++;
  }
  return engine_check_scalars(h);
}

int engine_create(ps_handle* h, const ps_config* cfg) { return create_impl(h, cfg); }

void post_order_set(ps_handle* h, int code, bool on) {
  std::vector<int> o;
  for (int c : h->post_order)
    if (c != code) o.push_back(c);
  if (on) o.push_back(code);
  h->post_order = o;
}

void engine_free(ps_handle* h) { free_all(h); }

}  // namespace psb

using namespace psb;

extern "C" {

const char* ps_version(void) { return "pswift-b200 0.1 (sm_100a)"; }

const char* ps_gpu_last_error(const ps_handle* h) {
  if (!h) return g_thread_err.c_str();
  return h->err.c_str();
}

int ps_gpu_create(const ps_config* cfg, ps_handle** out) {
  if (!cfg || !out) {
    g_thread_err = "null argument";
    return PS_ATTRIB_ERR;
  }
  *out = nullptr;
  ps_handle* h = new ps_handle();
  int rc = create_impl(h, cfg);
  if (rc != PS_OK) {
    g_thread_err = h->err;
    free_all(h);
    delete h;
    // a failed allocation leaves a (non-sticky) error in the runtime's
    // last-error slot; clear it so the next launch check does not report it
    cudaGetLastError();
    return rc;
  }
  *out = h;
  return PS_OK;
}

int ps_gpu_destroy(ps_handle* h) {
  if (!h) return PS_OK;
  cudaSetDevice(h->dev);
  if (h->st) cudaStreamSynchronize(h->st);
  free_all(h);
  delete h;
  return PS_OK;
}

// The caller's (polymer, block) -> (chain, block of the chain).  A polyDisperseBCP
// numbers its quadrature blocks seed-major, as the reference's block list does
// (pspolymer/PsPolyDisperseBCP.cpp:155-208): block b is seed b / n_g of chain b % n_g.
static bool user_block(const ps_handle* h, int up, int ub, int* ch, int* b) {
  if (up < 0 || up >= (int)h->user_first.size() || ub < 0) return false;
  const int ng = h->user_ng[up];
  const int nseed = h->ucfg.polymers[up].n_blocks;
  if (ub >= nseed * ng) return false;
  if (h->ucfg.polydisperse[up].enabled) {
    *ch = h->user_first[up] + ub % ng;
    *b = ub / ng;
  } else {
    *ch = h->user_first[up];
    *b = ub;
  }
  return *ch < (int)h->blocks.size() && *b < (int)h->blocks[*ch].size();
}

int ps_gpu_block_steps(const ps_handle* h, int ip, int ib, int* steps) {
  int ch = 0, b = 0;
  if (!h || !steps || !user_block(h, ip, ib, &ch, &b)) return PS_ATTRIB_ERR;
  *steps = h->blocks[ch][b].steps;
  return PS_OK;
}

static double* field_ptr(ps_handle* h, int which, int index) {
  if (which == PS_FIELD_PRES) return h->d_p;
  if (which == PS_FIELD_CHARGE || which == PS_FIELD_POTENTIAL) {
    if (index < 0 || index >= h->nq) return nullptr;
    return (which == PS_FIELD_CHARGE ? h->d_rho : h->d_psi) + (size_t)index * h->N;
  }
  if (index < 0 || index >= h->nf) return nullptr;
  if (which == PS_FIELD_W) return h->d_w + (size_t)index * h->N;
  if (which == PS_FIELD_PHI) return h->d_phi + (size_t)index * h->N;
  return nullptr;
}

// Work on st that touches p goes after an asynchronous upload of it.
static int order_uploads(ps_handle* h) {
  if (h->up_st) PS_CUDA(h, cudaStreamWaitEvent(h->st, h->p_ready, 0));
  return PS_OK;
}

int ps_gpu_set_fields(ps_handle* h, int which, int index, const double* data, int on_device) {
  if (!h || !data) return PS_ATTRIB_ERR;
  double* dst = field_ptr(h, which, index);
  if (!dst) {
    h->err = "bad field selector";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  int rc = order_uploads(h);
  if (rc) return rc;
  PS_CUDA(h, cudaMemcpyAsync(dst, data, sizeof(double) * (size_t)h->N,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int ps_gpu_set_fields_async(ps_handle* h, int which, int index, const double* host) {
  if (!h || !host) return PS_ATTRIB_ERR;
  double* dst = field_ptr(h, which, index);
  if (!dst) {
    h->err = "bad field selector";
    return PS_ATTRIB_ERR;
  }
  if (h->in_batch) {  // the batch owns the launches: a blocking copy
    cudaPointerAttributes pa;
    const bool dev = cudaPointerGetAttributes(&pa, host) == cudaSuccess && pa.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    return ps_gpu_set_fields(h, which, index, host, dev ? 1 : 0);
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  const size_t bytes = sizeof(double) * (size_t)h->N;
  if (which != PS_FIELD_PRES) {
    PS_CUDA(h, cudaMemcpyAsync(dst, host, bytes, cudaMemcpyDefault, h->st));
    return PS_OK;
  }
  if (!h->up_st) {
    PS_CUDA(h, cudaStreamCreateWithFlags(&h->up_st, cudaStreamNonBlocking));
    PS_CUDA(h, cudaEventCreateWithFlags(&h->up_ev, cudaEventDisableTiming));
  }
  // after the work enqueued so far (the last update, read-back snapshots of p),
  // before the next update, overlapping the next iteration's sweeps
  PS_CUDA(h, cudaEventRecord(h->up_ev, h->st));
  PS_CUDA(h, cudaStreamWaitEvent(h->up_st, h->up_ev, 0));
  PS_CUDA(h, cudaMemcpyAsync(dst, host, bytes, cudaMemcpyDefault, h->up_st));
  PS_CUDA(h, cudaEventRecord(h->p_ready, h->up_st));
  return PS_OK;
}

int ps_gpu_get_fields(ps_handle* h, int which, int index, double* data, int on_device) {
  if (!h || !data) return PS_ATTRIB_ERR;
  double* src = field_ptr(h, which, index);
  if (!src) {
    h->err = "bad field selector";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  int rc = order_uploads(h);
  if (rc) return rc;
  PS_CUDA(h, cudaMemcpyAsync(data, src, sizeof(double) * (size_t)h->N,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int ps_gpu_get_fields_async(ps_handle* h, int which, int index, double* host) {
  if (!h || !host) return PS_ATTRIB_ERR;
  double* src = field_ptr(h, which, index);
  if (!src) {
    h->err = "bad field selector";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  int rc = order_uploads(h);
  if (rc) return rc;
  if (!h->io_st) PS_CUDA(h, cudaStreamCreateWithFlags(&h->io_st, cudaStreamNonBlocking));
  ps_handle::ReadSlot& rs = h->read_slots[std::make_pair(which, index)];
  const size_t bytes = sizeof(double) * (size_t)h->N;
  if (!rs.d) {
    PS_CUDA(h, cudaMalloc((void**)&rs.d, bytes));
    PS_CUDA(h, cudaEventCreateWithFlags(&rs.snap, cudaEventDisableTiming));
    PS_CUDA(h, cudaEventCreateWithFlags(&rs.done, cudaEventDisableTiming));
    PS_CUDA(h, cudaEventRecord(rs.done, h->io_st));
  }
  // the previous host copy out of this snapshot has finished before it is overwritten
  PS_CUDA(h, cudaStreamWaitEvent(h->st, rs.done, 0));
  PS_CUDA(h, cudaMemcpyAsync(rs.d, src, bytes, cudaMemcpyDeviceToDevice, h->st));
  PS_CUDA(h, cudaEventRecord(rs.snap, h->st));
  PS_CUDA(h, cudaStreamWaitEvent(h->io_st, rs.snap, 0));
  PS_CUDA(h, cudaMemcpyAsync(host, rs.d, bytes, cudaMemcpyDeviceToHost, h->io_st));
  PS_CUDA(h, cudaEventRecord(rs.done, h->io_st));
  return PS_OK;
}

int ps_gpu_fields_wait(ps_handle* h) {
  if (!h) return PS_ATTRIB_ERR;
  if (!h->io_st && !h->up_st) return PS_OK;
  PS_CUDA(h, cudaSetDevice(h->dev));
  if (h->io_st) PS_CUDA(h, cudaStreamSynchronize(h->io_st));
  if (h->up_st) PS_CUDA(h, cudaStreamSynchronize(h->up_st));
  return PS_OK;
}

int ps_gpu_init_random(ps_handle* h) {
  if (!h) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  if (h->up_st) PS_CUDA(h, cudaStreamSynchronize(h->up_st));
  int rc = settle_rng(h);
  if (rc) return rc;
  std::vector<double> buf((size_t)h->N);
  for (int i = 0; i < h->nf; ++i) {
    for (long long r = 0; r < h->N; ++r) {
      const double u = h->rng.real();
      buf[(size_t)r] = 1.0 * (u + (-0.5));
    }
    PS_CUDA(h, cudaMemcpy(h->d_w + (size_t)i * h->N, buf.data(), sizeof(double) * (size_t)h->N,
                          cudaMemcpyHostToDevice));
  }
  PS_CUDA(h, cudaMemset(h->d_p, 0, sizeof(double) * (size_t)h->N));
  return PS_OK;
}

int ps_gpu_iterate(ps_handle* h, int n_iter) {
  if (!h) return PS_ATTRIB_ERR;
  if (n_iter < 0) {
    h->err = "n_iter must be >= 0";
    return PS_ATTRIB_ERR;
  }
  return iterate_impl(h, n_iter);
}

int ps_gpu_get_scalars(ps_handle* h, ps_scalars* out) {
  if (!h || !out) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaMemcpyAsync(h->h_sc, h->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  const DevScalars& s = *h->h_sc;
  memset(out, 0, sizeof(*out));
  out->free_energy = s.free_energy;
  out->free_energy_nodis = s.free_energy_nodis;
  for (int up = 0; up < h->ucfg.n_polymers && up < (int)h->user_first.size(); ++up) {
    const int c0 = h->user_first[up];
    if (h->user_ng[up] == 1 && !h->ucfg.polydisperse[up].enabled) {
      out->q[up] = s.q[c0];
      out->log_q[up] = s.log_q[c0];
      continue;
    }
    // PsPolyDisperseBCP::getLogBigQ (pspolymer/PsPolyDisperseBCP.cpp:282-305)
    double sum = 0.0;
    for (int k = 0; k < h->user_ng[up]; ++k) sum = sum + (log(s.q[c0 + k]) * h->chain_dwt[c0 + k]);
    out->log_q[up] = sum;
    out->q[up] = exp(sum);
  }
  out->max_incomp = s.max_incomp;
  out->dh_norm = s.dh_norm;
  out->pressure_mean = s.pressure_mean;
  out->iteration = s.iteration;
  out->error_flags = s.error_flags;
  return PS_OK;
}

int ps_gpu_get_propagator(ps_handle* h, int uip, int uib, int end, int n, double* out) {
  int ip = 0, ib = 0;
  if (!h || !out || !user_block(h, uip, uib, &ip, &ib)) return PS_ATTRIB_ERR;
  const BlockMap& b = h->blocks[ip][ib];
  if (n < 0 || n > b.steps) {
    h->err = "slice index out of range";
    return PS_ATTRIB_ERR;
  }
  const int sweep = (end == PS_FROM_HEAD) ? b.sweep_head : b.sweep_tail;
  const int off = (end == PS_FROM_HEAD) ? b.off_head : b.off_tail;
  const int storage = h->sweeps[sweep].storage;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  const size_t N = (size_t)h->N;
  if (h->prec == PS_PREC_MIXED) {
    std::vector<float> tmp(N);
    PS_CUDA(h, cudaMemcpy(tmp.data(), h->bf.slices[storage] + (size_t)(off + n) * N,
                          sizeof(float) * N, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < N; ++i) out[i] = tmp[i];
  } else {
    PS_CUDA(h, cudaMemcpy(out, h->bd.slices[storage] + (size_t)(off + n) * N, sizeof(double) * N,
                          cudaMemcpyDeviceToHost));
  }
  return PS_OK;
}

int ps_gpu_synchronize(ps_handle* h) {
  if (!h) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (h->up_st) PS_CUDA(h, cudaStreamSynchronize(h->up_st));
  return PS_OK;
}

// Kernel launches one iteration issues (all of them this library's kernels).
long long ps_gpu_launches_per_iteration(const ps_handle* h) { return h ? h->launches_per_iter : 0; }

void* ps_gpu_stream(const ps_handle* h) { return h ? (void*)h->st : nullptr; }

int ps_gpu_set_variant(ps_handle* h, int variant) {
  if (!h || variant < -1 || variant >= VARIANT_COUNT) return PS_ATTRIB_ERR;
  if (variant >= 0 && (variant & VARIANT_XY) && !h->xy_ok) {
    h->err = "the row + x-y plane design does not exist for this grid";
    return PS_ATTRIB_ERR;
  }
  if (variant >= 0 && (variant & VARIANT_CLUSTER) && !h->cluster_ok) {
    h->err = "the cluster plane pass exists for 256 x 256 y-z planes only";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  h->node_start = h->node_end = nullptr;
  h->graph_has_timing = false;
  h->variant = variant;
  return PS_OK;
}

int ps_gpu_set_precision(ps_handle* h, int precision) {
  if (!h) return PS_ATTRIB_ERR;
  if (precision != PS_PREC_FP64 && precision != PS_PREC_MIXED) {
    h->err = "precision must be PS_PREC_FP64 or PS_PREC_MIXED";
    return PS_ATTRIB_ERR;
  }
  if (precision == h->prec) return PS_OK;
  if (h->in_batch) {
    h->err = "the precision of a batch instance is fixed by its batch";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  h->node_start = h->node_end = nullptr;
  h->graph_has_timing = false;
  const int old = h->prec;
  const bool built = (precision == PS_PREC_MIXED) ? !h->bf.slices.empty() : !h->bd.slices.empty();
  h->prec = precision;
  if (!built) {
    int rc = (precision == PS_PREC_MIXED) ? build_device_tables<float>(h) : build_device_tables<double>(h);
    if (rc == PS_OK && cudaStreamSynchronize(h->st) != cudaSuccess) rc = PS_GPU_ERR;
    if (rc != PS_OK) {
      if (precision == PS_PREC_MIXED) free_buffers(h->bf);
      else free_buffers(h->bd);
      h->prec = old;
      return rc;
    }
  }
  const int pb = (precision == PS_PREC_MIXED) ? 4 : 8;
  h->fused_plane = plane_fused_supported(pb, h->n[1], h->n[2]);
  h->xy_ok = xy_supported(pb, h->n[0], h->n[1], h->n[2]);
  h->cluster_ok = !h->fused_plane && cluster_plane_supported(pb, h->n[1], h->n[2]);
  h->sweep_bytes = 3.0 * (double)h->N * (double)pb * (double)h->sweep_steps;
  h->variant = -1;
  h->eager_iters = 0;
  return PS_OK;
}

int ps_gpu_get_variant(const ps_handle* h, int* variant, float* tune_ms, int n_tune) {
  if (!h || !variant) return PS_ATTRIB_ERR;
  *variant = h->variant;
  for (int i = 0; tune_ms && i < n_tune && i < VARIANT_COUNT; ++i) tune_ms[i] = h->tune_ms[i];
  return PS_OK;
}

int ps_gpu_enable_sweep_timing(ps_handle* h, int max_samples) {
  if (!h || max_samples < 0) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  h->node_start = h->node_end = nullptr;
  h->graph_has_timing = false;
  if (!h->ev_cap_start) PS_CUDA(h, cudaEventCreate(&h->ev_cap_start));
  if (!h->ev_cap_end) PS_CUDA(h, cudaEventCreate(&h->ev_cap_end));
  while ((int)h->ev_start.size() < max_samples) {
    cudaEvent_t a, b;
    PS_CUDA(h, cudaEventCreate(&a));
    PS_CUDA(h, cudaEventCreate(&b));
    h->ev_start.push_back(a);
    h->ev_end.push_back(b);
  }
  h->timing_cap = max_samples;
  h->timing_count = 0;
  h->eager_ms.clear();
  return PS_OK;
}

int ps_gpu_sweep_timing(ps_handle* h, double* ms_out, int max_out, int* n_out,
                        double* bytes_per_iter, long long* steps_per_iter) {
  if (!h || !n_out) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  int n = 0;
  for (float ms : h->eager_ms) {
    if (ms_out && n < max_out) ms_out[n] = ms;
    ++n;
  }
  for (int i = 0; i < h->timing_count; ++i) {
    float ms = 0.f;
    PS_CUDA(h, cudaEventElapsedTime(&ms, h->ev_start[i], h->ev_end[i]));
    if (ms_out && n < max_out) ms_out[n] = ms;
    ++n;
  }
  *n_out = n;
  if (bytes_per_iter) *bytes_per_iter = h->sweep_bytes;
  if (steps_per_iter) *steps_per_iter = h->sweep_steps;
  h->timing_count = 0;
  h->eager_ms.clear();
  return PS_OK;
}

}  // extern "C"
