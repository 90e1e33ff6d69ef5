// poissonUpdater on the device (pseffhamil/PsPoissonUpdater.cpp:140-262;
// schedule psbase/PsUpdater.cpp:60-206).
//
// For each listed chargeDens field c, at the scheduled steps:
//   rho_c += -sum(rho_c) / N                                  (in place)
//   res = IFFT(K FFT(rho_c)),  K = 4 (3.1415) lB / |k|^2, 0 at |k|^2 < 1e-9
//   psi_c = res / N, except where |res / N - psi_c| > 0.2 |psi_c|: 1.2 psi_c / N
// K is even in k, so the r2c half spectrum carries it; the k-table is built on
// the host with the reference's k-vector arithmetic (psbase/PsGridField.cpp:66-104).
// FP64 on the handle's stream, after the iteration's graph.
#include <math.h>
#include <string.h>

#include <vector>

#include "engine_state.h"
#include "spectral.cuh"

namespace psb {

struct PoissonState {
  ps_poisson_config cfg;
  bool fused = true;
  double2* spec = nullptr;
  double* kc = nullptr;   // half-spectrum Coulomb factors [nx][ny][nzh]
  double* res = nullptr;  // N: unnormalised inverse transform
  double2 *tw_x = nullptr, *tw_y = nullptr, *tw_z = nullptr, *tw_zh = nullptr;
  PlaneWork<double>* d_pw = nullptr;  // 2 per field: FIRST (src = rho), LAST (store = res)
  PencilWork<double>* d_xw = nullptr;
  double* part = nullptr;
  double* scal = nullptr;  // [0] -mean(rho)
};

__global__ void coulomb_multiply(double2* __restrict__ spec, const double* __restrict__ kc, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = spec[i];
    const double f = kc[i];
    spec[i] = make_double2(v.x * f, v.y * f);
  }
}

// psi = res * scale, with the reference's clamp on a relative change above 0.2
// (psi = 0 gives inf or nan there, as on the host: inf clamps, nan does not).
__global__ void potential_update(double* __restrict__ psi, const double* __restrict__ res, long long N,
                                 double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const double psi0 = psi[i];
    double r = res[i];
    const double psi1 = r * scale;
    const double frac = fabs((psi1 - psi0) / psi0);
    if (frac > 0.2) r = psi0 * 1.2;
    psi[i] = r * (1.0 * scale);
  }
}

void poisson_free(ps_handle* h) {
  PoissonState* p = static_cast<PoissonState*>(h->poisson);
  if (!p) return;
  auto fr = [](void* q) { if (q) cudaFree(q); };
  fr(p->spec); fr(p->kc); fr(p->res); fr(p->tw_x); fr(p->tw_y); fr(p->tw_z); fr(p->tw_zh);
  fr(p->d_pw); fr(p->d_xw); fr(p->part); fr(p->scal);
  delete p;
  h->poisson = nullptr;
}

// |k|^2 at grid index (i, j, k): PsGridField::calck2 (psbase/PsGridField.cpp:66-104).
static double calck2(const ps_handle* h, int i, int j, int k) {
  const double twopi = 2.0 * acos(-1.0);
  const int idx[3] = {i, j, k};
  double kv[3];
  for (int d = 0; d < 3; ++d) {
    const double n2 = (double)h->n[d] / 2.0;
    const double nk = n2 - fabs((double)idx[d] - n2);
    kv[d] = twopi * nk / (double)h->n[d];
    kv[d] = kv[d] / h->cfg.cell[d];
  }
  return kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
}

static int poisson_build(ps_handle* h, const ps_poisson_config* c) {
  PoissonState* p = new PoissonState();
  h->poisson = p;
  p->cfg = *c;
  const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
  const size_t nspec = (size_t)nx * ny * h->nzh;
  p->fused = plane_fused_supported(8, ny, nz);
  PS_CUDA(h, cudaMalloc((void**)&p->spec, sizeof(double2) * nspec));
  PS_CUDA(h, cudaMalloc((void**)&p->res, sizeof(double) * (size_t)h->N));
  // PsPoissonUpdater::build_k2 (pseffhamil/PsPoissonUpdater.cpp:140-175)
  std::vector<double> kc(nspec);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int kz = 0; kz < h->nzh; ++kz) {
        const double k2 = calck2(h, i, j, kz);
        kc[((size_t)i * ny + j) * h->nzh + kz] =
            (k2 < 0.000000001) ? 0.0 : (4.0 * 3.1415 * c->bjerrum_len) / k2;
      }
  PS_CUDA(h, cudaMalloc((void**)&p->kc, sizeof(double) * nspec));
  PS_CUDA(h, cudaMemcpy(p->kc, kc.data(), sizeof(double) * nspec, cudaMemcpyHostToDevice));
  PS_CUDA(h, twiddles64(&p->tw_x, nx));
  PS_CUDA(h, twiddles64(&p->tw_y, ny));
  PS_CUDA(h, twiddles64(&p->tw_z, nz));
  PS_CUDA(h, twiddles64(&p->tw_zh, nz / 2 > 0 ? nz / 2 : 1));
  std::vector<PlaneWork<double>> pw(2 * (size_t)c->n_fields);
  memset(pw.data(), 0, sizeof(PlaneWork<double>) * pw.size());
  for (int i = 0; i < c->n_fields; ++i) {
    pw[2 * i].mode = MODE_FIRST;
    pw[2 * i].src = h->d_rho + (size_t)c->fields[i] * h->N;
    pw[2 * i].spec = p->spec;
    pw[2 * i + 1].mode = MODE_LAST;
    pw[2 * i + 1].spec = p->spec;
    pw[2 * i + 1].store = p->res;
  }
  PencilWork<double> xw;
  memset(&xw, 0, sizeof(xw));
  xw.spec = p->spec;
  PS_CUDA(h, cudaMalloc((void**)&p->d_pw, sizeof(PlaneWork<double>) * pw.size()));
  PS_CUDA(h, cudaMemcpy(p->d_pw, pw.data(), sizeof(PlaneWork<double>) * pw.size(), cudaMemcpyHostToDevice));
  PS_CUDA(h, cudaMalloc((void**)&p->d_xw, sizeof(xw)));
  PS_CUDA(h, cudaMemcpy(p->d_xw, &xw, sizeof(xw), cudaMemcpyHostToDevice));
  PS_CUDA(h, cudaMalloc((void**)&p->part, sizeof(double) * kRedBlocks));
  PS_CUDA(h, cudaMalloc((void**)&p->scal, sizeof(double) * 2));
  return PS_OK;
}

static int poisson_apply(ps_handle* h) {
  PoissonState* p = static_cast<PoissonState*>(h->poisson);
  const ps_poisson_config& c = p->cfg;
  const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
  const long long N = h->N;
  const long long nspec = (long long)nx * ny * h->nzh;
  cudaStream_t st = h->st;
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  for (int i = 0; i < c.n_fields; ++i) {
    double* rho = h->d_rho + (size_t)c.fields[i] * N;
    double* psi = h->d_psi + (size_t)c.fields[i] * N;
    filter_sum_partials<<<kRedBlocks, kFT, 0, st>>>(rho, N, p->part, 0, nullptr);
    filter_finalize<<<1, kFT, 0, st>>>(p->part, kRedBlocks, 0, (double)N, p->scal);
    filter_shift<<<blocks, 256, 0, st>>>(rho, N, p->scal);
    PS_CUDA(h, cudaGetLastError());
    if (p->fused) {
      PS_CUDA(h, launch_plane<double>(p->d_pw + 2 * i, 1, nx, ny, nz, p->tw_y, p->tw_zh, p->tw_z, 0, st));
    } else {
      PS_CUDA(h, launch_rows<double>(p->d_pw + 2 * i, 1, nx * ny, nz, p->tw_zh, p->tw_z, st));
      if (ny > 1) PS_CUDA(h, launch_pencil<double>(p->d_xw, 1, PENCIL_FWD, ny, nx, h->nzh, p->tw_y, nx, ny, nz, 0, st));
    }
    PS_CUDA(h, launch_pencil<double>(p->d_xw, 1, PENCIL_FWD, nx, 1, ny * h->nzh, p->tw_x, nx, ny, nz, 0, st));
    coulomb_multiply<<<blocks, 256, 0, st>>>(p->spec, p->kc, nspec);
    PS_CUDA(h, cudaGetLastError());
    PS_CUDA(h, launch_pencil<double>(p->d_xw, 1, PENCIL_INV, nx, 1, ny * h->nzh, p->tw_x, nx, ny, nz, 0, st));
    if (p->fused) {
      PS_CUDA(h, launch_plane<double>(p->d_pw + 2 * i + 1, 1, nx, ny, nz, p->tw_y, p->tw_zh, p->tw_z, 0, st));
    } else {
      if (ny > 1) PS_CUDA(h, launch_pencil<double>(p->d_xw, 1, PENCIL_INV, ny, nx, h->nzh, p->tw_y, nx, ny, nz, 0, st));
      PS_CUDA(h, launch_rows<double>(p->d_pw + 2 * i + 1, 1, nx * ny, nz, p->tw_zh, p->tw_z, st));
    }
    potential_update<<<blocks, 256, 0, st>>>(psi, p->res, N, 1.0 / ((double)N));
    PS_CUDA(h, cudaGetLastError());
  }
  return PS_OK;
}

int poisson_after_iteration(ps_handle* h, long long step) {
  PoissonState* p = static_cast<PoissonState*>(h->poisson);
  if (!p) return PS_OK;
  const ps_poisson_config& c = p->cfg;
  if (step < c.apply_start || (c.apply_end >= 0 && step > c.apply_end)) return PS_OK;
  if ((step - c.apply_start) % c.apply_frequency != 0) return PS_OK;
  return poisson_apply(h);
}

}  // namespace psb

using namespace psb;

extern "C" {

int ps_gpu_set_poisson(ps_handle* h, const ps_poisson_config* c) {
  if (!h) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  poisson_free(h);
  post_order_set(h, POST_POISSON, false);
  if (!c) return PS_OK;
  if (c->n_fields < 1 || c->n_fields > h->nq) {
    h->err = "poissonUpdater: updatefields must name chargeDens PhysFields";
    return PS_ATTRIB_ERR;
  }
  for (int i = 0; i < c->n_fields; ++i)
    if (c->fields[i] < 0 || c->fields[i] >= h->nq) {
      h->err = "poissonUpdater: field index out of range";
      return PS_ATTRIB_ERR;
    }
  if (c->apply_frequency < 1) {
    h->err = "poissonUpdater: apply_frequency must be >= 1";
    return PS_ATTRIB_ERR;
  }
  if (c->apply_end >= 0 && c->apply_start >= c->apply_end) {
    h->err = "PsUpdater::setAttrib: applyStart >= applyEnd";
    return PS_ATTRIB_ERR;
  }
  if (c->apply_end >= 0 && (c->apply_end - c->apply_start) <= c->apply_frequency) {
    h->err = "PsUpdater::setAttrib: applyFrequency too large";
    return PS_ATTRIB_ERR;
  }
  int rc = poisson_build(h, c);
  if (rc) {
    poisson_free(h);
    return rc;
  }
  post_order_set(h, POST_POISSON, true);
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int ps_gpu_apply_poisson(ps_handle* h) {
  if (!h) return PS_ATTRIB_ERR;
  if (!h->poisson) {
    h->err = "no Poisson updater set";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  int rc = poisson_apply(h);
  if (rc) return rc;
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

}  // extern "C"
