// simpleSpecFilter updater on the device (pseffhamil/PsSimpleSpecFilter.cpp:75-140,
// pseffhamil/PsSpecFilterUpdater.cpp:155-250, schedule psbase/PsUpdater.cpp:60-206).
//
// For each listed conjugate field w, at the scheduled steps:
//   w += -mean(w);                                  (subtractAverage)
//   P = |FFT(w)|^2, cutoff = cutoffFactor * max(P);   (forwardFFTAbs, findMaxVal)
//   mask = filterStrength where P < cutoff, else 1;
//   w = Re(IFFT(mask * FFT(w))) / N.                 (scaledFFTPair, scaleFFT)
// The power spectrum of a real field is even in k, so the mask is too and the
// half spectrum of an r2c transform carries all of it.  Runs in FP64 on the
// FP64 fields whatever the sweep precision, on the handle's stream, after the
// iteration's graph.
//
// multiSpecFilter (pseffhamil/PsMultiSpecFilter.cpp:130-262) takes the max per
// region of spectrum indices.  Its region map is not even in k, so the mask M
// is not either; Re(IFFT(M W)) of a real field equals IFFT(W (M(k) + M(-k))/2),
// and the half spectrum carries that symmetrised mask: each element looks up
// the regions of both k and -k.
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "engine_state.h"
#include "spectral.cuh"

namespace psb {

struct FilterState {
  ps_filter_config cfg;
  bool fused = true;
  double2* spec = nullptr;
  double2 *tw_x = nullptr, *tw_y = nullptr, *tw_z = nullptr, *tw_zh = nullptr;
  PlaneWork<double>* d_pw = nullptr;  // 2 per field: FIRST (src = w), LAST (store = w)
  PencilWork<double>* d_xw = nullptr;
  double* part = nullptr;  // kRedBlocks partials
  double* scal = nullptr;  // [0] -mean, [1] max power
  // multiSpecFilter
  bool multi = false;
  long long ncells = 0;
  double* cut = nullptr;   // max power per region
};

// Region geometry of multiSpecFilter: cell sizes and cells per axis.
struct Regions {
  int nx, ny, nz, nzh;
  int sx, sy, sz;
  long long cx, cy;
};

// Region of linear spectrum index n, read in (y, x, z) order as the serial
// reference numbers its map (pseffhamil/PsMultiSpecFilter.cpp:185-205).
__device__ __forceinline__ long long region_of(const Regions& g, long long n) {
  const long long jj = n / ((long long)g.nx * g.nz);
  const long long ii = (n / g.nz) % g.nx;
  const long long kk = n % g.nz;
  return (kk / g.sz) * (g.cx * g.cy) + (jj / g.sy) * g.cx + ii / g.sx;
}

// Spectrum indices (x, y, z order) of half-spectrum element e and of its mirror -k.
__device__ __forceinline__ void pair_indices(const Regions& g, long long e, long long& n1, long long& n2) {
  const long long i = e / ((long long)g.ny * g.nzh);
  const long long j = (e / g.nzh) % g.ny;
  const long long kz = e % g.nzh;
  n1 = (i * g.ny + j) * g.nz + kz;
  n2 = (((g.nx - i) % g.nx) * g.ny + (g.ny - j) % g.ny) * g.nz + (g.nz - kz) % g.nz;
}

constexpr int kShCells = 4096;

// Max power per region.  Powers are >= +0, so their bit patterns order like
// the values and an integer atomicMax is a max on doubles.  With few regions
// each block reduces into shared memory first.
template <bool SH>
__global__ void filter_region_max(const double2* __restrict__ spec, long long nspec, Regions g,
                                  unsigned long long* __restrict__ cut, long long ncells) {
  __shared__ unsigned long long sh[SH ? kShCells : 1];
  if (SH) {
    for (long long r = threadIdx.x; r < ncells; r += blockDim.x) sh[r] = 0ull;
    __syncthreads();
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nspec;
       e += (long long)gridDim.x * blockDim.x) {
    const double2 v = spec[e];
    const unsigned long long p = (unsigned long long)__double_as_longlong(v.x * v.x + v.y * v.y);
    long long n1, n2;
    pair_indices(g, e, n1, n2);
    const long long r1 = region_of(g, n1), r2 = region_of(g, n2);
    if (SH) {
      atomicMax(&sh[r1], p);
      if (r2 != r1) atomicMax(&sh[r2], p);
    } else {
      atomicMax(&cut[r1], p);
      if (r2 != r1) atomicMax(&cut[r2], p);
    }
  }
  if (SH) {
    __syncthreads();
    for (long long r = threadIdx.x; r < ncells; r += blockDim.x)
      if (sh[r]) atomicMax(&cut[r], sh[r]);
  }
}

__global__ void filter_mask_multi(double2* __restrict__ spec, long long nspec, Regions g,
                                  const double* __restrict__ cut, double cutoff_factor, double strength,
                                  double inv_n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nspec;
       e += (long long)gridDim.x * blockDim.x) {
    const double2 v = spec[e];
    const double p = v.x * v.x + v.y * v.y;
    long long n1, n2;
    pair_indices(g, e, n1, n2);
    const double m1 = (p < cutoff_factor * cut[region_of(g, n1)]) ? strength : 1.0;
    const double m2 = (p < cutoff_factor * cut[region_of(g, n2)]) ? strength : 1.0;
    const double m = 0.5 * (m1 + m2) * inv_n;
    spec[e] = make_double2(v.x * m, v.y * m);
  }
}

static Regions regions_of(const ps_handle* h, const ps_filter_config& c) {
  Regions g;
  g.nx = h->n[0]; g.ny = h->n[1]; g.nz = h->n[2]; g.nzh = (int)h->nzh;
  g.sx = c.spec_cells[0]; g.sy = c.spec_cells[1]; g.sz = c.spec_cells[2];
  g.cx = g.nx / g.sx; g.cy = g.ny / g.sy;
  return g;
}

__global__ void filter_sum_partials(const double* __restrict__ w, long long N, double* __restrict__ part,
                                    int is_max, const double2* __restrict__ spec) {
  __shared__ double sh[kFT];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)kFT + threadIdx.x; i < N; i += (long long)gridDim.x * kFT) {
    if (is_max) {
      const double2 v = spec[i];
      acc = fmax(acc, v.x * v.x + v.y * v.y);
    } else {
      acc += w[i];
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = kFT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = is_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + o])
                                                  : sh[threadIdx.x] + sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void filter_finalize(const double* __restrict__ part, int np, int is_max, double N,
                                double* __restrict__ out) {
  __shared__ double sh[kFT];
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += kFT) acc = is_max ? fmax(acc, part[i]) : acc + part[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = kFT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = is_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + o])
                                                  : sh[threadIdx.x] + sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = is_max ? sh[0] : -1.0 * (sh[0] / (1.0 * N));
}

__global__ void filter_shift(double* __restrict__ w, long long N, const double* __restrict__ wtot) {
  const double s = *wtot;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    w[i] = w[i] + s;
}

__global__ void filter_mask(double2* __restrict__ spec, long long n, const double* __restrict__ maxp,
                            double cutoff_factor, double strength, double inv_n) {
  const double cut = cutoff_factor * (*maxp);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = spec[i];
    const double p = v.x * v.x + v.y * v.y;
    const double m = ((p < cut) ? strength : 1.0) * inv_n;
    spec[i] = make_double2(v.x * m, v.y * m);
  }
}

cudaError_t twiddles64(double2** dst, int L) {
  std::vector<double2> tw(L > 0 ? L : 1);
  const double twopi = 2.0 * acos(-1.0);
  for (int m = 0; m < L; ++m) tw[m] = make_double2(cos(twopi * m / L), -sin(twopi * m / L));
  cudaError_t e = cudaMalloc((void**)dst, sizeof(double2) * tw.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice);
}

void filter_free(ps_handle* h) {
  FilterState* f = static_cast<FilterState*>(h->filter);
  if (!f) return;
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(f->spec); fr(f->tw_x); fr(f->tw_y); fr(f->tw_z); fr(f->tw_zh);
  fr(f->d_pw); fr(f->d_xw); fr(f->part); fr(f->scal); fr(f->cut);
  delete f;
  h->filter = nullptr;
}

static int filter_build(ps_handle* h, const ps_filter_config* c) {
  FilterState* f = new FilterState();
  h->filter = f;
  f->cfg = *c;
  const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
  f->fused = plane_fused_supported(8, ny, nz);
  PS_CUDA(h, cudaMalloc((void**)&f->spec, sizeof(double2) * (size_t)nx * ny * h->nzh));
  PS_CUDA(h, twiddles64(&f->tw_x, nx));
  PS_CUDA(h, twiddles64(&f->tw_y, ny));
  PS_CUDA(h, twiddles64(&f->tw_z, nz));
  PS_CUDA(h, twiddles64(&f->tw_zh, nz / 2 > 0 ? nz / 2 : 1));
  std::vector<PlaneWork<double>> pw(2 * (size_t)c->n_fields);
  memset(pw.data(), 0, sizeof(PlaneWork<double>) * pw.size());
  for (int i = 0; i < c->n_fields; ++i) {
    double* w = h->d_w + (size_t)c->fields[i] * h->N;
    pw[2 * i].mode = MODE_FIRST;
    pw[2 * i].src = w;
    pw[2 * i].spec = f->spec;
    pw[2 * i + 1].mode = MODE_LAST;
    pw[2 * i + 1].spec = f->spec;
    pw[2 * i + 1].store = w;
  }
  PencilWork<double> xw;
  memset(&xw, 0, sizeof(xw));
  xw.spec = f->spec;
  PS_CUDA(h, cudaMalloc((void**)&f->d_pw, sizeof(PlaneWork<double>) * pw.size()));
  PS_CUDA(h, cudaMemcpy(f->d_pw, pw.data(), sizeof(PlaneWork<double>) * pw.size(), cudaMemcpyHostToDevice));
  PS_CUDA(h, cudaMalloc((void**)&f->d_xw, sizeof(xw)));
  PS_CUDA(h, cudaMemcpy(f->d_xw, &xw, sizeof(xw), cudaMemcpyHostToDevice));
  PS_CUDA(h, cudaMalloc((void**)&f->part, sizeof(double) * kRedBlocks));
  PS_CUDA(h, cudaMalloc((void**)&f->scal, sizeof(double) * 2));
  f->multi = c->spec_cells[0] || c->spec_cells[1] || c->spec_cells[2];
  if (f->multi) {
    f->ncells = (long long)(nx / c->spec_cells[0]) * (ny / c->spec_cells[1]) * (nz / c->spec_cells[2]);
    PS_CUDA(h, cudaMalloc((void**)&f->cut, sizeof(double) * (size_t)f->ncells));
  }
  return PS_OK;
}

static int filter_apply(ps_handle* h) {
  FilterState* f = static_cast<FilterState*>(h->filter);
  const ps_filter_config& c = f->cfg;
  if (c.cutoff_factor <= 0.0) return PS_OK;  // even a zero cutoff would perturb the fields
  const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
  const long long N = h->N;
  const long long nspec = (long long)nx * ny * h->nzh;
  cudaStream_t st = h->st;
  int blocks = (int)((N + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  for (int i = 0; i < c.n_fields; ++i) {
    double* w = h->d_w + (size_t)c.fields[i] * N;
    filter_sum_partials<<<kRedBlocks, kFT, 0, st>>>(w, N, f->part, 0, nullptr);
    filter_finalize<<<1, kFT, 0, st>>>(f->part, kRedBlocks, 0, (double)N, f->scal);
    filter_shift<<<blocks, 256, 0, st>>>(w, N, f->scal);
    PS_CUDA(h, cudaGetLastError());
    // forward r2c
    if (f->fused) {
      PS_CUDA(h, launch_plane<double>(f->d_pw + 2 * i, 1, nx, ny, nz, f->tw_y, f->tw_zh, f->tw_z, 0, st));
    } else {
      PS_CUDA(h, launch_rows<double>(f->d_pw + 2 * i, 1, nx * ny, nz, f->tw_zh, f->tw_z, st));
      if (ny > 1) PS_CUDA(h, launch_pencil<double>(f->d_xw, 1, PENCIL_FWD, ny, nx, h->nzh, f->tw_y, nx, ny, nz, 0, st));
    }
    PS_CUDA(h, launch_pencil<double>(f->d_xw, 1, PENCIL_FWD, nx, 1, ny * h->nzh, f->tw_x, nx, ny, nz, 0, st));
    if (f->multi) {
      const Regions g = regions_of(h, c);
      PS_CUDA(h, cudaMemsetAsync(f->cut, 0, sizeof(double) * (size_t)f->ncells, st));
      unsigned long long* cu = reinterpret_cast<unsigned long long*>(f->cut);
      if (f->ncells <= kShCells)
        filter_region_max<true><<<blocks, 256, 0, st>>>(f->spec, nspec, g, cu, f->ncells);
      else
        filter_region_max<false><<<blocks, 256, 0, st>>>(f->spec, nspec, g, cu, f->ncells);
      filter_mask_multi<<<blocks, 256, 0, st>>>(f->spec, nspec, g, f->cut, c.cutoff_factor, c.filter_strength,
                                                1.0 / (double)N);
    } else {
      filter_sum_partials<<<kRedBlocks, kFT, 0, st>>>(nullptr, nspec, f->part, 1, f->spec);
      filter_finalize<<<1, kFT, 0, st>>>(f->part, kRedBlocks, 1, (double)N, f->scal + 1);
      filter_mask<<<blocks, 256, 0, st>>>(f->spec, nspec, f->scal + 1, c.cutoff_factor, c.filter_strength,
                                          1.0 / (double)N);
    }
    PS_CUDA(h, cudaGetLastError());
    // inverse c2r, stored back into w
    PS_CUDA(h, launch_pencil<double>(f->d_xw, 1, PENCIL_INV, nx, 1, ny * h->nzh, f->tw_x, nx, ny, nz, 0, st));
    if (f->fused) {
      PS_CUDA(h, launch_plane<double>(f->d_pw + 2 * i + 1, 1, nx, ny, nz, f->tw_y, f->tw_zh, f->tw_z, 0, st));
    } else {
      if (ny > 1) PS_CUDA(h, launch_pencil<double>(f->d_xw, 1, PENCIL_INV, ny, nx, h->nzh, f->tw_y, nx, ny, nz, 0, st));
      PS_CUDA(h, launch_rows<double>(f->d_pw + 2 * i + 1, 1, nx * ny, nz, f->tw_zh, f->tw_z, st));
    }
  }
  return PS_OK;
}

int filter_after_iteration(ps_handle* h, long long step) {
  FilterState* f = static_cast<FilterState*>(h->filter);
  if (!f) return PS_OK;
  const ps_filter_config& c = f->cfg;
  if (step < c.apply_start || (c.apply_end >= 0 && step > c.apply_end)) return PS_OK;
  if ((step - c.apply_start) % c.apply_frequency != 0) return PS_OK;
  return filter_apply(h);
}

}  // namespace psb

using namespace psb;

extern "C" {

int ps_gpu_set_spectral_filter(ps_handle* h, const ps_filter_config* c) {
  if (!h) return PS_ATTRIB_ERR;
  PS_CUDA(h, cudaSetDevice(h->dev));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  filter_free(h);
  post_order_set(h, POST_FILTER, false);
  if (!c) return PS_OK;
  if (c->n_fields < 1 || c->n_fields > h->nf) {
    h->err = "spectral filter: n_fields out of range";
    return PS_ATTRIB_ERR;
  }
  for (int i = 0; i < c->n_fields; ++i)
    if (c->fields[i] < 0 || c->fields[i] >= h->nf) {
      h->err = "spectral filter: field index out of range";
      return PS_ATTRIB_ERR;
    }
  if (c->spec_cells[0] || c->spec_cells[1] || c->spec_cells[2])
    for (int d = 0; d < 3; ++d)
      if (c->spec_cells[d] < 1 || h->n[d] % c->spec_cells[d] != 0) {
        h->err = "multiSpecFilter: each specCellSizes entry must divide its grid extent";
        return PS_ATTRIB_ERR;
      }
  if (c->apply_frequency < 1) {
    h->err = "spectral filter: apply_frequency must be >= 1";
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
  int rc = filter_build(h, c);
  if (rc) {
    filter_free(h);
    return rc;
  }
  post_order_set(h, POST_FILTER, true);
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

int ps_gpu_apply_spectral_filter(ps_handle* h) {
  if (!h) return PS_ATTRIB_ERR;
  if (!h->filter) {
    h->err = "no spectral filter set";
    return PS_ATTRIB_ERR;
  }
  PS_CUDA(h, cudaSetDevice(h->dev));
  int rc = filter_apply(h);
  if (rc) return rc;
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  return PS_OK;
}

}  // extern "C"
