// FFT plugin: PsFFTBase<double,3> on the device (psbase/PsFFTBase.h:40-134;
// serial semantics of psfft/PsFFTW.cpp:122-297).
//
// scaledFFTPair: res = Re(IFFT(kdata * FFT(data))) with both transforms
// unnormalised.  The reference computes it as a c2c pair of real data; here it
// is the same plane / pencil kernels as the propagator (r2c -> pencils -> c2r)
// with the k multiplier taken from the full real kdata array, symmetrised as
// (kdata(k) + kdata(-k)) / 2, which is what the real part of the c2c result
// sees.  The other operations of the interface reuse the same passes:
//   scaledFFTPairIm: c2r of i (kdata(k) - kdata(-k))/2 FFT(data);
//   convolveRe:      c2r of FFT(data1) FFT(data2);
//   forwardFFTAbs, calcForwardFFT, calcBackwardFFT: the r2c half spectrum
//     expanded to the full grid by X(-k) = conj(X(k)) and reduced to |X|^2 or
//     Re X (for real input Re(IFFT(d)) = Re(FFT(d)): both are sum d cos(k.r)).
// Host arrays in and out (H2D and D2H copies on the plugin's stream per call).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/pswift.h"
#include "kernels.h"

namespace psb {
static thread_local std::string g_fft_err;
}

struct ps_fft {
  int n[3];
  long long N;
  int nzh;
  int dev;
  bool fused;
  cudaStream_t st;
  double* d_data;
  double* d_res;
  double* d_k;      // kdata, or the second input of convolveRe
  double2* d_spec;
  double2* d_spec2;  // convolveRe: the second operand's transform
  double2 *tw_x, *tw_y, *tw_z, *tw_zh;
  psb::PlaneWork<double>* d_pw;   // [0] FIRST data -> spec, [1] LAST spec -> res, [2] FIRST d_k -> spec2
  psb::PencilWork<double>* d_xw;  // [0] spec (kfull = d_k), [1] spec2, [2] spec (kspec = spec2)
};

namespace psb {

static cudaError_t twiddles(double2** dst, int L) {
  std::vector<double2> tw(L > 0 ? L : 1);
  const double twopi = 2.0 * acos(-1.0);
  for (int m = 0; m < L; ++m) {
    const double a = twopi * (double)m / (double)L;
    tw[m].x = cos(a);
    tw[m].y = -sin(a);
  }
  cudaError_t e = cudaMalloc((void**)dst, sizeof(double2) * tw.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice);
}

// Full-grid output from a fully transformed half spectrum S[x][y][kz]:
// X(x,y,z) = S[x][y][z] for z <= nz/2, conj(S[-x][-y][nz-z]) otherwise;
// res = |X|^2 (power) or Re X.
__global__ void fft_expand_kernel(const double2* __restrict__ spec, double* __restrict__ res, int nx,
                                  int ny, int nz, int power) {
  const int nzh = nz / 2 + 1;
  const long long N = (long long)nx * ny * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(i % nz);
    const long long xy = i / nz;
    const int y = (int)(xy % ny);
    const int x = (int)(xy / ny);
    double2 v;
    if (z < nzh) {
      v = spec[((size_t)x * ny + y) * nzh + z];
    } else {
      const int xm = (nx - x) % nx, ym = (ny - y) % ny;
      v = spec[((size_t)xm * ny + ym) * nzh + (nz - z)];
    }
    res[i] = power ? (v.x * v.x) + (v.y * v.y) : v.x;
  }
}

static void fft_free(ps_fft* f) {
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(f->d_data); fr(f->d_res); fr(f->d_k); fr(f->d_spec); fr(f->d_spec2);
  fr(f->tw_x); fr(f->tw_y); fr(f->tw_z); fr(f->tw_zh); fr(f->d_pw); fr(f->d_xw);
  if (f->st) cudaStreamDestroy(f->st);
}

}  // namespace psb

using namespace psb;

#define FFT_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      g_fft_err = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return PS_GPU_ERR;                                                       \
    }                                                                          \
  } while (0)

static int fft_create_impl(ps_fft* f, const int n[3], int device) {
  for (int d = 0; d < 3; ++d) {
    f->n[d] = n[d];
    if (!extent_supported(n[d])) {
      g_fft_err = "unsupported FFT extent " + std::to_string(n[d]);
      return PS_INPUT_ERR;
    }
  }
  f->N = (long long)n[0] * n[1] * n[2];
  f->nzh = n[2] / 2 + 1;
  f->dev = device;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    g_fft_err = "no CUDA device available";
    return PS_GPU_ERR;
  }
  FFT_CUDA(cudaSetDevice(device));
  FFT_CUDA(cudaStreamCreateWithFlags(&f->st, cudaStreamNonBlocking));
  f->fused = plane_fused_supported(8, n[1], n[2]);
  const size_t N = (size_t)f->N;
  FFT_CUDA(cudaMalloc((void**)&f->d_data, sizeof(double) * N));
  FFT_CUDA(cudaMalloc((void**)&f->d_res, sizeof(double) * N));
  FFT_CUDA(cudaMalloc((void**)&f->d_k, sizeof(double) * N));
  FFT_CUDA(cudaMalloc((void**)&f->d_spec, sizeof(double2) * (size_t)n[0] * n[1] * f->nzh));
  FFT_CUDA(cudaMalloc((void**)&f->d_spec2, sizeof(double2) * (size_t)n[0] * n[1] * f->nzh));
  FFT_CUDA(twiddles(&f->tw_x, n[0]));
  FFT_CUDA(twiddles(&f->tw_y, n[1]));
  FFT_CUDA(twiddles(&f->tw_z, n[2]));
  FFT_CUDA(twiddles(&f->tw_zh, n[2] / 2 > 0 ? n[2] / 2 : 1));
  PlaneWork<double> pw[3];
  memset(pw, 0, sizeof(pw));
  pw[0].mode = MODE_FIRST;
  pw[0].src = f->d_data;
  pw[0].spec = f->d_spec;
  pw[1].mode = MODE_LAST;
  pw[1].spec = f->d_spec;
  pw[1].store = f->d_res;
  pw[2].mode = MODE_FIRST;
  pw[2].src = f->d_k;
  pw[2].spec = f->d_spec2;
  PencilWork<double> xw[3];
  memset(xw, 0, sizeof(xw));
  xw[0].spec = f->d_spec;
  xw[0].kfull = f->d_k;
  xw[1].spec = f->d_spec2;
  xw[2].spec = f->d_spec;
  xw[2].kspec = f->d_spec2;
  FFT_CUDA(cudaMalloc((void**)&f->d_pw, sizeof(pw)));
  FFT_CUDA(cudaMemcpy(f->d_pw, pw, sizeof(pw), cudaMemcpyHostToDevice));
  FFT_CUDA(cudaMalloc((void**)&f->d_xw, sizeof(xw)));
  FFT_CUDA(cudaMemcpy(f->d_xw, xw, sizeof(xw), cudaMemcpyHostToDevice));
  return PS_OK;
}

// r2c of the plane work `pw` into its spectrum (xw's), all three axes.
static cudaError_t fft_r2c(ps_fft* f, const PlaneWork<double>* pw, const PencilWork<double>* xw) {
  const int nx = f->n[0], ny = f->n[1], nz = f->n[2];
  cudaError_t e;
  if (f->fused) {
    e = launch_plane<double>(pw, 1, nx, ny, nz, f->tw_y, f->tw_zh, f->tw_z, 0, f->st);
  } else {
    e = launch_rows<double>(pw, 1, nx * ny, nz, f->tw_zh, f->tw_z, f->st);
    if (e == cudaSuccess && ny > 1)
      e = launch_pencil<double>(xw, 1, PENCIL_FWD, ny, nx, f->nzh, f->tw_y, nx, ny, nz, 0, f->st);
  }
  if (e == cudaSuccess)
    e = launch_pencil<double>(xw, 1, PENCIL_FWD, nx, 1, ny * f->nzh, f->tw_x, nx, ny, nz, 0, f->st);
  return e;
}

static int check_args(const void* a, const void* b, const void* c) {
  if (!a || !b || !c) {
    g_fft_err = "null argument";
    return PS_ATTRIB_ERR;
  }
  return PS_OK;
}

// r2c of `data`, one x-pencil pass of mode `kmode` (forward x, multiply,
// inverse x), c2r into res.  `other` is kdata (KFULL, KFULL_IM) or the second
// input (KSPEC, transformed first into spec2).
static int fft_pair_call(ps_fft* f, const double* data, const double* other, double* res, int kmode) {
  if (!f) {
    g_fft_err = "null handle";
    return PS_ATTRIB_ERR;
  }
  if (int rc = check_args(data, other, res)) return rc;
  const size_t N = (size_t)f->N;
  const int nx = f->n[0], ny = f->n[1], nz = f->n[2];
  FFT_CUDA(cudaSetDevice(f->dev));
  FFT_CUDA(cudaMemcpyAsync(f->d_data, data, sizeof(double) * N, cudaMemcpyHostToDevice, f->st));
  FFT_CUDA(cudaMemcpyAsync(f->d_k, other, sizeof(double) * N, cudaMemcpyHostToDevice, f->st));
  const PencilWork<double>* xk = f->d_xw;
  if (kmode == PENCIL_KSPEC) {
    FFT_CUDA(fft_r2c(f, f->d_pw + 2, f->d_xw + 1));
    xk = f->d_xw + 2;
  }
  if (f->fused) {
    FFT_CUDA(launch_plane<double>(f->d_pw, 1, nx, ny, nz, f->tw_y, f->tw_zh, f->tw_z, 0, f->st));
    FFT_CUDA(launch_pencil<double>(xk, 1, kmode, nx, 1, ny * f->nzh, f->tw_x, nx, ny, nz, 0, f->st));
    FFT_CUDA(launch_plane<double>(f->d_pw + 1, 1, nx, ny, nz, f->tw_y, f->tw_zh, f->tw_z, 0, f->st));
  } else {
    FFT_CUDA(launch_rows<double>(f->d_pw, 1, nx * ny, nz, f->tw_zh, f->tw_z, f->st));
    if (ny > 1)
      FFT_CUDA(launch_pencil<double>(f->d_xw, 1, PENCIL_FWD, ny, nx, f->nzh, f->tw_y, nx, ny, nz, 0, f->st));
    FFT_CUDA(launch_pencil<double>(xk, 1, kmode, nx, 1, ny * f->nzh, f->tw_x, nx, ny, nz, 0, f->st));
    if (ny > 1)
      FFT_CUDA(launch_pencil<double>(f->d_xw, 1, PENCIL_INV, ny, nx, f->nzh, f->tw_y, nx, ny, nz, 0, f->st));
    FFT_CUDA(launch_rows<double>(f->d_pw + 1, 1, nx * ny, nz, f->tw_zh, f->tw_z, f->st));
  }
  FFT_CUDA(cudaMemcpyAsync(res, f->d_res, sizeof(double) * N, cudaMemcpyDeviceToHost, f->st));
  FFT_CUDA(cudaStreamSynchronize(f->st));
  return PS_OK;
}

// r2c of `data`, expanded to the full grid as |X|^2 (power) or Re X.
static int fft_forward_call(ps_fft* f, const double* data, double* res, int power) {
  if (!f) {
    g_fft_err = "null handle";
    return PS_ATTRIB_ERR;
  }
  if (int rc = check_args(data, res, res)) return rc;
  const size_t N = (size_t)f->N;
  FFT_CUDA(cudaSetDevice(f->dev));
  FFT_CUDA(cudaMemcpyAsync(f->d_data, data, sizeof(double) * N, cudaMemcpyHostToDevice, f->st));
  FFT_CUDA(fft_r2c(f, f->d_pw, f->d_xw));
  const int blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 8);
  fft_expand_kernel<<<blocks, 256, 0, f->st>>>(f->d_spec, f->d_res, f->n[0], f->n[1], f->n[2], power);
  FFT_CUDA(cudaGetLastError());
  FFT_CUDA(cudaMemcpyAsync(res, f->d_res, sizeof(double) * N, cudaMemcpyDeviceToHost, f->st));
  FFT_CUDA(cudaStreamSynchronize(f->st));
  return PS_OK;
}

extern "C" {

int ps_fft_create(const int n[3], int precision, int device, ps_fft** out) {
  if (!n || !out) {
    g_fft_err = "null argument";
    return PS_ATTRIB_ERR;
  }
  *out = nullptr;
  if (precision != PS_PREC_FP64) {
    g_fft_err = "the scaledFFTPair plugin computes in FP64 only";
    return PS_ATTRIB_ERR;
  }
  ps_fft* f = new ps_fft;
  memset(f, 0, sizeof(*f));
  int rc = fft_create_impl(f, n, device);
  if (rc != PS_OK) {
    fft_free(f);
    delete f;
    cudaGetLastError();  // clear a failed allocation's last-error state
    return rc;
  }
  *out = f;
  return PS_OK;
}

int ps_fft_destroy(ps_fft* f) {
  if (!f) return PS_OK;
  cudaSetDevice(f->dev);
  if (f->st) cudaStreamSynchronize(f->st);
  fft_free(f);
  delete f;
  return PS_OK;
}

int ps_fft_size(const ps_fft* f, size_t* n_total) {
  if (!f || !n_total) return PS_ATTRIB_ERR;
  *n_total = (size_t)f->N;
  return PS_OK;
}

int ps_fft_scaled_pair(ps_fft* f, const double* data, const double* kdata, double* res) {
  return fft_pair_call(f, data, kdata, res, PENCIL_KFULL);
}

int ps_fft_scaled_pair_im(ps_fft* f, const double* data, const double* kdata, double* res) {
  return fft_pair_call(f, data, kdata, res, PENCIL_KFULL_IM);
}

int ps_fft_convolve_re(ps_fft* f, const double* data1, const double* data2, double* res) {
  return fft_pair_call(f, data1, data2, res, PENCIL_KSPEC);
}

int ps_fft_forward_abs(ps_fft* f, const double* data, double* res) {
  return fft_forward_call(f, data, res, 1);
}

int ps_fft_forward(ps_fft* f, const double* data, double* res) {
  return fft_forward_call(f, data, res, 0);
}

int ps_fft_backward(ps_fft* f, const double* data, double* res) {
  return fft_forward_call(f, data, res, 0);
}

int ps_fft_get_grid(const ps_fft* f, int n[3]) {
  if (!f || !n) return PS_ATTRIB_ERR;
  for (int d = 0; d < 3; ++d) n[d] = f->n[d];
  return PS_OK;
}

const char* ps_fft_last_error(void) { return g_fft_err.c_str(); }

}  // extern "C"
