// scaledFFTPair that allocates nothing: ps_fft_scaled_pair_noalloc.
//
// For callers that cannot allocate device memory when they need the
// transform: a host whose device memory is entirely owned by another
// allocator (a framework's caching allocator or a memory pool that reserved
// the GPU up front), or a long-running solver loop that must not allocate
// after start-up.  They pass their own device buffers for the inputs and the
// output; the working storage (the half spectrum, twiddle tables and work
// descriptors) is a fixed file-scope device array below.
//
// Limits and behaviour:
// * the scratch is kNoAllocScratchBytes = 4 MiB per device, held by every GPU
//   that loads the library until the process exits; a grid needs
//   nx*ny*(nz/2+1)*16 bytes of half spectrum plus small tables (64^3 fits,
//   96^3 does not); larger grids are rejected with PS_INPUT_ERR;
// * every call on a device shares the same scratch and leaves its contents
//   behind; each call rewrites all of it before reading it, so nothing has to
//   start at zero, but calls that overlap on the GPU (different streams, or
//   host threads racing) corrupt each other's results;
// * the first call on a device resolves the scratch address
//   (cudaGetSymbolAddress) with that device current; make that first call
//   before any stream capture.  Later calls outside a capture resolve it
//   again (cheap, allocates nothing), so the address stays right after the
//   host application resets the device;
// * the call is asynchronous on `stream`: res is valid once the stream is
//   synchronised;
// * the transform kernels bound their waits on the bulk copies; a copy that
//   does not land in time leaves res unwritten, and this entry point does not
//   report it (it returns before the GPU runs).
// No cudaMalloc, cudaFree or allocating library routine is called.
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/pswift.h"
#include "kernels.h"

namespace psb {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[64] = {};  // device address of the scratch, per device ordinal
static thread_local std::string g_noalloc_err;

__global__ void noalloc_twiddle_kernel(double2* tw, int L) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)m / (double)L, &s, &c);
    tw[m] = make_double2(c, -s);
  }
}

__global__ void noalloc_works_kernel(PlaneWork<double>* pw, PencilWork<double>* xw,
                                     const double* data, const double* kdata, double* res,
                                     double2* spec) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  PlaneWork<double> a = {};
  a.mode = MODE_FIRST;
  a.src = data;
  a.spec = spec;
  PlaneWork<double> b = {};
  b.mode = MODE_LAST;
  b.spec = spec;
  b.store = res;
  pw[0] = a;
  pw[1] = b;
  PencilWork<double> x = {};
  x.spec = spec;
  x.kfull = kdata;
  xw[0] = x;
}

// Launched without programmatic serialisation between the set-up kernels and
// the first transform kernel.  The transform kernels are launched with it and
// read their work descriptors and twiddles before waiting on the kernel ahead
// of them; behind this ordinary launch that kernel cannot start before the
// set-up kernels have finished and their writes are visible.
__global__ void noalloc_order_kernel() {}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Resolve the scratch address for the current device: on the first call, and
// on every call made outside a stream capture (`refresh`).
static int noalloc_scratch(int dev, bool refresh, unsigned char** out) {
  if (dev < 0 || dev >= 64) {
    g_noalloc_err = "device ordinal out of range";
    return PS_GPU_ERR;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev] || refresh) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      g_noalloc_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return PS_GPU_ERR;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return PS_OK;
}

}  // namespace psb

using namespace psb;

#define NA_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      g_noalloc_err = std::string(#call) + ": " + cudaGetErrorString(e_);    \
      return PS_GPU_ERR;                                                     \
    }                                                                        \
  } while (0)

extern "C" {

size_t ps_fft_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

const char* ps_fft_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

int ps_fft_scaled_pair_noalloc(const int n[3], const double* d_data, const double* d_kdata,
                               double* d_res, void* stream) {
  if (!n || !d_data || !d_kdata || !d_res) {
    g_noalloc_err = "null argument";
    return PS_ATTRIB_ERR;
  }
  // data and res are read and written as 16-byte vectors.
  if ((reinterpret_cast<uintptr_t>(d_data) | reinterpret_cast<uintptr_t>(d_res)) & 15) {
    g_noalloc_err = "data and res must be 16-byte aligned device pointers";
    return PS_ATTRIB_ERR;
  }
  const int nx = n[0], ny = n[1], nz = n[2];
  for (int d = 0; d < 3; ++d) {
    if (!extent_supported(n[d])) {
      g_noalloc_err = "unsupported FFT extent " + std::to_string(n[d]);
      return PS_INPUT_ERR;
    }
  }
  const int nzh = nz / 2 + 1;
  const int nzhalf = nz / 2 > 0 ? nz / 2 : 1;
  // scratch layout: spectrum | tw_x | tw_y | tw_z | tw_zh | plane works | pencil work
  size_t off = 0;
  const size_t o_spec = off;
  off = align256(off + sizeof(double2) * (size_t)nx * ny * nzh);
  const size_t o_twx = off;
  off = align256(off + sizeof(double2) * (size_t)nx);
  const size_t o_twy = off;
  off = align256(off + sizeof(double2) * (size_t)ny);
  const size_t o_twz = off;
  off = align256(off + sizeof(double2) * (size_t)nz);
  const size_t o_twzh = off;
  off = align256(off + sizeof(double2) * (size_t)nzhalf);
  const size_t o_pw = off;
  off = align256(off + 2 * sizeof(PlaneWork<double>));
  const size_t o_xw = off;
  off = align256(off + sizeof(PencilWork<double>));
  if (off > kNoAllocScratchBytes) {
    g_noalloc_err = "grid " + std::to_string(nx) + "x" + std::to_string(ny) + "x" +
                    std::to_string(nz) + " needs " + std::to_string(off) +
                    " bytes of scratch; the allocation-free entry point has " +
                    std::to_string(kNoAllocScratchBytes);
    return PS_INPUT_ERR;
  }
  int dev = 0;
  NA_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  NA_CUDA(cudaStreamIsCapturing(st, &cap));
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(dev, cap == cudaStreamCaptureStatusNone, &base);
  if (rc) return rc;
  double2* spec = reinterpret_cast<double2*>(base + o_spec);
  double2* twx = reinterpret_cast<double2*>(base + o_twx);
  double2* twy = reinterpret_cast<double2*>(base + o_twy);
  double2* twz = reinterpret_cast<double2*>(base + o_twz);
  double2* twzh = reinterpret_cast<double2*>(base + o_twzh);
  PlaneWork<double>* pw = reinterpret_cast<PlaneWork<double>*>(base + o_pw);
  PencilWork<double>* xw = reinterpret_cast<PencilWork<double>*>(base + o_xw);
  noalloc_twiddle_kernel<<<1, 256, 0, st>>>(twx, nx);
  noalloc_twiddle_kernel<<<1, 256, 0, st>>>(twy, ny);
  noalloc_twiddle_kernel<<<1, 256, 0, st>>>(twz, nz);
  noalloc_twiddle_kernel<<<1, 256, 0, st>>>(twzh, nzhalf);
  noalloc_works_kernel<<<1, 1, 0, st>>>(pw, xw, d_data, d_kdata, d_res, spec);
  noalloc_order_kernel<<<1, 1, 0, st>>>();
  NA_CUDA(cudaGetLastError());
  if (plane_fused_supported(8, ny, nz)) {
    NA_CUDA(launch_plane<double>(pw, 1, nx, ny, nz, twy, twzh, twz, 0, st));
    NA_CUDA(launch_pencil<double>(xw, 1, PENCIL_KFULL, nx, 1, ny * nzh, twx, nx, ny, nz, 0, st));
    NA_CUDA(launch_plane<double>(pw + 1, 1, nx, ny, nz, twy, twzh, twz, 0, st));
  } else {
    NA_CUDA(launch_rows<double>(pw, 1, nx * ny, nz, twzh, twz, st));
    if (ny > 1)
      NA_CUDA(launch_pencil<double>(xw, 1, PENCIL_FWD, ny, nx, nzh, twy, nx, ny, nz, 0, st));
    NA_CUDA(launch_pencil<double>(xw, 1, PENCIL_KFULL, nx, 1, ny * nzh, twx, nx, ny, nz, 0, st));
    if (ny > 1)
      NA_CUDA(launch_pencil<double>(xw, 1, PENCIL_INV, ny, nx, nzh, twy, nx, ny, nz, 0, st));
    NA_CUDA(launch_rows<double>(pw + 1, 1, nx * ny, nz, twzh, twz, st));
  }
  return PS_OK;
}

}  // extern "C"
