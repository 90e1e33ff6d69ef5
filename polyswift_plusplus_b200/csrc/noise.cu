// Updater noise on the device: the reference's per-iteration Gaussian draws
// (addRandUpdateConjgFields, pseffhamil/PsPolymerUpdater.cpp:263-295;
// PsRandom::gauss, psstd/PsRandom.h:327-364) taken from the same MT19937
// stream, in the same order, without a host loop over nf * N draws.
//
// One iteration needs K = nf * N Gaussians.  The Marsaglia polar method takes
// pairs of consecutive uniforms, rejects pairs outside the unit disc, returns
// v2 * fac and caches v1 * fac for the next call.  On the device:
//   1. one block advances the MT19937 state G generations (one barrier per
//      generation) and stores the words of every generation, so that word p of
//      the stream after the current state is words[p];
//   2. one thread per pair attempt tempers its two words and tests acceptance;
//      blocks count their accepted pairs and one block scans the counts;
//   3. the accepted pair of rank q writes outputs off + 2q and off + 2q + 1
//      (off = 1 when a cached value is pending, which is output 0); the pair
//      that supplies output K - 1 marks where the stream stops;
//   4. one block moves the state there (a stored generation and an index), with
//      the cached value when that pair supplied only one output.
// G is set from K with a margin of more than 15 standard deviations of the
// rejection count; running short sets an error flag (read back with the
// iteration's status), it never reads past the stored words.
// The accept decisions and stream positions are exact (no contraction of the
// products and sums that decide them); the Gaussians equal the host's up to
// the rounding of log().
#include <math.h>
#include <string.h>

#include "engine_state.h"

namespace psb {

struct DevRng {
  uint32_t mt[624];
  int idx;
  int have_gauss;
  double gauss;
  int err;
  int pad;
};

struct RngFinal {
  long long j;  // attempt that supplied output K - 1 (-1: none)
  int have;
  int pad;
  double gauss;
};

struct NoiseState {
  DevRng* d_rng = nullptr;
  DevRng* h_rng = nullptr;  // pinned staging
  RngFinal* d_fin = nullptr;
  uint32_t* words = nullptr;  // (G + 1) * 624
  int* boff = nullptr;        // accepted pairs per block, then their exclusive scan
  long long K = 0;
  int G = 0;          // generations advanced per iteration
  long long J = 0;    // pair attempts evaluated per iteration (G * 312)
  int nblk = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_iter = nullptr, ev_noise = nullptr;
  bool on_device = false;  // the device state is the current one
};

constexpr int kPairT = 1024;
constexpr int kTwistT = 256;

__device__ __forceinline__ uint32_t temper(uint32_t y) {
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

__device__ __forceinline__ uint32_t twist_one(uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
  uint32_t v = c ^ (y >> 1);
  if (y & 1u) v ^= 0x9908b0dfu;
  return v;
}

// G generations of the twist.  New element k is built from old k, old k + 1 and
// the element 397 ahead (old for k < 227, else the new k - 227; new 0 for
// k = 623).  Thread t < 227 builds elements t, t + 227 and (t < 169) t + 454,
// each from old values and its own previous result; thread 169 also builds 623,
// recomputing new 0.  Old and new generations sit in two shared buffers, so a
// generation needs one barrier.
__global__ void __launch_bounds__(kTwistT) rng_twist_kernel(const DevRng* __restrict__ st,
                                                           uint32_t* __restrict__ words, int G) {
  __shared__ uint32_t buf[2][624];
  const int t = threadIdx.x;
  for (int k = t; k < 624; k += kTwistT) {
    const uint32_t x = st->mt[k];
    buf[0][k] = x;
    words[k] = x;
  }
  __syncthreads();
  for (int g = 1; g <= G; ++g) {
    const uint32_t* o = buf[(g - 1) & 1];
    uint32_t* nw = buf[g & 1];
    uint32_t* out = words + (size_t)g * 624;
    if (t < 227) {
      const uint32_t a = twist_one(o[t], o[t + 1], o[t + 397]);
      const uint32_t b = twist_one(o[t + 227], o[t + 228], a);
      nw[t] = a;
      nw[t + 227] = b;
      out[t] = a;
      out[t + 227] = b;
      if (t < 169) {
        const uint32_t c = twist_one(o[t + 454], o[t + 455], b);
        nw[t + 454] = c;
        out[t + 454] = c;
      }
      if (t == 169) {
        const uint32_t a0 = twist_one(o[0], o[1], o[397]);
        const uint32_t d = twist_one(o[623], a0, b);  // b is new element 396
        nw[623] = d;
        out[623] = d;
      }
    }
    __syncthreads();
  }
}

// Pair attempt j uses stream words idx + 2j and idx + 2j + 1 (psstd/PsRandom.h:
// real() = u32 * 2^-32, v = 2 real - 1, r = v1^2 + v2^2, reject r >= 1 or r == 0).
__device__ __forceinline__ bool pair_attempt(const uint32_t* __restrict__ words, long long pos, double& v1,
                                             double& v2, double& r) {
  const double a = (double)temper(words[pos]) * (1.0 / 4294967296.0);
  const double b = (double)temper(words[pos + 1]) * (1.0 / 4294967296.0);
  v1 = __dadd_rn(__dmul_rn(2.0, a), -1.0);
  v2 = __dadd_rn(__dmul_rn(2.0, b), -1.0);
  r = __dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2));
  return !((r >= 1.0) || (r == 0.0));
}

// Exclusive rank of this thread's flag inside the block; returns the block's
// count (valid in warp 0).
__device__ __forceinline__ int block_rank(int acc, int* wsum, int* rank) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, acc);
  *rank = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) wsum[warp] = __popc(m);
  __syncthreads();
  int total = 0;
  if (warp == 0) {
    const int x = (lane < kPairT / 32) ? wsum[lane] : 0;
    int inc = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane < kPairT / 32) wsum[lane] = inc - x;
    total = __shfl_sync(0xffffffffu, inc, 31);
  }
  __syncthreads();
  *rank += wsum[warp];
  return total;
}

__global__ void __launch_bounds__(kPairT) rng_count_kernel(const DevRng* __restrict__ st,
                                                          const uint32_t* __restrict__ words, long long J,
                                                          int* __restrict__ boff, RngFinal* __restrict__ fin) {
  __shared__ int wsum[kPairT / 32];
  const long long j = (long long)blockIdx.x * kPairT + threadIdx.x;
  int acc = 0;
  if (j < J) {
    double v1, v2, r;
    acc = pair_attempt(words, (long long)st->idx + 2 * j, v1, v2, r) ? 1 : 0;
  }
  int rank = 0;
  const int total = block_rank(acc, wsum, &rank);
  if (threadIdx.x == 0) {
    boff[blockIdx.x] = total;
    if (blockIdx.x == 0) fin->j = -1;
  }
}

// Exclusive scan of the block counts, in place (one block).
__global__ void __launch_bounds__(kPairT) rng_scan_kernel(int* __restrict__ boff, int nb) {
  __shared__ int s[kPairT];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kPairT) {
    const int i = base + threadIdx.x;
    const int x = (i < nb) ? boff[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < kPairT; o <<= 1) {
      const int y = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < nb) boff[i] = carry + s[threadIdx.x] - x;
    __syncthreads();
    if (threadIdx.x == kPairT - 1) carry += s[kPairT - 1];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kPairT) rng_out_kernel(const DevRng* __restrict__ st,
                                                        const uint32_t* __restrict__ words, long long J,
                                                        const int* __restrict__ boff, long long K, double sigma,
                                                        double* __restrict__ out, RngFinal* __restrict__ fin) {
  __shared__ int wsum[kPairT / 32];
  const long long j = (long long)blockIdx.x * kPairT + threadIdx.x;
  const int off = st->have_gauss ? 1 : 0;
  if (j == 0 && off) out[0] = sigma * st->gauss;
  bool acc = false;
  double v1 = 0.0, v2 = 0.0, r = 0.0;
  if (j < J) acc = pair_attempt(words, (long long)st->idx + 2 * j, v1, v2, r);
  int rank = 0;
  (void)block_rank(acc ? 1 : 0, wsum, &rank);
  if (!acc) return;
  const long long q = (long long)boff[blockIdx.x] + rank;
  const long long o1 = off + 2 * q, o2 = o1 + 1;
  if (o1 >= K) return;
  const double fac = sqrt(-2.0 * log(r) / r);
  out[o1] = sigma * (v2 * fac);
  if (o2 < K) out[o2] = sigma * (v1 * fac);
  if (o1 == K - 1) {
    fin->j = j;
    fin->have = 1;
    fin->gauss = v1 * fac;
  } else if (o2 == K - 1) {
    fin->j = j;
    fin->have = 0;
    fin->gauss = 0.0;
  }
}

// Move the state to just after the last pair used.
__global__ void __launch_bounds__(kTwistT) rng_final_kernel(DevRng* __restrict__ st,
                                                           const uint32_t* __restrict__ words,
                                                           const RngFinal* __restrict__ fin, long long K, int G) {
  const int off = st->have_gauss ? 1 : 0;
  const long long jl = fin->j;
  const long long p = (long long)st->idx + 2 * (jl + 1);
  __syncthreads();  // every thread has read the old state
  if (K - off <= 0) {  // only the cached value was used
    if (threadIdx.x == 0) st->have_gauss = 0;
    return;
  }
  // word p is next: generation p / 624 at index p % 624, or generation
  // p / 624 - 1 at index 624 when p is a multiple of 624
  long long gen = p / 624, idx = p - gen * 624;
  if (idx == 0) {
    gen -= 1;
    idx = 624;
  }
  if (jl < 0 || gen > G) {
    if (threadIdx.x == 0) st->err = 1;
    return;
  }
  for (int k = threadIdx.x; k < 624; k += kTwistT) st->mt[k] = words[gen * 624 + k];
  if (threadIdx.x == 0) {
    st->idx = (int)idx;
    st->have_gauss = fin->have;
    st->gauss = fin->gauss;
  }
}

void noise_free(ps_handle* h) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (!n) return;
  auto fr = [](void* p) {
    if (p) cudaFree(p);
  };
  fr(n->d_rng);
  fr(n->d_fin);
  fr(n->words);
  fr(n->boff);
  if (n->h_rng) cudaFreeHost(n->h_rng);
  if (n->st) cudaStreamDestroy(n->st);
  if (n->ev_iter) cudaEventDestroy(n->ev_iter);
  if (n->ev_noise) cudaEventDestroy(n->ev_noise);
  delete n;
  h->noise_gen = nullptr;
}

int noise_setup(ps_handle* h) {
  NoiseState* n = new NoiseState();
  h->noise_gen = n;
  n->K = (long long)h->nf * h->N;
  // P accepted pairs take P / (pi / 4) attempts on average, with a standard
  // deviation of 0.59 sqrt(P); the margin is 10 sqrt(P) + 64.
  const long long P = (n->K + 1) / 2 + 1;
  const long long need =
      (long long)ceil((double)P / 0.7853981) + 10 * (long long)ceil(sqrt((double)P)) + 64;
  n->G = (int)((2 * need + 623) / 624);
  n->J = (long long)n->G * 312;
  n->nblk = (int)((n->J + kPairT - 1) / kPairT);
  PS_CUDA(h, cudaMalloc((void**)&n->d_rng, sizeof(DevRng)));
  PS_CUDA(h, cudaMemset(n->d_rng, 0, sizeof(DevRng)));
  PS_CUDA(h, cudaMallocHost((void**)&n->h_rng, sizeof(DevRng)));
  PS_CUDA(h, cudaMalloc((void**)&n->d_fin, sizeof(RngFinal)));
  PS_CUDA(h, cudaMalloc((void**)&n->words, sizeof(uint32_t) * (size_t)(n->G + 1) * 624));
  PS_CUDA(h, cudaMalloc((void**)&n->boff, sizeof(int) * (size_t)n->nblk));
  PS_CUDA(h, cudaStreamCreateWithFlags(&n->st, cudaStreamNonBlocking));
  PS_CUDA(h, cudaEventCreateWithFlags(&n->ev_iter, cudaEventDisableTiming));
  PS_CUDA(h, cudaEventCreateWithFlags(&n->ev_noise, cudaEventDisableTiming));
  return PS_OK;
}

// Copy the host generator to the device before the first device draw.
int noise_upload(ps_handle* h) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (!n || n->on_device) return PS_OK;
  bool hg = false;
  int idx = 0;
  double g = 0.0;
  memset(n->h_rng, 0, sizeof(DevRng));
  h->rng.get_state(n->h_rng->mt, &idx, &hg, &g);
  n->h_rng->idx = idx;
  n->h_rng->have_gauss = hg ? 1 : 0;
  n->h_rng->gauss = g;
  PS_CUDA(h, cudaMemcpyAsync(n->d_rng, n->h_rng, sizeof(DevRng), cudaMemcpyHostToDevice, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  n->on_device = true;
  return PS_OK;
}

// Bring the host generator up to date after device draws.  Every iterate call
// (alone or in a batch) returns with its work finished, so the stored state is
// the last iteration's.
int noise_download(ps_handle* h) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (!n || !n->on_device) return PS_OK;
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  PS_CUDA(h, cudaMemcpyAsync(n->h_rng, n->d_rng, sizeof(DevRng), cudaMemcpyDeviceToHost, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (n->h_rng->err) {
    h->err = "device noise: the stored generations ran short";
    return PS_RUN_ERR;
  }
  h->rng.set_state(n->h_rng->mt, n->h_rng->idx, n->h_rng->have_gauss != 0, n->h_rng->gauss);
  n->on_device = false;
  return PS_OK;
}

// Queue this iteration's nf * N Gaussians (times the noise strength) into
// h->d_noise on the generator's stream, forked from h->st; noise_join makes
// h->st wait for them.  Legal inside stream capture.
int noise_launch(ps_handle* h, long long* nlaunch) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (!n) return PS_OK;
  PS_CUDA(h, cudaEventRecord(n->ev_iter, h->st));
  PS_CUDA(h, cudaStreamWaitEvent(n->st, n->ev_iter, 0));
  rng_twist_kernel<<<1, kTwistT, 0, n->st>>>(n->d_rng, n->words, n->G);
  rng_count_kernel<<<n->nblk, kPairT, 0, n->st>>>(n->d_rng, n->words, n->J, n->boff, n->d_fin);
  rng_scan_kernel<<<1, kPairT, 0, n->st>>>(n->boff, n->nblk);
  rng_out_kernel<<<n->nblk, kPairT, 0, n->st>>>(n->d_rng, n->words, n->J, n->boff, n->K,
                                                 h->cfg.updater.noise, h->d_noise, n->d_fin);
  rng_final_kernel<<<1, kTwistT, 0, n->st>>>(n->d_rng, n->words, n->d_fin, n->K, n->G);
  PS_CUDA(h, cudaGetLastError());
  PS_CUDA(h, cudaEventRecord(n->ev_noise, n->st));
  *nlaunch += 5;
  return PS_OK;
}

int noise_join(ps_handle* h) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (n) PS_CUDA(h, cudaStreamWaitEvent(h->st, n->ev_noise, 0));
  return PS_OK;
}

// Error flag of the device generator, read with the iteration's status.
int noise_check(ps_handle* h) {
  NoiseState* n = static_cast<NoiseState*>(h->noise_gen);
  if (!n || !n->on_device) return PS_OK;
  PS_CUDA(h, cudaMemcpyAsync(&n->h_rng->err, &n->d_rng->err, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  PS_CUDA(h, cudaStreamSynchronize(h->st));
  if (n->h_rng->err) {
    h->err = "device noise: the stored generations ran short";
    return PS_RUN_ERR;
  }
  return PS_OK;
}

}  // namespace psb
