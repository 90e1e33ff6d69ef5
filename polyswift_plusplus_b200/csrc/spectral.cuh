// Pieces shared by the updaters that run after the field update (spectral
// filters in filter.cu, the Poisson updater in poisson.cu): FP64 reductions
// over a field and its half spectrum, and twiddle tables.
#pragma once

#include <cuda_runtime.h>

namespace psb {

constexpr int kFT = 256;

// part[b] = block b's sum of w (is_max = 0) or max of |spec|^2 (is_max = 1).
__global__ void filter_sum_partials(const double* __restrict__ w, long long N, double* __restrict__ part,
                                    int is_max, const double2* __restrict__ spec);
// *out = max of the partials (is_max) or -(sum / N).
__global__ void filter_finalize(const double* __restrict__ part, int np, int is_max, double N,
                                double* __restrict__ out);
// w += *wtot
__global__ void filter_shift(double* __restrict__ w, long long N, const double* __restrict__ wtot);
// tw[m] = exp(-2 pi i m / L), L entries (1 when L = 0), in device memory.
cudaError_t twiddles64(double2** dst, int L);

}  // namespace psb
