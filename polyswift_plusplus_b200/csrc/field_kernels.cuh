// Field-level kernels (FP64 state, propagator slices in T) and their launchers.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/pswift.h"

namespace psb {

constexpr int kRedBlocks = 1184;  // 8 x 148 SMs; fixed so every reduction is deterministic
constexpr int kRedThreads = 256;

// Device-resident scalars of the current iteration.
struct DevScalars {
  double q[PS_MAX_POLYMERS];
  double log_q[PS_MAX_POLYMERS];
  double free_energy;
  double free_energy_nodis;
  double max_incomp;
  double dh_norm;
  double pressure_mean;
  long long iteration;
  int error_flags;
  int pad;
  // Anderson state
  long long am_k;       // Anderson iterations performed
  int am_nh;            // history terms used by the current mix
  int am_use;
  double am_c[64];      // solved coefficients
  double am_mix;        // mixing applied to the combined residual
  double solv_q[PS_MAX_SOLVENTS];  // simpleSolvent bigQ
};

// Static description of the field model handed to the update kernels.
struct FieldModel {
  int nf;
  int n_int;
  int int_a[PS_MAX_INTERACTIONS];
  int int_b[PS_MAX_INTERACTIONS];
  double chin[PS_MAX_INTERACTIONS];
  double dens_avg[PS_MAX_FIELDS];
  double lambda0, lambda1;
  int npol;
  double vf[PS_MAX_POLYMERS];
  double alpha[PS_MAX_POLYMERS];
  int nsolv;
  double solv_vf[PS_MAX_SOLVENTS];
  double scale_len;  // length of polymer 0 (a solvent's length ratio is 1 / scale_len)
  long long N;
};

struct FieldPtrs {
  double* w[PS_MAX_FIELDS];
  double* phi[PS_MAX_FIELDS];
  double* p;
  const double* noise;  // nf*N Gaussian increments (already scaled) or nullptr
};

// wfac = exp(ds2 * w) rounded to T.
template <typename T>
cudaError_t launch_wfac(const double* w, T* wfac, double ds2, long long N, cudaStream_t st);

// partials[b] = sum over the block's points of a*b (FP64).
template <typename T>
cudaError_t launch_dot_partials(const T* a, const T* b, long long N, double* partials,
                                cudaStream_t st);
// Q = sum(partials) / N for polymer ip; sets error flag on NaN.
cudaError_t launch_finalize_q(const double* partials, double N, int ip, DevScalars* sc,
                              cudaStream_t st);

// phi += densfac * Simpson(qs, qts) / Q  (pspolymer/PsBlock.cpp:255-380 + :153-196).
template <typename T>
cudaError_t launch_quadrature(const T* qs, const T* qts, int steps, long long N, double ds,
                              double densfac, const DevScalars* sc, int ip, double* phi,
                              cudaStream_t st);

cudaError_t launch_zero(double* p, long long n, cudaStream_t st);

// Junction of a branched polymer (PsBlock::combineSetJnt): out = 1 * q_0 * q_1 * ...
// over the final slices of the blocks joined there, in ascending block order.
template <typename T> struct JunctionIn {
  const T* q[PS_MAX_JOINS];
  int n;
};
template <typename T>
cudaError_t launch_junction(const JunctionIn<T>& in, long long N, T* out, cudaStream_t st);

// simpleSolvent (pssolvent/PsSimpleSolvent.cpp:86-140): Q = <exp(-w/L)> into
// sc->solv_q[is], then phi += (volfrac / Q) exp(-w/L).
cudaError_t launch_solvent(const double* w, double neg_inv_len, double volfrac, long long N, int is,
                           double* partials, DevScalars* sc, double* phi, cudaStream_t st);

// chargeFlexPseudoSpec: wfac = exp(ds2 w) exp(facz ds2 psi) rounded to T.
template <typename T>
cudaError_t launch_wfac_charged(const double* w, const double* psi, T* wfac, double ds2, double facz,
                                long long N, cudaStream_t st);

// simpleIons (pssolvent/PsSimpleIons.cpp:90-160): Q = <exp(-zc psi)> into
// sc->solv_q[is]; e = exp(-zc psi) (-neutral_factor / (Q zc)); block_rho = e
// (when not null); rho += zc e.
cudaError_t launch_ions(const double* psi, double zc, double neutral_factor, long long N, int is,
                        double* partials, DevScalars* sc, double* rho, double* block_rho,
                        cudaStream_t st);

// rho += (phi alpha) za after a charged block's density.
cudaError_t launch_charge_accum(const double* phi, double alpha, double za, long long N, double* rho,
                                cudaStream_t st);

// Steepest-descent update, pressure rebuild and free-energy partial sums.
cudaError_t launch_sd_update(const FieldModel& fm, const FieldPtrs& fp, double* partials,
                             cudaStream_t st);
// Anderson: residual + history store, Gram row, solve, mix (+ pressure / F partials).
cudaError_t launch_am_residual(const FieldModel& fm, const FieldPtrs& fp, double* hist_w,
                               double* hist_d, int slots, DevScalars* sc, double* partials,
                               cudaStream_t st);
cudaError_t launch_am_gram(long long nfN, const double* hist_d, int slots, int m, DevScalars* sc,
                           double* gram_partials, cudaStream_t st);
cudaError_t launch_am_solve(const double* gram_partials, double* gram, int slots, int m,
                            int start, double mix, double lambda0, DevScalars* sc,
                            cudaStream_t st);
cudaError_t launch_am_mix(const FieldModel& fm, const FieldPtrs& fp, const double* hist_w,
                          const double* hist_d, int slots, DevScalars* sc, double* partials,
                          cudaStream_t st);
// Reduce the update partials into DevScalars (F, mean p, diagnostics); iteration++.
cudaError_t launch_update_finalize(const FieldModel& fm, const double* partials, DevScalars* sc,
                                   cudaStream_t st);
cudaError_t launch_update_finalize_am(const FieldModel& fm, const double* partials,
                                      DevScalars* sc, cudaStream_t st);
// p -= mean(p)
cudaError_t launch_pressure_shift(double* p, long long N, const DevScalars* sc, cudaStream_t st);

// Number of partial-sum slots per reduction block used by the update kernels.
constexpr int kUpdQ = 6;  // sum p, sum fe, sum fe_nodis, sum dH^2, max incompressibility, spare

}  // namespace psb
