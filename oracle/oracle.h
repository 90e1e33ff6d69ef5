/*
 * oracle.h -- CPU FP64 restatement of PolySwift++'s SCFT inner loop.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this library, and only as the checker (or as the
 * timed CPU baseline); the product path never calls it.
 *
 * PARITY UNPINNED: the reference cannot be compiled here (its txbase/txutils
 * dependencies, FFTW 2, HDF5, Boost and MPI are absent) and it ships no golden
 * outputs.  This restatement follows the reference sources line by line (each
 * function cites file:line) and is pinned only by known-answer tests and by an
 * independent numpy restatement (numpy.fft, numpy's MT19937).
 */
#ifndef PSWIFT_ORACLE_H
#define PSWIFT_ORACLE_H

#include "../include/pswift.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_state oracle_state;

/* Threads used by the FFT and point loops (OpenMP); returns the count in use. */
int oracle_set_threads(int n);

/* MT19937 as psstd/PsRandom: init_genrand(seed), real() = u32 / 2^32,
 * polar Gaussian with one cached value. */
void oracle_mt_reals(unsigned long long seed, long n, double* out);
void oracle_mt_gauss(unsigned long long seed, long n, double* out);
void oracle_mt_u32(unsigned long long seed, long n, unsigned int* out);

/* Complex 3D FFT in place, FFTW sign convention (sign=-1 forward), unnormalised. */
void oracle_fft3d(const int n[3], double* re, double* im, int sign);

/* PsFFTW::scaledFFTPair: res = Re(IFFT(kdata*FFT(data))), c2c of real data. */
void oracle_scaled_fft_pair(const int n[3], const double* data, const double* kdata,
                            double* res);

/* The rest of PsFFTBase<T,3> as PsFFTW computes it in serial
 * (psfft/PsFFTW.cpp:122-297): |FFT|^2 (forwardFFTAbs), Re(IFFT(FFT(a)FFT(b)))
 * (convolveRe), Re(IFFT(kdata*FFT(i*data))) (scaledFFTPairIm), Re(FFT(data))
 * (calcForwardFFT) and Re(IFFT(data)) (calcBackwardFFT); unnormalised. */
void oracle_forward_fft_abs(const int n[3], const double* data, double* res);
void oracle_convolve_re(const int n[3], const double* data1, const double* data2, double* res);
void oracle_scaled_fft_pair_im(const int n[3], const double* data, const double* kdata,
                               double* res);
void oracle_calc_forward_fft(const int n[3], const double* data, double* res);
void oracle_calc_backward_fft(const int n[3], const double* data, double* res);

/* Build a whole SCFT instance (same checks as the device path). */
int oracle_create(const ps_config* cfg, oracle_state** out, char* err, int errlen);
void oracle_destroy(oracle_state* s);
int oracle_set_filter(oracle_state* s, const ps_filter_config* f);
void oracle_apply_filter(oracle_state* s);
int oracle_set_poisson(oracle_state* s, const ps_poisson_config* p);
int oracle_gauss_laguerre(int n, double a, double* x, double* w);
void oracle_apply_poisson(oracle_state* s);
int oracle_block_steps(const oracle_state* s, int polymer, int block);
void oracle_init_random(oracle_state* s);
void oracle_set_field(oracle_state* s, int which, int index, const double* data);
void oracle_get_field(const oracle_state* s, int which, int index, double* data);
/* Runs n iterations; writes one ps_scalars per iteration when hist != NULL.
 * Returns PS_OK or PS_RUN_ERR (non-finite Q). */
int oracle_iterate(oracle_state* s, int n, ps_scalars* hist);
void oracle_get_propagator(const oracle_state* s, int polymer, int block, int end,
                           int n, double* out);
/* The per-block k2 operator exp(-ds b^2 k^2) in normal (x,y,z) order. */
void oracle_get_k2(const oracle_state* s, int polymer, int block, double* out);

#ifdef __cplusplus
}
#endif

#endif
