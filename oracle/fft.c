/*
 * Mixed-radix complex FFT for the oracle (TEST INFRASTRUCTURE).
 *
 * Stands in for FFTW 2.x as called by PsFFTW (psfft/PsFFTW.cpp:71-75 plans,
 * :196-224 scaledFFTPair): complex-to-complex transforms of real data with the
 * imaginary part set to zero, forward sign -1, backward sign +1, neither
 * normalised.  FFTW 2 itself is not vendored in the reference tree and its
 * version is not pinned; this is a Stockham autosort FFT written from the
 * published algorithm, checked against numpy.fft in tests.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

typedef struct fft_plan1d {
  int n;
  int nf;
  int f[40];
  double* tw; /* exp(-2 pi i m / n), m = 0..n-1, interleaved re/im */
} fft_plan1d;

static void plan_init(fft_plan1d* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
  while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
  while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
  for (int q = 7; m > 1; q += 2) {
    while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
  }
  p->tw = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  const double twopi = 2.0 * acos(-1.0);
  for (int k = 0; k < n; ++k) {
    double a = twopi * (double)k / (double)n;
    p->tw[2 * k] = cos(a);
    p->tw[2 * k + 1] = -sin(a);
  }
}

static void plan_free(fft_plan1d* p) { free(p->tw); }

/* One Stockham pass: radix R, Ns = product of the previous radices. */
static void pass(const fft_plan1d* p, int R, int Ns, const double* x, double* y, int sign) {
  const int n = p->n;
  const int m = n / R;
  const int tstride = n / (Ns * R);
  double vr[64], vi[64], ur[64], ui[64];
  for (int j = 0; j < m; ++j) {
    const int k = j % Ns;
    for (int r = 0; r < R; ++r) {
      double a = x[2 * (j + r * m)], b = x[2 * (j + r * m) + 1];
      int ti = (r * k * tstride) % n;
      double c = p->tw[2 * ti], s = p->tw[2 * ti + 1];
      if (sign > 0) s = -s;
      vr[r] = a * c - b * s;
      vi[r] = a * s + b * c;
    }
    if (R == 2) {
      ur[0] = vr[0] + vr[1]; ui[0] = vi[0] + vi[1];
      ur[1] = vr[0] - vr[1]; ui[1] = vi[0] - vi[1];
    } else if (R == 4) {
      double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
      double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
      double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
      double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
      /* forward: y1 = d0 - i d1, y3 = d0 + i d1 */
      double jr = (sign < 0) ? d1i : -d1i;
      double ji = (sign < 0) ? -d1r : d1r;
      ur[0] = s0r + s1r; ui[0] = s0i + s1i;
      ur[2] = s0r - s1r; ui[2] = s0i - s1i;
      ur[1] = d0r + jr;  ui[1] = d0i + ji;
      ur[3] = d0r - jr;  ui[3] = d0i - ji;
    } else {
      /* generic DFT of length R using the plan's twiddle table */
      const int step = n / R;
      for (int q = 0; q < R; ++q) {
        double sr = 0.0, si = 0.0;
        for (int r = 0; r < R; ++r) {
          int ti = ((q * r) % R) * step;
          double c = p->tw[2 * ti], s = p->tw[2 * ti + 1];
          if (sign > 0) s = -s;
          sr += vr[r] * c - vi[r] * s;
          si += vr[r] * s + vi[r] * c;
        }
        ur[q] = sr;
        ui[q] = si;
      }
    }
    const int d = (j / Ns) * Ns * R + k;
    for (int r = 0; r < R; ++r) {
      y[2 * (d + r * Ns)] = ur[r];
      y[2 * (d + r * Ns) + 1] = ui[r];
    }
  }
}

/* In-place transform of a contiguous complex vector (work: 2n doubles). */
static void exec1d(const fft_plan1d* p, double* x, double* work, int sign) {
  if (p->n <= 1) return;
  double* a = x;
  double* b = work;
  int Ns = 1;
  for (int i = 0; i < p->nf; ++i) {
    pass(p, p->f[i], Ns, a, b, sign);
    Ns *= p->f[i];
    double* t = a; a = b; b = t;
  }
  if (a != x) memcpy(x, a, sizeof(double) * 2 * (size_t)p->n);
}

/* Transform a 3D complex array (interleaved) along one axis. */
static void fft_axis(const int n[3], double* c, int axis, int sign) {
  const int len = n[axis];
  if (len <= 1) return;
  fft_plan1d plan;
  plan_init(&plan, len);
  long stride = (axis == 2) ? 1 : (axis == 1 ? n[2] : (long)n[1] * n[2]);
  long npencil = ((long)n[0] * n[1] * n[2]) / len;
#pragma omp parallel
  {
    double* buf = (double*)malloc(sizeof(double) * 4 * (size_t)len);
    double* work = buf + 2 * len;
#pragma omp for schedule(static)
    for (long pi = 0; pi < npencil; ++pi) {
      long base;
      if (axis == 2) {
        base = pi * len;
      } else if (axis == 1) {
        long x = pi / n[2], z = pi % n[2];
        base = x * (long)n[1] * n[2] + z;
      } else {
        base = pi; /* (y,z) flattened */
      }
      for (int i = 0; i < len; ++i) {
        buf[2 * i] = c[2 * (base + i * stride)];
        buf[2 * i + 1] = c[2 * (base + i * stride) + 1];
      }
      exec1d(&plan, buf, work, sign);
      for (int i = 0; i < len; ++i) {
        c[2 * (base + i * stride)] = buf[2 * i];
        c[2 * (base + i * stride) + 1] = buf[2 * i + 1];
      }
    }
    free(buf);
  }
  plan_free(&plan);
}

/* fftwnd_one on an interleaved complex array, FFTW sign convention. */
void oracle_fftnd_inplace(const int n[3], double* c, int sign) {
  fft_axis(n, c, 2, sign);
  fft_axis(n, c, 1, sign);
  fft_axis(n, c, 0, sign);
}

void oracle_fft3d(const int n[3], double* re, double* im, int sign) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
  for (long i = 0; i < N; ++i) { c[2 * i] = re[i]; c[2 * i + 1] = im[i]; }
  oracle_fftnd_inplace(n, c, sign);
  for (long i = 0; i < N; ++i) { re[i] = c[2 * i]; im[i] = c[2 * i + 1]; }
  free(c);
}

/* PsFFTW::scaledFFTPair, serial branch (psfft/PsFFTW.cpp:196-224). */
void oracle_scaled_pair_buf(const int n[3], const double* data, const double* kdata,
                            double* res, double* c) {
  long N = (long)n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] = data[i]; c[2 * i + 1] = 0.0; }
  oracle_fftnd_inplace(n, c, -1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] *= kdata[i]; c[2 * i + 1] *= kdata[i]; }
  oracle_fftnd_inplace(n, c, +1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) res[i] = c[2 * i];
}

void oracle_scaled_fft_pair(const int n[3], const double* data, const double* kdata,
                            double* res) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
  oracle_scaled_pair_buf(n, data, kdata, res, c);
  free(c);
}

/* The other transforms of PsFFTBase<T,3> (psbase/PsFFTBase.h:83-134), serial
 * branch of PsFFTW (psfft/PsFFTW.cpp): each packs its real input into the
 * complex work array, runs the unnormalised c2c FFTW-sign transforms and keeps
 * what the reference keeps. */

/* PsFFTW::forwardFFTAbs (psfft/PsFFTW.cpp:122-149): res = re^2 + im^2 of the
 * forward transform (the squared modulus, as the reference computes it). */
void oracle_forward_fft_abs(const int n[3], const double* data, double* res) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] = data[i]; c[2 * i + 1] = 0.0; }
  oracle_fftnd_inplace(n, c, -1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) res[i] = (c[2 * i] * c[2 * i]) + (c[2 * i + 1] * c[2 * i + 1]);
  free(c);
}

/* PsFFTW::convolveRe (psfft/PsFFTW.cpp:150-189): both inputs forward, the
 * complex product, backward, real part. */
void oracle_convolve_re(const int n[3], const double* data1, const double* data2, double* res) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
  double* c2 = (double*)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) {
    c[2 * i] = data1[i]; c[2 * i + 1] = 0.0;
    c2[2 * i] = data2[i]; c2[2 * i + 1] = 0.0;
  }
  oracle_fftnd_inplace(n, c, -1);
  oracle_fftnd_inplace(n, c2, -1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) {
    const double ar = c[2 * i], ai = c[2 * i + 1], br = c2[2 * i], bi = c2[2 * i + 1];
    c[2 * i] = (ar * br) - (ai * bi);
    c[2 * i + 1] = (ai * br) + (ar * bi);
  }
  oracle_fftnd_inplace(n, c, +1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) res[i] = c[2 * i];
  free(c2);
  free(c);
}

/* PsFFTW::scaledFFTPairIm (psfft/PsFFTW.cpp:227-257): the input is the
 * imaginary part, the transform is scaled by the real kdata, real part kept. */
void oracle_scaled_fft_pair_im(const int n[3], const double* data, const double* kdata,
                               double* res) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] = 0.0; c[2 * i + 1] = data[i]; }
  oracle_fftnd_inplace(n, c, -1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] *= kdata[i]; c[2 * i + 1] *= kdata[i]; }
  oracle_fftnd_inplace(n, c, +1);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) res[i] = c[2 * i];
  free(c);
}

/* PsFFTW::calcForwardFFT / calcBackwardFFT (psfft/PsFFTW.cpp:260-297): the real
 * part of the forward (sign -1) or backward (sign +1) transform of real data. */
static void real_part_of_transform(const int n[3], const double* data, double* res, int sign) {
  long N = (long)n[0] * n[1] * n[2];
  double* c = (double*)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) { c[2 * i] = data[i]; c[2 * i + 1] = 0.0; }
  oracle_fftnd_inplace(n, c, sign);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) res[i] = c[2 * i];
  free(c);
}

void oracle_calc_forward_fft(const int n[3], const double* data, double* res) {
  real_part_of_transform(n, data, res, -1);
}

void oracle_calc_backward_fft(const int n[3], const double* data, double* res) {
  real_part_of_transform(n, data, res, +1);
}

int oracle_set_threads(int nt) {
#ifdef _OPENMP
  if (nt > 0) omp_set_num_threads(nt);
  return omp_get_max_threads();
#else
  (void)nt;
  return 1;
#endif
}
