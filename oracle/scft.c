/*
 * FP64 CPU restatement of the PolySwift++ SCFT inner loop (TEST INFRASTRUCTURE).
 *
 * PARITY UNPINNED: the reference cannot be built here and ships no golden
 * data; this file restates its algorithm from the sources and is checked by
 * known-answer tests and an independent numpy restatement.  It is loaded only
 * by tests, by the smoke check and by the benchmark's CPU-baseline leg.
 *
 * One update(t) follows pstrol/PsDomain.cpp:332-372:
 *   phi_i = 0                                   psphysf/PsMonomerDens.cpp:105-110,167-171
 *   PsBlockCopolymer::update                    pspolymer/PsBlockCopolymer.cpp:189-239
 *     reset: wfac = exp(-ds/2 w)                pspolymer/PsFlexPseudoSpec.cpp:158-181
 *     dependency-driven solveQ / publishQFrom   pspolymer/PsBlockCopolymer.cpp:248-313
 *     solveQ step loop                          pspolymer/PsFlexPseudoSpec.cpp:244-293
 *     Q = <qHeadInitial qHeadFinal>             pspolymer/PsBlock.cpp:205-237
 *     Simpson (0.33333) + trapezoid tail        pspolymer/PsBlock.cpp:256-380
 *     phi += vf/alpha * qqt                     pspolymer/PsBlock.cpp:154-196
 *   PsSteepDUpdater::update                     pseffhamil/PsSteepDUpdater.cpp:159-203
 *     dH_i = p - w_i + sum chiN(phi_j - avg_j)  :174-184, :208-236,
 *                                               pseffhamil/PsFloryInteraction.cpp:204-269
 *     w update, noise, pressure (2 / 3 fields)  :250-333, :350-453,
 *                                               pseffhamil/PsPolymerUpdater.cpp:244-295
 *     p -= mean(p)                              psphysf/PsConstraint.cpp:184-262
 *     F with the updated w                      pseffhamil/PsPolymerUpdater.cpp:173-226,303-341,
 *                                               pseffhamil/PsFloryInteraction.cpp:275-321
 * Bulk systems only: the constraint field phi0 is identically zero (no walls
 * or particles), so every mask is 1 and every volume is N.
 *
 * Anderson mixing has no counterpart in the reference; it is restated here
 * from the published method (D. G. Anderson 1965; as used for SCFT by
 * R. B. Thompson et al. 2004 and M. W. Matsen 2009) in exactly the form the
 * device updater uses (Gram-matrix normal equations, partial-pivot solve).
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mt19937.h"
#include "oracle.h"

void oracle_fftnd_inplace(const int n[3], double* c, int sign);
void oracle_scaled_pair_buf(const int n[3], const double* data, const double* kdata,
                            double* res, double* c);

enum { HEAD = 0, TAIL = 1 };

/* blocks per polymer here: a polyDisperseBCP has n_g quadrature copies of each seed block */
#define OMAX_BLOCKS 64

typedef struct oblock {
  ps_block_config cfg;
  int steps;
  /* connections: index of the joined block and the joined end of that block */
  int ncnt[2];
  int cnt_idx[2][PS_MAX_JOINS];
  int cnt_end[2][PS_MAX_JOINS];
  /* junction maps keyed by the joined block index (std::map order = ascending) */
  int njnt[2];
  int jnt_key[2][PS_MAX_JOINS];
  int jnt_set[2][PS_MAX_JOINS];
  double* jnt_q[2][PS_MAX_JOINS];
  double* q_init[2];
  double* q_final[2];
  int init_set[2];
  int final_set[2];
  double* qs;  /* solved from HEAD: (steps+1) slices */
  double* qts; /* solved from TAIL */
  double* wfac;
  double* k2;
  double* qqt;
} oblock;

typedef struct opolymer {
  ps_polymer_config cfg;
  double length_ratio;
  int nb;
  oblock b[OMAX_BLOCKS];
  double bigq;
  double logq;                 /* getLogBigQ */
  /* polyDisperseBCP (pspolymer/PsPolyDisperseBCP.cpp): quadrature blocks seed-major */
  int pd, n_g, n_seed, poly_block;
  double galpha;               /* Gamma(alpha) */
  double gw[OMAX_BLOCKS];      /* Gauss-Laguerre weights w_k */
  double lwt[OMAX_BLOCKS];     /* lengthWeight of each block */
  double dwt[OMAX_BLOCKS];     /* densityWeight of each block */
  double bq[OMAX_BLOCKS];      /* per-block calcBigQ */
} opolymer;

/* n-point generalized Gauss-Laguerre rule (weight x^a e^-x): the roots of
 * L_n^(a) are bracketed on a grid quadratic in x, bisected, and the weights
 * are Gamma(n + a + 1) / (n! x_i L_n^(a)'(x_i)^2).  L by the three-term
 * recurrence, x L_n' = n L_n - (n + a) L_{n-1}. */
static double laguerre(int n, double a, double x, double* dl) {
  double p0 = 1.0, p1 = 1.0 + a - x;
  if (n == 0) { *dl = 0.0; return 1.0; }
  for (int j = 1; j < n; ++j) {
    const double p2 = ((2.0 * j + 1.0 + a - x) * p1 - (j + a) * p0) / (j + 1.0);
    p0 = p1;
    p1 = p2;
  }
  *dl = (n * p1 - (n + a) * p0) / x;
  return p1;
}

int oracle_gauss_laguerre(int n, double a, double* x, double* w);
static int gauss_laguerre(int n, double a, double* x, double* w) { return oracle_gauss_laguerre(n, a, x, w); }
int oracle_gauss_laguerre(int n, double a, double* x, double* w) {
  if (n < 1 || n > 64 || !(a > -1.0)) return PS_ATTRIB_ERR;
  const double X = 4.0 * n + 2.0 * a + 10.0;
  const long M = 200000;
  double dl, xa = 0.0, fa = 1.0;  /* L_n^(a)(0) > 0 */
  int found = 0;
  for (long i = 1; i <= M && found < n; ++i) {
    const double t = (double)i / (double)M;
    const double xb = X * t * t;
    const double fb = laguerre(n, a, xb, &dl);
    if ((fa > 0.0) != (fb > 0.0)) {
      double lo = xa, hi = xb, flo = fa;
      for (int it = 0; it < 200 && hi - lo > 0.0; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        const double fm = laguerre(n, a, mid, &dl);
        if ((fm > 0.0) == (flo > 0.0)) { lo = mid; flo = fm; } else { hi = mid; }
      }
      x[found++] = 0.5 * (lo + hi);
    }
    xa = xb;
    fa = fb;
  }
  if (found != n) return PS_ATTRIB_ERR;
  const double c = exp(lgamma(n + a + 1.0) - lgamma(n + 1.0));
  for (int i = 0; i < n; ++i) {
    laguerre(n, a, x[i], &dl);
    w[i] = c / (x[i] * dl * dl);
  }
  return PS_OK;
}

struct oracle_state {
  ps_config cfg;
  int n[3];
  long N;
  int nf;
  double* w[PS_MAX_FIELDS];
  double* phi[PS_MAX_FIELDS];
  double* p;
  double dens_avg[PS_MAX_FIELDS];
  double chin[PS_MAX_INTERACTIONS];
  int npol;
  opolymer pol[PS_MAX_POLYMERS];
  double scale_length;
  double solv_q[PS_MAX_SOLVENTS];  /* simpleSolvent bigQ of the last iteration */
  int has_filter;                  /* simpleSpecFilter updater after the field update */
  ps_filter_config fcfg;
  double* fpow;                    /* N: |FFT(w)|^2, then the mask */
  double* fcut;                    /* multiSpecFilter: max power per region */
  long* fregion;                   /* multiSpecFilter: region of each spectrum index */
  long fncells;
  /* chargeDens PhysFields: charge density and electric potential */
  int nq;
  double* rho[PS_MAX_CHARGES];
  double* psi[PS_MAX_CHARGES];
  int has_poisson;                 /* poissonUpdater after the field update */
  ps_poisson_config pcfg;
  double* kcoul;                   /* N: 4 (3.1415) lB / |k|^2, 0 at |k|^2 < 1e-9 */
  int post[2];                     /* post-update updaters in run order: 1 filter, 2 Poisson */
  int npost;
  mt_state rng;
  long long iter;
  /* scratch */
  double* cwork;  /* 2N complex scratch for the FFT pair */
  double* qw;
  double* res;
  double* dh[PS_MAX_FIELDS];
  /* Anderson history (ring of depth m+1) */
  int am_m;
  double* am_w;   /* (m+1) * nf * N */
  double* am_d;   /* (m+1) * nf * N */
  double* am_g;   /* (m+1)^2 Gram matrix indexed by ring slots */
  long long am_k;
  /* wall time of the last iteration: propagator sweeps and total (seconds) */
  double t_sweeps;
  double t_total;
};

#include <time.h>
static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void* xcalloc(size_t n, size_t sz) {
  void* p = calloc(n ? n : 1, sz);
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

/* PsBlockBase::setBlockSteps (psbase/PsBlockBase.cpp:252-326). */
static int set_block_steps(double bs, int force, int* out, char* err, int errlen) {
  long bsint;
  double intpart = (double)((long)bs);
  double dx = bs - intpart;
  if (force) {
    bsint = (long)floor(bs + 0.5);
  } else {
    if ((dx > 0.0001) && (dx < 0.9999)) {
      snprintf(err, errlen, "non-integer # of block steps: blockSteps = %.17g", bs);
      return PS_INPUT_ERR;
    }
    long c = (long)ceil(bs), f = (long)floor(bs);
    if (c == f) bsint = c;
    else if (fabs(bs - (double)c) < fabs(bs - (double)f)) bsint = c;
    else bsint = f;
  }
  if (bsint < 4) {
    snprintf(err, errlen, "# of block steps too small: %ld < 4", bsint);
    return PS_INPUT_ERR;
  }
  *out = (int)bsint;
  return PS_OK;
}

/* Charge attributes of block ib of polymer ip (a quadrature block copies its seed's). */
static const ps_block_charge* block_charge_of(const oracle_state* s, int ip, int ib) {
  const opolymer* P = &s->pol[ip];
  const int seed = P->pd ? ib / P->n_g : ib;
  return &s->cfg.block_charge[ip][seed];
}

/* PsGridField::calck2 (psbase/PsGridField.cpp:66-104): |k|^2 at grid index (i, j, k). */
static double calck2(const oracle_state* s, int i, int j, int k) {
  const double twopi = 2.0 * acos(-1.0);
  double n2[3];
  for (int d = 0; d < 3; ++d) n2[d] = (double)s->n[d] / 2.0;
  double nk2 = n2[2] - fabs((double)k - n2[2]);
  double nk1 = n2[1] - fabs((double)j - n2[1]);
  double nk0 = n2[0] - fabs((double)i - n2[0]);
  double kv2 = twopi * nk2 / (double)s->n[2];
  double kv1 = twopi * nk1 / (double)s->n[1];
  double kv0 = twopi * nk0 / (double)s->n[0];
  kv2 = kv2 / s->cfg.cell[2];
  kv1 = kv1 / s->cfg.cell[1];
  kv0 = kv0 / s->cfg.cell[0];
  return kv0 * kv0 + kv1 * kv1 + kv2 * kv2;
}

/* PsFlexPseudoSpec::build_k2 (pspolymer/PsFlexPseudoSpec.cpp:188-206). */
static void build_k2(const oracle_state* s, const oblock* b, double* k2) {
  long idx = 0;
  for (int i = 0; i < s->n[0]; ++i)
    for (int j = 0; j < s->n[1]; ++j)
      for (int k = 0; k < s->n[2]; ++k) {
        double k2val = calck2(s, i, j, k);
        k2[idx++] = exp(-1.0 * b->cfg.ds * k2val * b->cfg.bseg_ratio * b->cfg.bseg_ratio);
      }
}

int oracle_create(const ps_config* cfg, oracle_state** out, char* err, int errlen) {
  char dummy[8];
  if (!err) { err = dummy; errlen = (int)sizeof(dummy); }
  *out = NULL;
  if (cfg->n_fields < 2 || cfg->n_fields > 3) {
    snprintf(err, errlen, "n_fields must be 2 or 3 (PsSteepDUpdater supports 2 or 3)");
    return PS_ATTRIB_ERR;
  }
  if (cfg->n_polymers < 1 || cfg->n_polymers > PS_MAX_POLYMERS) {
    snprintf(err, errlen, "n_polymers out of range");
    return PS_ATTRIB_ERR;
  }
  oracle_state* s = (oracle_state*)xcalloc(1, sizeof(oracle_state));
  s->cfg = *cfg;
  for (int d = 0; d < 3; ++d) s->n[d] = cfg->n[d];
  s->N = (long)cfg->n[0] * cfg->n[1] * cfg->n[2];
  s->nf = cfg->n_fields;
  long N = s->N;
  for (int i = 0; i < s->nf; ++i) {
    s->w[i] = (double*)xcalloc((size_t)N, sizeof(double));
    s->phi[i] = (double*)xcalloc((size_t)N, sizeof(double));
    s->dh[i] = (double*)xcalloc((size_t)N, sizeof(double));
  }
  s->p = (double*)xcalloc((size_t)N, sizeof(double));
  s->cwork = (double*)xcalloc((size_t)(2 * N), sizeof(double));
  s->qw = (double*)xcalloc((size_t)N, sizeof(double));
  s->res = (double*)xcalloc((size_t)N, sizeof(double));
  /* scaleLength = length of the first polymer (pspolymer/PsPolymerHldr.cpp:67-83) */
  s->scale_length = (double)cfg->polymers[0].length;
  s->npol = cfg->n_polymers;
  int rc = PS_OK;
  for (int ip = 0; ip < s->npol && rc == PS_OK; ++ip) {
    opolymer* P = &s->pol[ip];
    P->cfg = cfg->polymers[ip];
    P->nb = P->cfg.n_blocks;
    P->length_ratio = (double)P->cfg.length / s->scale_length;
    if (P->nb < 1 || P->nb > PS_MAX_BLOCKS) {
      snprintf(err, errlen, "polymer %d: n_blocks out of range", ip);
      rc = PS_ATTRIB_ERR;
      break;
    }
    const ps_polydisperse_config* D = &cfg->polydisperse[ip];
    for (int ib = 0; ib < OMAX_BLOCKS; ++ib) P->lwt[ib] = P->dwt[ib] = 1.0;
    if (D->enabled) {
      /* PsPolyDisperseBCP::setAttrib / calcPolyParams / makeQuadAttrib
       * (pspolymer/PsPolyDisperseBCP.cpp:41-145, 384-455, 495-600) */
      if (P->nb > 2 || D->poly_block < 0 || D->poly_block >= P->nb || D->n_g < 1 ||
          D->n_g * P->nb > OMAX_BLOCKS || !(D->alpha > 0.0)) {
        snprintf(err, errlen, "polymer %d: bad polyDisperseBCP (at most 2 blocks)", ip);
        rc = PS_ATTRIB_ERR;
        break;
      }
      double xg[64];
      if (gauss_laguerre(D->n_g, D->alpha - 1.0, xg, P->gw) != PS_OK) {
        snprintf(err, errlen, "polymer %d: Gauss-Laguerre rule failed", ip);
        rc = PS_ATTRIB_ERR;
        break;
      }
      P->pd = 1;
      P->n_g = D->n_g;
      P->n_seed = P->nb;
      P->poly_block = D->poly_block;
      P->galpha = tgamma(D->alpha);
      const double nlen = (double)P->cfg.length;
      const double poly_frac = P->cfg.blocks[D->poly_block].lengthfrac;
      const double const_frac = 1.0 - poly_frac;
      const double ncl = const_frac * nlen;
      const double n_b = (nlen - ncl) / D->alpha;
      for (int sb = 0; sb < P->n_seed; ++sb)
        for (int k = 0; k < P->n_g; ++k) {
          const int q = sb * P->n_g + k;
          ps_block_config bc = P->cfg.blocks[sb];
          for (int j = 0; j < bc.n_head; ++j) bc.head_joined[j] = bc.head_joined[j] * P->n_g + k;
          for (int j = 0; j < bc.n_tail; ++j) bc.tail_joined[j] = bc.tail_joined[j] * P->n_g + k;
          if (sb == D->poly_block) {
            bc.lengthfrac = ((xg[k] * n_b + ncl) / nlen) - const_frac;
            P->lwt[q] = P->gw[k] / P->galpha;
          } else {
            P->lwt[q] = 1.0 / (double)P->n_g;
          }
          P->dwt[q] = P->gw[k] / P->galpha;
          P->b[q].cfg = bc;
        }
      P->nb = P->n_seed * P->n_g;
      double tot = 0.0;
      for (int ib = 0; ib < P->nb; ++ib) tot = tot + (P->b[ib].cfg.lengthfrac * P->lwt[ib]);
      if (fabs(tot - 1.0) > 0.00001) {
        snprintf(err, errlen, "polymer %d: PsPolyDisperseBCP |totalFrac - 1.0| > tolerance", ip);
        rc = PS_INPUT_ERR;
        break;
      }
    } else {
      /* |sum f - 1| <= 1e-5 (pspolymer/PsBlockCopolymer.cpp:113-127) */
      double tot = 0.0;
      for (int ib = 0; ib < P->nb; ++ib) tot = tot + P->cfg.blocks[ib].lengthfrac;
      if (fabs(tot - 1.0) > 0.00001) {
        snprintf(err, errlen, "polymer %d: |totalFrac - 1.0| = %g > tolerance", ip, fabs(tot - 1.0));
        rc = PS_INPUT_ERR;
        break;
      }
      for (int ib = 0; ib < P->nb; ++ib) P->b[ib].cfg = P->cfg.blocks[ib];
    }
    for (int ib = 0; ib < P->nb && rc == PS_OK; ++ib) {
      oblock* B = &P->b[ib];
      if (B->cfg.field < 0 || B->cfg.field >= s->nf) {
        snprintf(err, errlen, "polymer %d block %d: field index out of range", ip, ib);
        rc = PS_ATTRIB_ERR;
        break;
      }
      if (!(B->cfg.ds > 0.0)) {
        snprintf(err, errlen, "polymer %d block %d: ds not set", ip, ib);
        rc = PS_ATTRIB_ERR;
        break;
      }
      /* psbase/PsBlockBase.cpp:187-198 */
      s->dens_avg[B->cfg.field] = s->dens_avg[B->cfg.field] + P->lwt[ib] * B->cfg.lengthfrac * P->cfg.volfrac;
      double bstmp = P->length_ratio * B->cfg.lengthfrac / B->cfg.ds;
      char e2[200];
      rc = set_block_steps(bstmp, B->cfg.force_block_steps, &B->steps, e2, sizeof(e2));
      if (rc != PS_OK) {
        snprintf(err, errlen, "polymer %d block %d: %s", ip, ib, e2);
        break;
      }
      B->qs = (double*)xcalloc((size_t)(B->steps + 1) * N, sizeof(double));
      B->qts = (double*)xcalloc((size_t)(B->steps + 1) * N, sizeof(double));
      B->wfac = (double*)xcalloc((size_t)N, sizeof(double));
      B->k2 = (double*)xcalloc((size_t)N, sizeof(double));
      B->qqt = (double*)xcalloc((size_t)N, sizeof(double));
      for (int e = 0; e < 2; ++e) {
        B->q_init[e] = (double*)xcalloc((size_t)N, sizeof(double));
        B->q_final[e] = (double*)xcalloc((size_t)N, sizeof(double));
      }
    }
    if (rc != PS_OK) break;
    /* setCntToLists (psbase/PsBlockBase.cpp:214-245) */
    for (int ib = 0; ib < P->nb && rc == PS_OK; ++ib) {
      oblock* B = &P->b[ib];
      B->ncnt[HEAD] = B->cfg.n_head;
      B->ncnt[TAIL] = B->cfg.n_tail;
      for (int e = 0; e < 2; ++e) {
        const int* lst = (e == HEAD) ? B->cfg.head_joined : B->cfg.tail_joined;
        for (int c = 0; c < B->ncnt[e]; ++c) {
          if (lst[c] < 0 || lst[c] >= P->nb) {
            snprintf(err, errlen, "polymer %d block %d: joined block index out of range", ip, ib);
            rc = PS_ATTRIB_ERR;
          }
          B->cnt_idx[e][c] = lst[c];
          B->cnt_end[e][c] = HEAD;
        }
        /* junction map in ascending key order */
        int keys[PS_MAX_JOINS];
        int nk = 0;
        for (int c = 0; c < B->ncnt[e]; ++c) {
          int key = lst[c], dup = 0;
          for (int t = 0; t < nk; ++t) dup |= (keys[t] == key);
          if (!dup) keys[nk++] = key;
        }
        for (int a = 0; a < nk; ++a)
          for (int c = a + 1; c < nk; ++c)
            if (keys[c] < keys[a]) { int t = keys[a]; keys[a] = keys[c]; keys[c] = t; }
        B->njnt[e] = nk;
        for (int a = 0; a < nk; ++a) {
          B->jnt_key[e][a] = keys[a];
          B->jnt_q[e][a] = (double*)xcalloc((size_t)N, sizeof(double));
        }
      }
    }
    /* buildCntBlockType (pspolymer/PsBlockCopolymer.cpp:157-182) */
    for (int ib = 0; ib < P->nb; ++ib) {
      for (int e = 0; e < 2; ++e) {
        oblock* B = &P->b[ib];
        for (int c = 0; c < B->ncnt[e]; ++c) {
          int j = B->cnt_idx[e][c];
          oblock* J = &P->b[j];
          for (int t = 0; t < J->ncnt[TAIL]; ++t)
            if (J->cnt_idx[TAIL][t] == ib) B->cnt_end[e][c] = TAIL;
        }
      }
    }
    for (int ib = 0; ib < P->nb; ++ib) build_k2(s, &P->b[ib], P->b[ib].k2);
  }
  if (rc == PS_OK && (cfg->n_solvents < 0 || cfg->n_solvents > PS_MAX_SOLVENTS)) {
    snprintf(err, errlen, "n_solvents out of range");
    rc = PS_ATTRIB_ERR;
  }
  if (rc == PS_OK && (cfg->n_charges < 0 || cfg->n_charges > PS_MAX_CHARGES)) {
    snprintf(err, errlen, "n_charges out of range");
    rc = PS_ATTRIB_ERR;
  }
  if (rc == PS_OK) {
    s->nq = cfg->n_charges;
    for (int c = 0; c < s->nq; ++c) {
      s->rho[c] = (double*)xcalloc((size_t)N, sizeof(double));
      s->psi[c] = (double*)xcalloc((size_t)N, sizeof(double));
    }
  }
  for (int is = 0; is < cfg->n_solvents && rc == PS_OK; ++is) {
    const ps_solvent_config* S = &cfg->solvents[is];
    if (S->field < 0 || S->field >= s->nf) {
      snprintf(err, errlen, "solvent %d: scfield out of range", is);
      rc = PS_ATTRIB_ERR;
      break;
    }
    if (S->kind == PS_SOLV_IONS) {
      if (S->charge_field < 0 || S->charge_field >= s->nq ||
          (S->has_block_field && (S->block_field < 0 || S->block_field >= s->nq)) || S->zc == 0.0) {
        snprintf(err, errlen, "solvent %d: simpleIons needs chargefield (and blockfield) and zc != 0", is);
        rc = PS_ATTRIB_ERR;
        break;
      }
    } else if (S->kind == PS_SOLV_SIMPLE) {
      /* PsSimpleSolvent::buildSolvers: addToDensAverage(volfrac) */
      s->dens_avg[S->field] = s->dens_avg[S->field] + S->volfrac;
    } else {
      snprintf(err, errlen, "solvent %d: unknown kind", is);
      rc = PS_ATTRIB_ERR;
      break;
    }
  }
  /* chargeFlexPseudoSpec blocks: chargefield in range, and (a restriction of this
   * restatement and of the device path) the only contributor to their scfield, so
   * that rho += za alpha phi_f sees the block's own density as the reference does */
  for (int ip = 0; ip < s->npol && rc == PS_OK; ++ip)
    for (int ib = 0; ib < s->pol[ip].nb && rc == PS_OK; ++ib) {
      const ps_block_charge* Z = block_charge_of(s, ip, ib);
      if (!Z->charged) continue;
      if (Z->charge_field < 0 || Z->charge_field >= s->nq) {
        snprintf(err, errlen, "polymer %d block %d: chargefield out of range", ip, ib);
        rc = PS_ATTRIB_ERR;
        break;
      }
      const int f = s->pol[ip].b[ib].cfg.field;
      int others = 0;
      for (int jp = 0; jp < s->npol; ++jp)
        for (int jb = 0; jb < s->pol[jp].nb; ++jb)
          if ((jp != ip || jb != ib) && s->pol[jp].b[jb].cfg.field == f) ++others;
      for (int is = 0; is < cfg->n_solvents; ++is)
        if (cfg->solvents[is].kind == PS_SOLV_SIMPLE && cfg->solvents[is].field == f) ++others;
      if (others) {
        snprintf(err, errlen, "polymer %d block %d: a charged block must be the only density "
                 "source of its scfield", ip, ib);
        rc = PS_INPUT_ERR;
      }
    }
  if (rc == PS_OK) {
    /* sum of volume fractions of polymers and solvents
       (psphysf/PsPhysFieldHldr.cpp:190-257) */
    double vt = 0.0;
    for (int is = 0; is < cfg->n_solvents; ++is) vt += cfg->solvents[is].volfrac;
    for (int ip = 0; ip < s->npol; ++ip) vt += cfg->polymers[ip].volfrac;
    if (fabs(vt - 1.0) > 0.00001) {
      snprintf(err, errlen, "sum of volume fractions %g != 1", vt);
      rc = PS_INPUT_ERR;
    }
  }
  for (int it = 0; it < cfg->n_interactions && rc == PS_OK; ++it) {
    const ps_interaction_config* I = &cfg->interactions[it];
    if (I->field_a < 0 || I->field_a >= s->nf || I->field_b < 0 || I->field_b >= s->nf ||
        I->field_a == I->field_b) {
      snprintf(err, errlen, "interaction %d: bad scfields", it);
      rc = PS_ATTRIB_ERR;
    }
    /* chiN = chi * Nlen (pseffhamil/PsFloryInteraction.cpp:159-161) */
    s->chin[it] = I->chi * s->scale_length;
  }
  if (rc == PS_OK && cfg->updater.kind == PS_UPD_ANDERSON) {
    int m = cfg->updater.anderson_depth;
    if (m < 0 || m > 64) {
      snprintf(err, errlen, "anderson_depth out of range");
      rc = PS_ATTRIB_ERR;
    } else {
      s->am_m = m;
      s->am_w = (double*)xcalloc((size_t)(m + 1) * s->nf * N, sizeof(double));
      s->am_d = (double*)xcalloc((size_t)(m + 1) * s->nf * N, sizeof(double));
      s->am_g = (double*)xcalloc((size_t)(m + 1) * (m + 1), sizeof(double));
    }
  }
  /* psSrandom(randomSeed + rank), rank 0 (pstrol/PsDomain.cpp:213) */
  mt_seed(&s->rng, (uint32_t)(cfg->seed & 0xffffffffULL));
  if (rc != PS_OK) {
    oracle_destroy(s);
    return rc;
  }
  *out = s;
  return PS_OK;
}

void oracle_destroy(oracle_state* s) {
  if (!s) return;
  for (int i = 0; i < PS_MAX_FIELDS; ++i) { free(s->w[i]); free(s->phi[i]); free(s->dh[i]); }
  free(s->p); free(s->cwork); free(s->qw); free(s->res); free(s->fpow);
  free(s->fcut); free(s->fregion); free(s->kcoul);
  for (int c = 0; c < PS_MAX_CHARGES; ++c) { free(s->rho[c]); free(s->psi[c]); }
  for (int ip = 0; ip < PS_MAX_POLYMERS; ++ip)
    for (int ib = 0; ib < OMAX_BLOCKS; ++ib) {
      oblock* B = &s->pol[ip].b[ib];
      free(B->qs); free(B->qts); free(B->wfac); free(B->k2); free(B->qqt);
      for (int e = 0; e < 2; ++e) {
        free(B->q_init[e]); free(B->q_final[e]);
        for (int a = 0; a < PS_MAX_JOINS; ++a) free(B->jnt_q[e][a]);
      }
    }
  free(s->am_w); free(s->am_d); free(s->am_g);
  free(s);
}

int oracle_block_steps(const oracle_state* s, int ip, int ib) { return s->pol[ip].b[ib].steps; }

/* PsMonomerDens::initialize "random" then PsConstraint::initialize (p = 0):
 * psphysf/PsMonomerDens.cpp:116-127, psbase/PsGridField.cpp:389-401,
 * psphysf/PsConstraint.cpp:146-152. */
void oracle_init_random(oracle_state* s) {
  for (int i = 0; i < s->nf; ++i)
    for (long r = 0; r < s->N; ++r) {
      double u = mt_real(&s->rng);
      s->w[i][r] = 1.0 * (u + (-0.5));
    }
  memset(s->p, 0, sizeof(double) * (size_t)s->N);
}

static double* field_ptr(const oracle_state* s, int which, int index) {
  switch (which) {
    case PS_FIELD_W: return s->w[index];
    case PS_FIELD_PHI: return s->phi[index];
    case PS_FIELD_CHARGE: return s->rho[index];
    case PS_FIELD_POTENTIAL: return s->psi[index];
    default: return s->p;
  }
}

void oracle_set_field(oracle_state* s, int which, int index, const double* data) {
  memcpy(field_ptr(s, which, index), data, sizeof(double) * (size_t)s->N);
}

void oracle_get_field(const oracle_state* s, int which, int index, double* data) {
  memcpy(data, field_ptr(s, which, index), sizeof(double) * (size_t)s->N);
}

void oracle_get_propagator(const oracle_state* s, int ip, int ib, int end, int n, double* out) {
  const oblock* B = &s->pol[ip].b[ib];
  const double* src = (end == PS_FROM_HEAD) ? B->qs : B->qts;
  memcpy(out, src + (size_t)n * s->N, sizeof(double) * (size_t)s->N);
}

void oracle_get_k2(const oracle_state* s, int ip, int ib, double* out) {
  memcpy(out, s->pol[ip].b[ib].k2, sizeof(double) * (size_t)s->N);
}

/* ---------------------------------------------------------------------------
 * Propagators
 * ------------------------------------------------------------------------- */

/* PsFlexPseudoSpec::solveQ (pspolymer/PsFlexPseudoSpec.cpp:244-293). */
static void solve_q(oracle_state* s, oblock* B, int from) {
  const long N = s->N;
  double* dst = (from == HEAD) ? B->qs : B->qts;
  const double scale_fft = 1.0 / ((double)N);
  double* qx = dst; /* slice 0 */
  memcpy(qx, B->q_init[from], sizeof(double) * (size_t)N);
  for (int ss = 1; ss <= B->steps; ++ss) {
    const double* prev = dst + (size_t)(ss - 1) * N;
    double* next = dst + (size_t)ss * N;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) s->qw[n] = prev[n] * B->wfac[n];
    oracle_scaled_pair_buf(s->n, s->qw, B->k2, s->res, s->cwork);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      double v = s->res[n] * B->wfac[n];
      next[n] = scale_fft * v;
    }
  }
  /* setFinalQ(getOtherEnd(from), qX) */
  int other = (from == HEAD) ? TAIL : HEAD;
  memcpy(B->q_final[other], dst + (size_t)B->steps * N, sizeof(double) * (size_t)N);
  B->final_set[other] = 1;
}

/* PsBlock::combineSetJnt (pspolymer/PsBlock.cpp:386-416). */
static void combine_set_jnt(oracle_state* s, oblock* B, int end) {
  const long N = s->N;
  double* prod = B->q_init[end];
  for (long r = 0; r < N; ++r) prod[r] = 1.0;
  for (int a = 0; a < B->njnt[end]; ++a) {
    const double* q = B->jnt_q[end][a];
    for (long r = 0; r < N; ++r) prod[r] *= q[r];
  }
  B->init_set[end] = 1;
}

static int jnts_set(const oblock* B, int end) {
  int all = 1;
  for (int a = 0; a < B->njnt[end]; ++a)
    if (!B->jnt_set[end][a]) all = 0;
  return all;
}

/* PsBlockCopolymer::publishQFrom + PsBlock::setJctQ (pspolymer/PsBlockCopolymer.cpp:283-313,
 * pspolymer/PsBlock.cpp:435-472). */
static void publish_q_from(oracle_state* s, opolymer* P, int end, int from) {
  oblock* F = &P->b[from];
  if (!F->final_set[end]) return;
  for (int c = 0; c < F->ncnt[end]; ++c) {
    oblock* T = &P->b[F->cnt_idx[end][c]];
    int tend = F->cnt_end[end][c];
    for (int a = 0; a < T->njnt[tend]; ++a) {
      if (T->jnt_key[tend][a] == from) {
        memcpy(T->jnt_q[tend][a], F->q_final[end], sizeof(double) * (size_t)s->N);
        T->jnt_set[tend][a] = 1;
      }
    }
  }
}

/* PsBlockCopolymer::updateBlockQ (pspolymer/PsBlockCopolymer.cpp:247-272). */
static void update_block_q(oracle_state* s, opolymer* P, int ib, int end) {
  oblock* B = &P->b[ib];
  int other = (end == HEAD) ? TAIL : HEAD;
  if (!B->init_set[end]) {
    if (jnts_set(B, end)) combine_set_jnt(s, B, end);
  }
  if (B->init_set[end] && !B->final_set[other]) {
    solve_q(s, B, end);
    publish_q_from(s, P, other, ib);
  }
}

/* PsBlock::setCalcQQTIntegral (pspolymer/PsBlock.cpp:255-380). */
static void calc_qqt(oracle_state* s, oblock* B, double bq) {
  const long N = s->N;
  const size_t num = (size_t)B->steps + 1;
  const size_t npts = num - 1;
  size_t numstail;
  int even;
  double modval = fmod((double)num, 2.0);
  if (modval == 0.0) { even = 1; numstail = npts - 3; }
  else { even = 0; numstail = npts - 2; }
  const double simp = 0.33333 * B->cfg.ds;
  const double trap = B->cfg.ds * 0.5;
  const double inv_bq = 1.0 / bq;
#pragma omp parallel for schedule(static)
  for (long r = 0; r < N; ++r) {
    double acc = 0.0;
    for (size_t n = 0; n <= numstail; n += 2) {
      double p1 = B->qs[n * N + r] * B->qts[(num - n - 1) * N + r];
      double p2 = B->qs[(n + 1) * N + r] * B->qts[(num - n - 2) * N + r];
      double p3 = B->qs[(n + 2) * N + r] * B->qts[(num - n - 3) * N + r];
      p2 = p2 * 4.0;
      acc = acc + p1;
      acc = acc + p2;
      acc = acc + p3;
    }
    acc = acc * simp;
    if (even) {
      double p1 = B->qs[(num - 2) * N + r] * B->qts[1 * N + r];
      double p2 = B->qs[(num - 1) * N + r] * B->qts[0 * N + r];
      double t = 0.0;
      t = t + p1;
      t = t + p2;
      t = t * trap;
      acc = acc + t;
    }
    B->qqt[r] = inv_bq * acc;
  }
}

/* PsBlockCopolymer::update (pspolymer/PsBlockCopolymer.cpp:188-239). */
static int polymer_update(oracle_state* s, opolymer* P) {
  const long N = s->N;
  for (int ib = 0; ib < P->nb; ++ib) {
    oblock* B = &P->b[ib];
    /* PsBlockBase::reset */
    B->init_set[HEAD] = B->init_set[TAIL] = 0;
    B->final_set[HEAD] = B->final_set[TAIL] = 0;
    for (int e = 0; e < 2; ++e)
      for (int a = 0; a < B->njnt[e]; ++a) B->jnt_set[e][a] = 0;
    /* PsBlock::reset: free ends get q0 = 1 */
    for (int e = 0; e < 2; ++e) {
      if (B->ncnt[e] == 0) {
        for (long r = 0; r < N; ++r) B->q_init[e][r] = 1.0;
        B->init_set[e] = 1;
      }
    }
    /* PsFlexPseudoSpec::reset: wfac = exp(-0.5 ds w) */
    const double ds2 = -0.5 * B->cfg.ds;
    const double* w = s->w[B->cfg.field];
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) B->wfac[n] = exp(ds2 * w[n]);
    /* PsChargeFlexPseudoSpec::reset (pspolymer/PsChargeFlexPseudoSpec.cpp:97-130):
     * wfac *= exp(facZ ds2 psi), facZ = za alpha L */
    const ps_block_charge* Z = block_charge_of(s, (int)(P - s->pol), ib);
    if (Z->charged) {
      const double facz = Z->za * Z->alpha * s->scale_length;
      const double* psi = s->psi[Z->charge_field];
      for (long n = 0; n < N; ++n) B->wfac[n] = B->wfac[n] * exp(facz * ds2 * psi[n]);
    }
  }
  int guard = 0;
  const double t0 = now_s();
  for (;;) {
    int all = 1;
    for (int ib = 0; ib < P->nb; ++ib)
      if (!(P->b[ib].final_set[HEAD] && P->b[ib].final_set[TAIL])) all = 0;
    if (all) break;
    if (++guard > 4 * OMAX_BLOCKS + 4) return PS_INPUT_ERR; /* unreachable blocks */
    for (int ib = 0; ib < P->nb; ++ib) {
      update_block_q(s, P, ib, HEAD);
      update_block_q(s, P, ib, TAIL);
    }
  }
  s->t_sweeps += now_s() - t0;
  /* PsBlock::calcBigQ of block 0 (pspolymer/PsBlock.cpp:204-237) */
  {
    oblock* B0 = &P->b[0];
    double tot = 0.0;
    for (long r = 0; r < N; ++r) {
      double v = (0.0 + B0->q_init[HEAD][r]) * B0->q_final[HEAD][r];
      tot = tot + v;
    }
    double q = tot / ((double)(1 * (double)N));
    P->bigq = q;
    P->logq = log(q);
    if (q != q) return PS_RUN_ERR;
  }
  if (P->pd) {
    /* PsPolyDisperseBCP::update / getLogBigQ (pspolymer/PsPolyDisperseBCP.cpp:282-377):
     * every quadrature block normalises with its own calcBigQ; ln Q sums the first
     * seed block's copies with weights w_k / Gamma(alpha) */
    for (int ib = 0; ib < P->nb; ++ib) {
      oblock* B = &P->b[ib];
      double tot = 0.0;
      for (long r = 0; r < N; ++r) {
        double v = (0.0 + B->q_init[HEAD][r]) * B->q_final[HEAD][r];
        tot = tot + v;
      }
      P->bq[ib] = tot / ((double)(1 * (double)N));
      if (P->bq[ib] != P->bq[ib]) return PS_RUN_ERR;
    }
    double sum = 0.0;
    for (int k = 0; k < P->n_g; ++k) sum = sum + ((log(P->bq[k]) * P->gw[k]) / P->galpha);
    P->logq = sum;
    P->bigq = exp(sum);
    for (int ib = 0; ib < P->nb; ++ib) calc_qqt(s, &P->b[ib], P->bq[ib]);
  } else {
    for (int ib = 0; ib < P->nb; ++ib) calc_qqt(s, &P->b[ib], P->bigq);
  }
  /* PsBlock::setPhysFields (pspolymer/PsBlock.cpp:153-196) */
  for (int ib = 0; ib < P->nb; ++ib) {
    oblock* B = &P->b[ib];
    double densfac = P->dwt[ib] * P->cfg.volfrac / P->length_ratio;
    double* phi = s->phi[B->cfg.field];
#pragma omp parallel for schedule(static)
    for (long r = 0; r < N; ++r) {
      double v = densfac * B->qqt[r];
      phi[r] = phi[r] + v;
    }
    /* PsChargeFlexPseudoSpec::setPhysFields (pspolymer/PsChargeFlexPseudoSpec.cpp:136-165):
     * rho += (phi_f alpha) za */
    const ps_block_charge* Z = block_charge_of(s, (int)(P - s->pol), ib);
    if (Z->charged) {
      double* rho = s->rho[Z->charge_field];
      for (long r = 0; r < N; ++r) {
        double t = 0.0 + phi[r];
        t = t * Z->alpha;
        t = t * Z->za;
        rho[r] = rho[r] + t;
      }
    }
  }
  return PS_OK;
}

/* ---------------------------------------------------------------------------
 * Field update
 * ------------------------------------------------------------------------- */

static int interaction_has(const ps_interaction_config* I, int f) {
  return I->field_a == f || I->field_b == f;
}

/* dH_i = p - w_i + sum_{int ∋ i} chiN (phi_other - avg_other):
 * pseffhamil/PsSteepDUpdater.cpp:174-184, :208-236 and
 * pseffhamil/PsFloryInteraction.cpp:204-269. */
static void compute_dh(oracle_state* s) {
  const long N = s->N;
  const int nf = s->nf;
#pragma omp parallel for schedule(static)
  for (long r = 0; r < N; ++r) {
    for (int i = 0; i < nf; ++i) {
      double d = 0.0;
      d = d + s->p[r];
      d = d - s->w[i][r];
      for (int it = 0; it < s->cfg.n_interactions; ++it) {
        const ps_interaction_config* I = &s->cfg.interactions[it];
        if (!interaction_has(I, i)) continue;
        int other = (i == I->field_a) ? I->field_b : I->field_a;
        double mask = -1.0 * s->dens_avg[other]; /* ((0 + wall)*-1 + 1) * -avg, wall = 0 */
        double x = 0.0;
        x = x + s->phi[other][r];
        x = x + mask;
        x = x * s->chin[it];
        d = d + x;
      }
      s->dh[i][r] = d;
    }
  }
}

/* Pressure rebuild after the w update: setConjgFieldsToPres + mixed terms,
 * scaled by 1/n_fields (pseffhamil/PsSteepDUpdater.cpp:283-332, :398-452),
 * then PsConstraint::updatePres / shiftPresField (psphysf/PsConstraint.cpp:184-262). */
static double rebuild_pressure(oracle_state* s) {
  const long N = s->N;
  const int nf = s->nf;
  for (long r = 0; r < N; ++r) {
    double pr = 0.0;
    for (int i = 0; i < nf; ++i) pr = pr + s->w[i][r];
    if (nf == 2) {
      for (int it = 0; it < s->cfg.n_interactions; ++it) {
        const ps_interaction_config* I = &s->cfg.interactions[it];
        if (interaction_has(I, 0) && interaction_has(I, 1)) {
          double x = 0.0; /* phi0 * chiN with phi0 = 0 */
          x = x * s->chin[it];
          pr = pr + x;
        }
      }
      pr = 0.5 * pr;
    } else {
      for (int it = 0; it < s->cfg.n_interactions; ++it) {
        const ps_interaction_config* I = &s->cfg.interactions[it];
        for (int n = 0; n < nf; ++n) {
          if (interaction_has(I, n)) continue;
          double x = 0.0;
          x = x + (s->phi[n][r] - s->dens_avg[n]);
          x = x + 0.0; /* phi0 */
          x = x * s->chin[it];
          pr = pr + x;
        }
      }
      double inv = 1.0 / 3.0;
      pr = inv * pr;
    }
    s->p[r] = pr;
  }
  /* updatePres with phi0 = 0: p *= 1; p -= mean; p *= 1; p += 0 */
  double tot = 0.0;
  for (long r = 0; r < N; ++r) tot = tot + s->p[r];
  double mean = tot / ((double)((double)N * 1));
  for (long r = 0; r < N; ++r) s->p[r] = s->p[r] - mean;
  return mean;
}

/* PsSimpleSolvent::setPhysFields (pssolvent/PsSimpleSolvent.cpp:86-140):
 * wFactor = exp(-w / L), Q = sum(wFactor) / N, phi += (vf / Q) wFactor. */
static void solvent_update(oracle_state* s, int is) {
  const long N = s->N;
  const ps_solvent_config* S = &s->cfg.solvents[is];
  const double* w = s->w[S->field];
  double* wf = s->res;  /* N doubles of scratch */
  const double negscale = -1.0 / s->scale_length;
  double tot = 0.0;
  for (long r = 0; r < N; ++r) {
    double v = 0.0 + w[r];
    v = v * negscale;
    wf[r] = exp(v);
    tot = tot + wf[r];
  }
  const double q = tot / ((double)1 * (double)N);
  s->solv_q[is] = q;
  const double f = S->volfrac / q;
  double* phi = s->phi[S->field];
  for (long r = 0; r < N; ++r) phi[r] = phi[r] + wf[r] * f;
}

/* PsSimpleIons::setPhysFields (pssolvent/PsSimpleIons.cpp:90-160):
 * e = exp(-zc psi), Q = sum(e) / N, e *= -neutralFactor / (Q zc);
 * blockfield density = e; rho += zc e. */
static void ions_update(oracle_state* s, int is) {
  const long N = s->N;
  const ps_solvent_config* S = &s->cfg.solvents[is];
  const double* psi = s->psi[S->charge_field];
  double* e = s->res;  /* N doubles of scratch */
  const double negfac = -1.0 * S->zc;
  double tot = 0.0;
  for (long r = 0; r < N; ++r) {
    double v = 0.0 + psi[r];
    v = v * negfac;
    e[r] = exp(v);
    tot = tot + e[r];
  }
  const double q = tot / ((double)1 * (double)N);
  s->solv_q[is] = q;
  const double cfac = -S->neutral_factor / (q * S->zc);
  for (long r = 0; r < N; ++r) e[r] = e[r] * cfac;
  if (S->has_block_field) {
    double* bf = s->rho[S->block_field];
    for (long r = 0; r < N; ++r) bf[r] = 0.0 + e[r];
  }
  double* rho = s->rho[S->charge_field];
  for (long r = 0; r < N; ++r) rho[r] = rho[r] + e[r] * S->zc;
}

/* PsPoissonUpdater::update (pseffhamil/PsPoissonUpdater.cpp:196-262) on every listed
 * chargeDens field; k2 list from build_k2 (:140-175). */
static void poisson_apply(oracle_state* s) {
  const ps_poisson_config* P = &s->pcfg;
  const long N = s->N;
  const double scale = 1.0 / ((double)N);
  for (int i = 0; i < P->n_fields; ++i) {
    double* rho = s->rho[P->fields[i]];
    double* psi = s->psi[P->fields[i]];
    double sum = 0.0;
    for (long r = 0; r < N; ++r) sum = sum + rho[r];
    const double gcd = sum / ((double)1 * (double)N);
    const double totc = -1.0 * gcd;
    for (long r = 0; r < N; ++r) rho[r] = rho[r] + totc;
    oracle_scaled_pair_buf(s->n, rho, s->kcoul, s->res, s->cwork);
    for (long r = 0; r < N; ++r) {
      const double psi0 = psi[r];
      const double psi1 = s->res[r] * scale;
      const double frac = fabs((psi1 - psi0) / psi0);
      if (frac > 0.2) s->res[r] = psi0 * 1.2;
    }
    for (long r = 0; r < N; ++r) psi[r] = s->res[r] * (1.0 * scale);
  }
}

static void post_order_set(oracle_state* s, int code, int on) {
  int k = 0;
  for (int i = 0; i < s->npost; ++i)
    if (s->post[i] != code) s->post[k++] = s->post[i];
  if (on) s->post[k++] = code;
  s->npost = k;
}

int oracle_set_poisson(oracle_state* s, const ps_poisson_config* p) {
  if (!p) {
    s->has_poisson = 0;
    post_order_set(s, 2, 0);
    return PS_OK;
  }
  if (p->n_fields < 1 || p->n_fields > s->nq || p->apply_frequency < 1) return PS_ATTRIB_ERR;
  for (int i = 0; i < p->n_fields; ++i)
    if (p->fields[i] < 0 || p->fields[i] >= s->nq) return PS_ATTRIB_ERR;
  if (!s->kcoul) s->kcoul = (double*)xcalloc((size_t)s->N, sizeof(double));
  long n = 0;
  for (int i = 0; i < s->n[0]; ++i)
    for (int j = 0; j < s->n[1]; ++j)
      for (int k = 0; k < s->n[2]; ++k) {
        const double k2 = calck2(s, i, j, k);
        s->kcoul[n++] = (k2 < 0.000000001) ? 0.0 : (4.0 * 3.1415 * p->bjerrum_len) / k2;
      }
  s->pcfg = *p;
  s->has_poisson = 1;
  post_order_set(s, 2, 1);
  return PS_OK;
}

void oracle_apply_poisson(oracle_state* s) {
  if (s->has_poisson) poisson_apply(s);
}

static int scheduled(long long t, long long start, long long freq, long long end) {
  return t >= start && (end < 0 || t <= end) && (t - start) % freq == 0;
}

/* PsSimpleSpecFilter::update / applyFilter (pseffhamil/PsSimpleSpecFilter.cpp:75-140),
 * PsSpecFilterUpdater::subtractAverage and findMaxVal (pseffhamil/PsSpecFilterUpdater.cpp:
 * 180-250), scaledFFTPair and scaleFFT = 1/N. */
static void filter_apply(oracle_state* s) {
  const ps_filter_config* F = &s->fcfg;
  if (F->cutoff_factor <= 0.0) return;
  const long N = s->N;
  double* c = s->cwork;
  double* pw = s->fpow;
  for (int i = 0; i < F->n_fields; ++i) {
    double* w = s->w[F->fields[i]];
    double sum = 0.0;
    for (long r = 0; r < N; ++r) sum = sum + w[r];
    const double wtot = -1.0 * (sum / ((double)1 * (double)N));
    for (long r = 0; r < N; ++r) w[r] = w[r] + wtot;
    for (long r = 0; r < N; ++r) { c[2 * r] = w[r]; c[2 * r + 1] = 0.0; }
    oracle_fftnd_inplace(s->n, c, -1);
    double mx = -1000000.00;
    for (long r = 0; r < N; ++r) {
      pw[r] = (c[2 * r] * c[2 * r]) + (c[2 * r + 1] * c[2 * r + 1]);
      if (pw[r] > mx) mx = pw[r];
    }
    if (s->fregion) {
      /* PsMultiSpecFilter::applyFilter (pseffhamil/PsMultiSpecFilter.cpp:222-262):
       * the cutoff is cutoffFactor times the max power of the index's region. */
      for (long c2 = 0; c2 < s->fncells; ++c2) s->fcut[c2] = 0.0;
      for (long r = 0; r < N; ++r) {
        const double kcut = F->cutoff_factor * pw[r];
        if (kcut > s->fcut[s->fregion[r]]) s->fcut[s->fregion[r]] = kcut;
      }
      for (long r = 0; r < N; ++r) pw[r] = (pw[r] < s->fcut[s->fregion[r]]) ? F->filter_strength : 1.0;
    } else {
      const double cut = F->cutoff_factor * mx;
      for (long r = 0; r < N; ++r) pw[r] = (pw[r] < cut) ? F->filter_strength : 1.0;
    }
    oracle_scaled_pair_buf(s->n, w, pw, s->res, c);
    const double scale = 1.0 / (double)N;
    for (long r = 0; r < N; ++r) w[r] = scale * s->res[r];
  }
}

int oracle_set_filter(oracle_state* s, const ps_filter_config* f) {
  if (!f) {
    s->has_filter = 0;
    post_order_set(s, 1, 0);
    return PS_OK;
  }
  if (f->n_fields < 1 || f->n_fields > s->nf || f->apply_frequency < 1) return PS_ATTRIB_ERR;
  for (int i = 0; i < f->n_fields; ++i)
    if (f->fields[i] < 0 || f->fields[i] >= s->nf) return PS_ATTRIB_ERR;
  const int multi = f->spec_cells[0] || f->spec_cells[1] || f->spec_cells[2];
  if (multi)
    for (int d = 0; d < 3; ++d)
      if (f->spec_cells[d] < 1 || s->n[d] % f->spec_cells[d] != 0) return PS_ATTRIB_ERR;
  if (!s->fpow) s->fpow = (double*)xcalloc((size_t)s->N, sizeof(double));
  free(s->fcut); free(s->fregion);
  s->fcut = NULL; s->fregion = NULL; s->fncells = 0;
  if (multi) {
    /* PsMultiSpecFilter::build_specCells_transpose (pseffhamil/PsMultiSpecFilter.cpp:
     * 175-212), serial: loops j (y), i (x), k (z) and numbers the index
     * nn = (j nx + i) nz + k, which the serial FFT then reads in (x, y, z) order. */
    const long nx = s->n[0], ny = s->n[1], nz = s->n[2];
    const long cx = nx / f->spec_cells[0], cy = ny / f->spec_cells[1], cz = nz / f->spec_cells[2];
    s->fncells = cx * cy * cz;
    s->fcut = (double*)xcalloc((size_t)s->fncells, sizeof(double));
    s->fregion = (long*)xcalloc((size_t)s->N, sizeof(long));
    for (long j = 0; j < ny; ++j)
      for (long i = 0; i < nx; ++i)
        for (long k = 0; k < nz; ++k) {
          const long ic0 = i / f->spec_cells[0], ic1 = j / f->spec_cells[1], ic2 = k / f->spec_cells[2];
          s->fregion[(j * nx + i) * nz + k] = ic2 * (cx * cy) + ic1 * cx + ic0;
        }
  }
  s->fcfg = *f;
  s->has_filter = 1;
  post_order_set(s, 1, 1);
  return PS_OK;
}

void oracle_apply_filter(oracle_state* s) {
  if (s->has_filter) filter_apply(s);
}

/* PsPolymerUpdater::calcFeField (pseffhamil/PsPolymerUpdater.cpp:172-226). */
static void calc_fe(oracle_state* s, double* fe_out, double* fe_nodis_out) {
  const long N = s->N;
  const int nf = s->nf;
  const double inv_vol = 1.0 / (double)N;
  double sum_tmp = 0.0;
  for (int ip = 0; ip < s->npol; ++ip) {
    double logq = s->pol[ip].logq;
    double vf = s->pol[ip].cfg.volfrac;
    double lr = s->pol[ip].length_ratio;
    sum_tmp = sum_tmp - ((vf * logq) / lr);
  }
  /* solvents: length ratio 1 / (length of polymer 0) */
  for (int is = 0; is < s->cfg.n_solvents; ++is) {
    double logq = log(s->solv_q[is]);
    double vf = s->cfg.solvents[is].volfrac;
    double lr = 1.0 / s->scale_length;
    sum_tmp = sum_tmp - ((vf * logq) / lr);
  }
  double tot = 0.0, tot_nd = 0.0;
  for (long r = 0; r < N; ++r) {
    double fe = 0.0;
    for (int i = 0; i < nf; ++i) {
      double prod = (0.0 + s->phi[i][r]) * s->w[i][r];
      prod = -1.0 * prod;
      fe = fe + prod;
    }
    fe = fe * 1.0;
    fe = inv_vol * fe;
    double ft = 0.0 + fe, ftn = 0.0 + fe;
    for (int it = 0; it < s->cfg.n_interactions; ++it) {
      const ps_interaction_config* I = &s->cfg.interactions[it];
      double a0 = s->dens_avg[I->field_a], a1 = s->dens_avg[I->field_b];
      double dis = (((0.0 + 1.0) * 1.0) * a0) * a1;
      dis = dis * s->chin[it];
      double v = (0.0 + s->phi[I->field_a][r]) * s->phi[I->field_b][r];
      v = v * s->chin[it];
      double vd = v - dis;
      ft = ft + inv_vol * vd;
      ftn = ftn + inv_vol * v;
    }
    tot = tot + ft;
    tot_nd = tot_nd + ftn;
  }
  *fe_out = sum_tmp + tot;
  *fe_nodis_out = sum_tmp + tot_nd;
}

/* Gaussian elimination with partial pivoting on an m x m system (row major);
 * returns 0 on success, 1 when a pivot is zero (caller then uses c = 0). */
int oracle_solve_small(int m, double* a, double* b) {
  for (int k = 0; k < m; ++k) {
    int piv = k;
    double best = fabs(a[k * m + k]);
    for (int i = k + 1; i < m; ++i)
      if (fabs(a[i * m + k]) > best) { best = fabs(a[i * m + k]); piv = i; }
    if (!(best > 0.0)) return 1;
    if (piv != k) {
      for (int j = 0; j < m; ++j) { double t = a[k * m + j]; a[k * m + j] = a[piv * m + j]; a[piv * m + j] = t; }
      double t = b[k]; b[k] = b[piv]; b[piv] = t;
    }
    for (int i = k + 1; i < m; ++i) {
      double f = a[i * m + k] / a[k * m + k];
      for (int j = k; j < m; ++j) a[i * m + j] = a[i * m + j] - f * a[k * m + j];
      b[i] = b[i] - f * b[k];
    }
  }
  for (int i = m - 1; i >= 0; --i) {
    double t = b[i];
    for (int j = i + 1; j < m; ++j) t = t - a[i * m + j] * b[j];
    b[i] = t / a[i * m + i];
  }
  return 0;
}

/* Steepest descent w update (pseffhamil/PsSteepDUpdater.cpp:264-278, :368-393). */
static void sd_direction(const oracle_state* s, long r, double* dir) {
  const int nf = s->nf;
  const double lam1 = s->cfg.updater.lambda1;
  for (int i = 0; i < nf; ++i) {
    double x = 0.0;
    for (int j = 0; j < nf; ++j)
      if (j != i) x = x + s->dh[j][r];
    x = x * (-1.0 * lam1);
    x = x + s->dh[i][r];
    dir[i] = x;
  }
}

static void update_fields(oracle_state* s, ps_scalars* sc) {
  const long N = s->N;
  const int nf = s->nf;
  compute_dh(s);
  /* residual statistics (diagnostic only) */
  {
    double ss = 0.0;
    for (long r = 0; r < N; ++r)
      for (int i = 0; i < nf; ++i) ss = ss + s->dh[i][r] * s->dh[i][r];
    sc->dh_norm = sqrt(ss / (double)N);
  }
  const ps_updater_config* U = &s->cfg.updater;
  if (U->kind == PS_UPD_ANDERSON) {
    const int m = s->am_m;
    const int slots = m + 1;
    const long long k = s->am_k;
    const int cur = (int)(k % slots);
    double* Wc = s->am_w + (size_t)cur * nf * N;
    double* Dc = s->am_d + (size_t)cur * nf * N;
#pragma omp parallel for schedule(static)
    for (long r = 0; r < N; ++r) {
      double dir[PS_MAX_FIELDS];
      sd_direction(s, r, dir);
      for (int i = 0; i < nf; ++i) {
        Wc[(size_t)i * N + r] = s->w[i][r];
        Dc[(size_t)i * N + r] = dir[i];
      }
    }
    int nh = (int)(k < m ? k : m);
    /* Gram row: G[cur][slot(k-j)] = D^k . D^{k-j}, j = 0..nh */
    for (int j = 0; j <= nh; ++j) {
      int sj = (int)((k - j) % slots);
      const double* Dj = s->am_d + (size_t)sj * nf * N;
      double g = 0.0;
      for (long t = 0; t < (long)nf * N; ++t) g = g + Dc[t] * Dj[t];
      s->am_g[cur * slots + sj] = g;
      s->am_g[sj * slots + cur] = g;
    }
    double c[64];
    int use = (k >= U->anderson_start) && nh > 0;
    if (use) {
      double A[64 * 64], V[64];
      for (int a = 1; a <= nh; ++a) {
        int sa = (int)((k - a) % slots);
        V[a - 1] = s->am_g[cur * slots + cur] - s->am_g[cur * slots + sa];
        for (int b = 1; b <= nh; ++b) {
          int sb = (int)((k - b) % slots);
          A[(a - 1) * nh + (b - 1)] = s->am_g[cur * slots + cur] - s->am_g[cur * slots + sa] -
                                      s->am_g[cur * slots + sb] + s->am_g[sa * slots + sb];
        }
      }
      if (oracle_solve_small(nh, A, V) != 0) {
        for (int a = 0; a < nh; ++a) V[a] = 0.0;
      }
      for (int a = 0; a < nh; ++a) c[a] = V[a];
    } else {
      nh = 0;
    }
    const double mix = use ? U->anderson_mix : U->lambda0;
#pragma omp parallel for schedule(static)
    for (long r = 0; r < N; ++r) {
      for (int i = 0; i < nf; ++i) {
        double wk = Wc[(size_t)i * N + r];
        double dk = Dc[(size_t)i * N + r];
        double wh = wk, dhh = dk;
        for (int a = 1; a <= nh; ++a) {
          int sa = (int)((k - a) % slots);
          wh = wh + c[a - 1] * (s->am_w[(size_t)sa * nf * N + (size_t)i * N + r] - wk);
          dhh = dhh + c[a - 1] * (s->am_d[(size_t)sa * nf * N + (size_t)i * N + r] - dk);
        }
        s->w[i][r] = wh + mix * dhh;
      }
    }
    s->am_k = k + 1;
  } else {
    const double lam0 = s->cfg.updater.lambda0;
#pragma omp parallel for schedule(static)
    for (long r = 0; r < N; ++r) {
      double dir[PS_MAX_FIELDS];
      sd_direction(s, r, dir);
      for (int i = 0; i < nf; ++i) {
        double x = dir[i] * lam0;
        s->w[i][r] = s->w[i][r] + x;
      }
    }
  }
  /* addRandUpdateConjgFields (pseffhamil/PsPolymerUpdater.cpp:263-295): one
   * Gaussian per point per field, drawn even when noise = 0. */
  if (U->noise != 0.0) {
    for (int i = 0; i < nf; ++i)
      for (long r = 0; r < N; ++r) {
        double g = U->noise * mt_gauss(&s->rng);
        double v = 0.0 + g;
        v = v * 1.0;
        s->w[i][r] = s->w[i][r] + v;
      }
  } else {
    for (int i = 0; i < nf; ++i)
      for (long r = 0; r < N; ++r) (void)mt_gauss(&s->rng);
  }
  sc->pressure_mean = rebuild_pressure(s);
  calc_fe(s, &sc->free_energy, &sc->free_energy_nodis);
}

int oracle_iterate(oracle_state* s, int niter, ps_scalars* hist) {
  const long N = s->N;
  for (int it = 0; it < niter; ++it) {
    ps_scalars sc;
    memset(&sc, 0, sizeof(sc));
    const double t_begin = now_s();
    s->t_sweeps = 0.0;
    for (int i = 0; i < s->nf; ++i) memset(s->phi[i], 0, sizeof(double) * (size_t)N);
    /* PsChargeDens::update: resetDensField (psphysf/PsChargeDens.cpp:180-190) */
    for (int c = 0; c < s->nq; ++c) memset(s->rho[c], 0, sizeof(double) * (size_t)N);
    /* PsDomain::update: solvents, then polymers (pstrol/PsDomain.cpp:359-362) */
    for (int is = 0; is < s->cfg.n_solvents; ++is) {
      if (s->cfg.solvents[is].kind == PS_SOLV_IONS) ions_update(s, is);
      else solvent_update(s, is);
    }
    for (int ip = 0; ip < s->npol; ++ip) {
      int rc = polymer_update(s, &s->pol[ip]);
      if (rc != PS_OK) return rc;
      sc.q[ip] = s->pol[ip].bigq;
      sc.log_q[ip] = s->pol[ip].logq;
    }
    double mx = 0.0;
    for (long r = 0; r < N; ++r) {
      double t = 0.0;
      for (int i = 0; i < s->nf; ++i) t += s->phi[i][r];
      double d = fabs(t - 1.0);
      if (d > mx) mx = d;
    }
    sc.max_incomp = mx;
    update_fields(s, &sc);
    /* the other updaters of updaterSequence (pseffhamil/PsEffHamil.cpp:190-203), each on
     * the PsUpdater::update schedule (psbase/PsUpdater.cpp:180-206) */
    for (int k = 0; k < s->npost; ++k) {
      const long long t = s->iter;
      if (s->post[k] == 1 && s->has_filter &&
          scheduled(t, s->fcfg.apply_start, s->fcfg.apply_frequency, s->fcfg.apply_end))
        filter_apply(s);
      if (s->post[k] == 2 && s->has_poisson &&
          scheduled(t, s->pcfg.apply_start, s->pcfg.apply_frequency, s->pcfg.apply_end))
        poisson_apply(s);
    }
    s->t_total = now_s() - t_begin;
    s->iter++;
    sc.iteration = s->iter;
    if (!(sc.free_energy == sc.free_energy)) sc.error_flags |= 2;
    if (hist) hist[it] = sc;
  }
  return PS_OK;
}

void oracle_last_timing(const oracle_state* s, double* t_sweeps, double* t_total) {
  *t_sweeps = s->t_sweeps;
  *t_total = s->t_total;
}

/* A bounded sample of the sweep work: nsteps operator-split steps of the
 * first polymer's first block from its head (same arithmetic as solve_q),
 * with wfac from the current w.  Returns the wall time in seconds. */
double oracle_propagate_sample(oracle_state* s, int nsteps) {
  const long N = s->N;
  opolymer* P = &s->pol[0];
  oblock* B = &P->b[0];
  const double t0 = now_s();
  const double ds2 = -0.5 * B->cfg.ds;
  const double* w = s->w[B->cfg.field];
#pragma omp parallel for schedule(static)
  for (long n = 0; n < N; ++n) B->wfac[n] = exp(ds2 * w[n]);
  for (long r = 0; r < N; ++r) B->qs[r] = 1.0;
  const double scale_fft = 1.0 / ((double)N);
  for (int ss = 1; ss <= nsteps; ++ss) {
    const double* prev = B->qs + (size_t)((ss - 1) % B->steps) * N;
    double* next = B->qs + (size_t)(((ss - 1) % B->steps) + 1) * N;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) s->qw[n] = prev[n] * B->wfac[n];
    oracle_scaled_pair_buf(s->n, s->qw, B->k2, s->res, s->cwork);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      double v = s->res[n] * B->wfac[n];
      next[n] = scale_fft * v;
    }
  }
  return now_s() - t0;
}

void oracle_mt_reals(unsigned long long seed, long n, double* out) {
  mt_state st;
  mt_seed(&st, (uint32_t)(seed & 0xffffffffULL));
  for (long i = 0; i < n; ++i) out[i] = mt_real(&st);
}

void oracle_mt_gauss(unsigned long long seed, long n, double* out) {
  mt_state st;
  mt_seed(&st, (uint32_t)(seed & 0xffffffffULL));
  for (long i = 0; i < n; ++i) out[i] = mt_gauss(&st);
}

void oracle_mt_u32(unsigned long long seed, long n, unsigned int* out) {
  mt_state st;
  mt_seed(&st, (uint32_t)(seed & 0xffffffffULL));
  for (long i = 0; i < n; ++i) out[i] = mt_u32(&st);
}
