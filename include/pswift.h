/*
 * pswift.h -- C-ABI of the B200 SCFT inner loop (PolySwift++ hot path).
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross this boundary and no C++ exception escapes it.  Fields cross the
 * boundary as contiguous row-major (x slowest, z fastest) arrays of double,
 * whatever precision the device path computes in.  Status codes mirror the
 * reference's PS_ERR codes (polyswift/polyswift/polyswift.cxx:115-125).
 *
 * Reference interfaces replaced (paths inside the PolySwift++ tree):
 *   ps_gpu_create          PsDomain::buildData/buildSolvers      pstrol/PsDomain.cpp:207-285
 *   ps_gpu_set_fields      PsPhysFldFuncs::restore (dens, conj)  psphysf/PsPhysFldFuncs.cpp:150-166
 *   ps_gpu_init_random     PsMonomerDens::initialize "random"    psphysf/PsMonomerDens.cpp:116-127
 *   ps_gpu_iterate         PsDomain::update(t)                   pstrol/PsDomain.cpp:332-372
 *                          (PsBlockCopolymer::update pspolymer/PsBlockCopolymer.cpp:189-239 +
 *                           PsSteepDUpdater::update pseffhamil/PsSteepDUpdater.cpp:159-203)
 *   ps_gpu_get_scalars     PsPolymerUpdater::getFreeE / PsBlockCopolymer::getLogBigQ
 *                          pseffhamil/PsPolymerUpdater.h:124, pspolymer/PsBlockCopolymer.h:114-116
 *   ps_gpu_get_propagator  PsBlock qs/qts storage                pspolymer/PsBlock.cpp:131-134
 *   ps_fft_scaled_pair     PsFFTBase::scaledFFTPair              psbase/PsFFTBase.h:105,
 *                                                               psfft/PsFFTW.cpp:196-224
 *   ps_fft_scaled_pair_im  PsFFTBase::scaledFFTPairIm            psbase/PsFFTBase.h:116,
 *                                                               psfft/PsFFTW.cpp:227-257
 *   ps_fft_convolve_re     PsFFTBase::convolveRe                 psbase/PsFFTBase.h:94,
 *                                                               psfft/PsFFTW.cpp:150-189
 *   ps_fft_forward_abs     PsFFTBase::forwardFFTAbs              psbase/PsFFTBase.h:83,
 *                                                               psfft/PsFFTW.cpp:122-149
 *   ps_fft_forward         PsFFTBase::calcForwardFFT             psbase/PsFFTBase.h:125,
 *                                                               psfft/PsFFTW.cpp:260-278
 *   ps_fft_backward        PsFFTBase::calcBackwardFFT            psbase/PsFFTBase.h:134,
 *                                                               psfft/PsFFTW.cpp:281-297
 *   ps_fft_size            PsFFTBase::getFFTSize                 psbase/PsFFTBase.h:75
 *   ps_fft_get_grid        PsFFTBase::getGrid (the grid extents) psbase/PsFFTBase.h:70
 */
#ifndef PSWIFT_H
#define PSWIFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_MAX_BLOCKS 8
#define PS_MAX_JOINS 4
#define PS_MAX_POLYMERS 16 /* polymers, counting each quadrature chain of a
                              polyDisperseBCP as one */
#define PS_MAX_FIELDS 4
#define PS_MAX_INTERACTIONS 6
#define PS_MAX_SOLVENTS 2
#define PS_MAX_CHARGES 2

/* Status codes: same numbers as the reference's quitPolyswift() codes. */
enum {
  PS_OK = 0,
  PS_ATTRIB_ERR = 3, /* bad attribute / configuration                    */
  PS_RUN_ERR = 4,    /* NaN/Inf in Q or F (PsBlock::calcBigQ throw)      */
  PS_INPUT_ERR = 6,  /* block steps, fractions, unsupported grid         */
  PS_GPU_ERR = 7     /* CUDA error or missing device                     */
};

/* Arithmetic of the propagator sweeps.  Q, F, the contour quadrature and the
 * field update are FP64 in both modes. */
enum { PS_PREC_FP64 = 0, PS_PREC_MIXED = 1 };

/* Updater kinds: "steepestDescent" (pseffhamil/PsSteepDUpdater.cpp) and
 * Anderson mixing (added; the reference has no Anderson updater). */
enum { PS_UPD_STEEPEST = 0, PS_UPD_ANDERSON = 1 };

/* Field selectors for get/set: conjugate field w_i, density phi_i, pressure p;
 * for chargeDens PhysField c (psphysf/PsChargeDens.cpp:20-30) its charge
 * density rho_c ("ChargeDensity") and electric potential psi_c
 * ("ElectricPotential"). */
enum { PS_FIELD_W = 0, PS_FIELD_PHI = 1, PS_FIELD_PRES = 2, PS_FIELD_CHARGE = 3,
       PS_FIELD_POTENTIAL = 4 };

/* Solvent kinds: simpleSolvent (pssolvent/PsSimpleSolvent.cpp) and
 * simpleIons (pssolvent/PsSimpleIons.cpp). */
enum { PS_SOLV_SIMPLE = 0, PS_SOLV_IONS = 1 };

/* Block end selectors for propagator access. */
enum { PS_FROM_HEAD = 0, PS_FROM_TAIL = 1 };

/* <Block name> kind = flexPseudoSpec (psbase/PsBlockBase.cpp:67-145,
 * pspolymer/PsFlexPseudoSpec.cpp:58-82). */
typedef struct ps_block_config {
  int field;               /* scfield: index of the monomerDens PhysField   */
  double lengthfrac;       /* lengthfrac                                    */
  double ds;               /* ds                                            */
  double bseg_ratio;       /* bSegRatio (1.0 by default)                    */
  int force_block_steps;   /* forceBlockSteps option                        */
  int n_head;              /* number of entries in head_joined (0 = freeEnd)*/
  int n_tail;              /* number of entries in tail_joined (0 = freeEnd)*/
  int head_joined[PS_MAX_JOINS]; /* block indices inside the same polymer   */
  int tail_joined[PS_MAX_JOINS];
} ps_block_config;

/* <Polymer name> kind = blockCopolymer (psbase/PsPolymer.cpp:42-73). */
typedef struct ps_polymer_config {
  double volfrac;          /* volfrac                                       */
  int length;              /* length (statistical units)                    */
  int n_blocks;
  ps_block_config blocks[PS_MAX_BLOCKS];
} ps_polymer_config;

/* <Polymer name> kind = polyDisperseBCP (pspolymer/PsPolyDisperseBCP.cpp:41-455):
 * block poly_block (polyblock) has a Schulz length distribution of exponent
 * alpha, integrated by n_g-point generalized Gauss-Laguerre quadrature
 * (x^(alpha-1) e^-x).  The polymer becomes n_g chains; chain k copies the
 * blocks with the polydisperse block's lengthfrac
 *   f_k = (x_k n_b + N_c) / N - (1 - f_poly),  N_c = (1 - f_poly) N,
 *   n_b = (N - N_c) / alpha,
 * densities weighted by w_k / Gamma(alpha), and ln Q = sum_k w_k ln Q_k / Gamma(alpha).
 * At most two blocks (as in the reference); the chains count towards
 * PS_MAX_POLYMERS.  Block index b of such a polymer in the ABI is the
 * reference's quadrature block b: seed block b / n_g of chain b % n_g. */
typedef struct ps_polydisperse_config {
  int enabled;
  int poly_block;          /* polyblock: index of the polydisperse block    */
  int n_g;                 /* n_g                                           */
  double alpha;            /* alpha (Schulz exponent, > 0)                  */
} ps_polydisperse_config;

/* <Interaction name> kind = flory (pseffhamil/PsFloryInteraction.cpp:65-89). */
typedef struct ps_interaction_config {
  int field_a;             /* scfields[0]                                   */
  int field_b;             /* scfields[1]                                   */
  double chi;              /* chi; chiN = chi * length of the first polymer */
} ps_interaction_config;

/* <Updater name> (pseffhamil/PsSteepDUpdater.cpp:47-76). */
typedef struct ps_updater_config {
  int kind;                /* PS_UPD_STEEPEST or PS_UPD_ANDERSON            */
  double lambda0;          /* relaxlambdas[0]                               */
  double lambda1;          /* relaxlambdas[1]                               */
  double noise;            /* noise (Gaussian strength)                     */
  int anderson_depth;      /* history depth m (Anderson only)               */
  double anderson_mix;     /* mixing applied to the combined residual       */
  int anderson_start;      /* plain steps before the history is used        */
} ps_updater_config;

/* <Solvent name> kind = simpleSolvent | simpleIons (psbase/PsSolvent.cpp:40-60,
 * pssolvent/PsSimpleIons.cpp:30-60). */
typedef struct ps_solvent_config {
  int field;               /* scfield: index of the monomerDens PhysField   */
  double volfrac;          /* volfrac                                       */
  int kind;                /* PS_SOLV_SIMPLE or PS_SOLV_IONS                */
  int charge_field;        /* simpleIons: chargefield (chargeDens index)    */
  int has_block_field;     /* simpleIons: blockfield given                  */
  int block_field;         /* simpleIons: blockfield (chargeDens index)     */
  double zc;               /* simpleIons: zc, the ion charge                */
  double neutral_factor;   /* simpleIons: neutralFactor                     */
} ps_solvent_config;

/* <Block name> kind = chargeFlexPseudoSpec (pspolymer/PsChargeFlexPseudoSpec.cpp:42-75):
 * the block's Boltzmann factor gains exp(-ds/2 za alpha L psi_c) (L = length
 * of polymer 0) and rho_c += za alpha phi_f after its density
 * (pspolymer/PsChargeFlexPseudoSpec.cpp:97-165).  The device path needs the
 * charged block to be the only contributor to its scfield. */
typedef struct ps_block_charge {
  int charged;             /* 0: flexPseudoSpec                              */
  int charge_field;        /* chargefield (chargeDens index)                */
  double za;               /* za                                            */
  double alpha;            /* alpha                                         */
} ps_block_charge;

typedef struct ps_config {
  int n[3];                /* numCellsGlobal                                */
  double cell[3];          /* cellSizes (Rg units)                          */
  int precision;           /* PS_PREC_FP64 or PS_PREC_MIXED                 */
  int n_fields;            /* monomerDens PhysFields (2 or 3)               */
  int n_polymers;
  ps_polymer_config polymers[PS_MAX_POLYMERS];
  int n_interactions;
  ps_interaction_config interactions[PS_MAX_INTERACTIONS];
  ps_updater_config updater;
  unsigned long long seed; /* randomSeed (MT19937 init_genrand(seed+rank)) */
  int calc_disorder;       /* History freeEnergy calcDisorder (default 1)   */
  int device;              /* CUDA device ordinal                           */
  /* <Solvent name> kind = simpleSolvent (pssolvent/PsSimpleSolvent.cpp:86-140):
   * Q_s = <exp(-w_f / L)>, phi_f += volfrac exp(-w_f / L) / Q_s, F -= volfrac L ln Q_s,
   * L = length of polymer 0.  Appended at the end so the fields above keep their offsets. */
  int n_solvents;
  ps_solvent_config solvents[PS_MAX_SOLVENTS];
  /* chargeDens PhysFields: rho_c is reset every iteration (PsChargeDens::update)
   * and filled by simpleIons solvents and charged blocks; psi_c changes only
   * through ps_gpu_set_fields and the Poisson updater.  Appended at the end. */
  int n_charges;
  ps_block_charge block_charge[PS_MAX_POLYMERS][PS_MAX_BLOCKS];
  ps_polydisperse_config polydisperse[PS_MAX_POLYMERS];
} ps_config;

/* n-point generalized Gauss-Laguerre rule for the weight x^a e^-x on [0, inf):
 * nodes ascending into x[n], weights into w[n] (sum w = Gamma(a + 1)); the
 * rule PsGaussLagQuad(n, a) computes (pspolymer/PsGaussLagQuad.cpp), found
 * here as the eigen-decomposition of the Jacobi matrix (Golub-Welsch).
 * 1 <= n <= 64, a > -1. */
int ps_gauss_laguerre(int n, double a, double* x, double* w);

typedef struct ps_scalars {
  double free_energy;        /* sumFe, disorder term subtracted            */
  double free_energy_nodis;  /* sumFeNoDis                                 */
  double log_q[PS_MAX_POLYMERS];
  double q[PS_MAX_POLYMERS];
  double max_incomp;         /* max_r |sum_i phi_i(r) - 1|                 */
  double dh_norm;            /* sqrt(mean_r sum_i dH_i(r)^2)               */
  double pressure_mean;      /* mean removed from p by updatePres          */
  long long iteration;       /* number of completed iterations             */
  int error_flags;           /* bit 0: non-finite Q, bit 1: non-finite F   */
} ps_scalars;

typedef struct ps_handle ps_handle;
typedef struct ps_fft ps_fft;

/* Library version string. */
const char* ps_version(void);

/* Message for the last error of a handle (or of the calling thread when the
 * handle is NULL, e.g. after a failed create). */
const char* ps_gpu_last_error(const ps_handle* h);

/* Build the device state for one SCFT instance.  Performs the reference's
 * setAttrib/buildData/buildSolvers checks: block-step rounding, sum of length
 * fractions, sum of volume fractions, supported grid extents.  Polymers may be
 * linear or branched (trees of blocks joined at their ends, as head_joined /
 * tail_joined describe; a junction joins at most PS_MAX_JOINS + 1 block ends);
 * cyclic block graphs are PS_INPUT_ERR (pspolymer/PsBlockCopolymer.cpp:189-313). */
int ps_gpu_create(const ps_config* cfg, ps_handle** out);
int ps_gpu_destroy(ps_handle* h);

/* Number of contour steps a block takes (PsBlockBase::setBlockSteps). */
int ps_gpu_block_steps(const ps_handle* h, int polymer, int block, int* steps);

/* Copy a field in or out.  which = PS_FIELD_W / PS_FIELD_PHI (index = field)
 * or PS_FIELD_PRES (index ignored).  on_device != 0: data is a device pointer
 * on the handle's device.  Sizes are n[0]*n[1]*n[2] doubles. */
int ps_gpu_set_fields(ps_handle* h, int which, int index, const double* data, int on_device);
int ps_gpu_get_fields(ps_handle* h, int which, int index, double* data, int on_device);

/* Read a field back without waiting for it (no reference counterpart: the
 * reference's PhysFields live in host memory).  The field's current value is
 * copied on the handle's stream into a device snapshot, and from there into
 * `host` on a separate copy stream, so the transfer overlaps the iterations
 * that follow; `host` should be pinned (page-locked) memory for the copy to
 * run asynchronously.  `host` holds the field once ps_gpu_fields_wait returns.
 * Each (which, index) has one snapshot, allocated on its first use: a second
 * read of the same field waits (on the device) for the first one's host copy
 * before its snapshot is taken. */
int ps_gpu_get_fields_async(ps_handle* h, int which, int index, double* host);
/* Copy a field in from host memory without waiting (no reference counterpart).
 * A field w_i goes up on the handle's stream, ahead of the next iteration.
 * The pressure field goes up on its own stream after the work enqueued so
 * far, and only the next iteration's field update (its first reader) waits
 * for it, so the copy overlaps that iteration's sweeps.  `host` should be
 * pinned memory (a device pointer on the handle's device also works), and
 * must stay unchanged until ps_gpu_fields_wait, ps_gpu_synchronize or
 * ps_gpu_get_scalars returns.  Batch instances copy synchronously. */
int ps_gpu_set_fields_async(ps_handle* h, int which, int index, const double* host);
/* Wait for every asynchronous read-back and upload of the handle. */
int ps_gpu_fields_wait(ps_handle* h);

/* Reference initialisation: every monomerDens w_i = U[0,1) - 0.5 drawn from
 * MT19937 seeded with cfg->seed, fields in declaration order; p = 0. */
int ps_gpu_init_random(ps_handle* h);

/* Run n_iter SCFT iterations (PsDomain::update order). */
int ps_gpu_iterate(ps_handle* h, int n_iter);

/* Scalars of the last completed iteration (copies a few doubles to host). */
int ps_gpu_get_scalars(ps_handle* h, ps_scalars* out);

/* Read one stored propagator slice q(r, s_n) of a block: end = PS_FROM_HEAD
 * gives qs[n], PS_FROM_TAIL gives qts[n] (values of the last iteration). */
int ps_gpu_get_propagator(ps_handle* h, int polymer, int block, int end, int n,
                          double* out);

/* Wait for all work of the handle (stream synchronise). */
int ps_gpu_synchronize(ps_handle* h);

/* Number of this library's kernel launches one iteration issues (0 before the
 * first iteration).  No reference counterpart: launch accounting for benchmarks. */
long long ps_gpu_launches_per_iteration(const ps_handle* h);

/* Sweep timing (no reference counterpart; the reference only times whole
 * updates, polyswift/polyswift/polyswift.cxx:540-600).  After enabling, the
 * next max_samples iterations record CUDA events on the handle's stream
 * around their propagator sweeps.  ps_gpu_sweep_timing returns those
 * durations in ms (and clears them), the algorithmic bytes of one iteration's
 * sweeps (3 * N * sizeof(slice element) per propagator step) and the number
 * of propagator steps per iteration. */
int ps_gpu_enable_sweep_timing(ps_handle* h, int max_samples);
/* The handle's CUDA stream (a cudaStream_t), for callers that order their own
 * work or events against the handle's iterations. */
void* ps_gpu_stream(const ps_handle* h);

/* Kernel variant of the propagator sweeps (no reference counterpart).  Every
 * variant computes the same result; they differ in how passes are fused
 * (bits 0, 1), in the FFT decomposition (bit 2: row + x-y planes; bit 4:
 * 256 x 256 y-z planes on a cluster of eight CTAs instead of a row pass and
 * y pencils, PS_ATTRIB_ERR for other plane sizes) and in whether an
 * instance's sweeps share launches or run as concurrent launch chains
 * (bit 3).  variant = -1 (the default) times all variants on the handle's
 * own sweeps before its first captured iteration and keeps the fastest;
 * 0..31 forces one.  Branched polymers take every variant: with bit 3 a
 * sweep that starts at a junction is a launch chain that waits for the chains
 * arriving there; without it, all sweeps share launches step by step and a
 * sweep leaving a junction starts one step after the last arriving sweep
 * ends, its junction product launched in between (so branched polymers also
 * run in batches).
 * ps_gpu_get_variant also returns the measured sweep time of each variant (ms). */
int ps_gpu_set_variant(ps_handle* h, int variant);
int ps_gpu_get_variant(const ps_handle* h, int* variant, float* tune_ms, int n_tune);

/* Switch the arithmetic of the propagator sweeps between iterations (no
 * reference counterpart).  w, p, phi and the FP64 Anderson history carry over
 * unchanged, so a run can iterate in PS_PREC_MIXED until the FP32 noise floor
 * of the sweeps and finish in PS_PREC_FP64 (precision escalation).  The first
 * switch to a precision allocates its slice storage; the kernel variant is
 * re-tuned.  Not allowed on a batch instance (PS_ATTRIB_ERR). */
int ps_gpu_set_precision(ps_handle* h, int precision);
int ps_gpu_sweep_timing(ps_handle* h, double* ms_out, int max_out, int* n_out,
                        double* bytes_per_iter, long long* steps_per_iter);

/* --- Spectral filter updater: <Updater name> kind = simpleSpecFilter
 * (pseffhamil/PsSimpleSpecFilter.cpp:75-140, pseffhamil/PsSpecFilterUpdater.cpp:155-250;
 * schedule psbase/PsUpdater.cpp:60-206).  After each iteration t (0-based) with
 * apply_start <= t <= apply_end (apply_end < 0: no end) and (t - apply_start) %
 * apply_frequency == 0, every listed conjugate field w loses its mean and is
 * filtered: w = Re(IFFT(mask FFT(w))) / N with mask = filter_strength where
 * |FFT(w)|^2 < cutoff_factor * max |FFT(w)|^2 and 1 elsewhere.  cutoff_factor
 * <= 0 leaves the fields alone.  FP64 whatever the sweep precision.  Passing
 * NULL removes the filter; not allowed on a batch instance.
 *
 * kind = multiSpecFilter (pseffhamil/PsMultiSpecFilter.cpp:130-262) sets
 * spec_cells (specCellSizes, each dividing its grid extent): the spectrum is
 * cut into (nx/sx)(ny/sy)(nz/sz) regions and the max, hence the cutoff, is
 * taken per region.  The region of linear spectrum index n is found as the
 * serial reference does, by reading n in (y, x, z) order:
 * y = n / (nx nz), x = (n / nz) % nx, z = n % nz
 * (pseffhamil/PsMultiSpecFilter.cpp:175-212).  The mask applies at n in
 * (x, y, z) order.  All spec_cells 0 selects simpleSpecFilter. */
typedef struct ps_filter_config {
  int n_fields;              /* updatefields                                  */
  int fields[PS_MAX_FIELDS]; /* monomerDens PhysField indices                 */
  double cutoff_factor;      /* cutoffFactor                                  */
  double filter_strength;    /* filterStrength                                */
  long long apply_start;     /* applyStart                                    */
  long long apply_frequency; /* applyFrequency                                */
  long long apply_end;       /* applyEnd (< 0: until the end of the run)      */
  int spec_cells[3];         /* specCellSizes (multiSpecFilter); 0 0 0: simple */
  int pad;
} ps_filter_config;
int ps_gpu_set_spectral_filter(ps_handle* h, const ps_filter_config* filter);
/* Apply the filter once now, outside its schedule. */
int ps_gpu_apply_spectral_filter(ps_handle* h);

/* --- Poisson updater: <Updater name> kind = poissonUpdater
 * (pseffhamil/PsPoissonUpdater.cpp:50-270; schedule psbase/PsUpdater.cpp:60-206).
 * At the scheduled steps (as for the spectral filter), for every listed
 * chargeDens field c: rho_c loses its mean (in place), res = IFFT(K FFT(rho_c))
 * with K(k) = 4 (3.1415) bjerrum_len / |k|^2 (0 where |k|^2 < 1e-9), and
 * psi_c = res / N, except where |res/N - psi_c| > 0.2 |psi_c|, which take
 * 1.2 psi_c / N (the reference's clamp, psi_c = 0 included).  FP64, after the
 * iteration's graph; updaters installed later run later.  NULL removes it. */
typedef struct ps_poisson_config {
  int n_fields;              /* updatefields: chargeDens indices              */
  int fields[PS_MAX_CHARGES];
  double bjerrum_len;        /* bjerrumLen                                    */
  double relaxlambda;        /* relaxlambda (read, unused, as in the reference) */
  long long apply_start;
  long long apply_frequency;
  long long apply_end;       /* < 0: no end                                   */
} ps_poisson_config;
int ps_gpu_set_poisson(ps_handle* h, const ps_poisson_config* poisson);
int ps_gpu_apply_poisson(ps_handle* h);

/* --- Batched instances (no reference counterpart: the reference runs one
 * PsDomain per process, polyswift/polyswift/polyswift.cxx:544-588) ----------
 * ps_gpu_batch_create builds `count` independent instances on one device
 * (each exactly as ps_gpu_create would, updater noise included: each instance
 * draws from its own generator; spectral filters and Poisson updaters set on an
 * instance run on its stream between batch iterations, at their scheduled
 * steps) and groups them into
 * size classes of equal grid and precision.  ps_gpu_batch_iterate runs n_iter
 * iterations of every instance: each class's propagator sweeps are merged into
 * one launch per contour step, the per-instance field updates run as parallel
 * branches, and the whole iteration is one captured CUDA graph after the
 * first.  Instances may hold linear or branched polymers (branched sweeps
 * are offset to start after their junction's arriving sweeps, see
 * ps_gpu_set_variant).  Each instance's result equals ps_gpu_iterate on it
 * alone with the same kernel variant.  ps_gpu_batch_instance returns the instance's handle
 * for ps_gpu_set_fields / get_fields / get_scalars / get_propagator (owned by
 * the batch: do not destroy it; do not iterate it while the batch runs).
 * Within a size class the instances' sweeps either share one launch per
 * contour step, or (variant bit 3) run as each instance's own concurrent
 * launch chains; the per-class autotuner times both, and
 * ps_gpu_batch_set_variant forces one kernel variant for every class (-1:
 * autotune each class on its merged sweeps). */
typedef struct ps_batch ps_batch;
int ps_gpu_batch_create(const ps_config* cfgs, int count, ps_batch** out);
int ps_gpu_batch_destroy(ps_batch* b);
int ps_gpu_batch_size(const ps_batch* b);
ps_handle* ps_gpu_batch_instance(ps_batch* b, int index);
int ps_gpu_batch_iterate(ps_batch* b, int n_iter);
int ps_gpu_batch_set_variant(ps_batch* b, int variant);
/* Size classes: class_of[i] for each instance, variants[c] for each class. */
int ps_gpu_batch_classes(const ps_batch* b, int* n_classes, int* class_of, int max_inst,
                         int* variants, int max_classes);
long long ps_gpu_batch_launches_per_iteration(const ps_batch* b);
void* ps_gpu_batch_stream(const ps_batch* b);
/* Message for the last error of a batch (or of the calling thread when b is NULL). */
const char* ps_gpu_batch_last_error(const ps_batch* b);

/* --- Adjoint of the propagator sweeps (no reference counterpart) ----------
 * For one block copolymer chain (FP64): linear chains with block 0
 * starting at a free end are checkpointed (mirror-symmetric chains such as
 * homopolymers and ABA triblocks run both sweeps); branched chains keep every
 * slice.  ps_adj_create takes a one-polymer melt; ps_adj_create_polymer takes
 * quadrature chain `chain` (0 unless the polymer is a polyDisperseBCP, then
 * 0..n_g-1) of polymer `polymer` of any configuration (a blend with other
 * polymers and solvents) and computes that chain's contribution to phi and
 * its ln Q: the blend's phi is the sum over its chains and solvents, and its
 * dL/dw the sum of the chains' adjoints and the solvents' closed-form terms.
 * ps_adj_species reports the chain's free-energy weight (volfrac times the
 * polydisperse density weight), its length ratio and the configuration's
 * average density per field (n_fields doubles), for the free energy
 * F = -sum weight ln Q / ratio + ...  ps_adj_forward computes, from the fields
 * w (device, n_fields*N doubles), the densities phi (device, n_fields*N) and
 * ln Q exactly as one iteration of ps_gpu_iterate computes them
 * (PsBlockCopolymer::update, pspolymer/PsBlockCopolymer.cpp:189-239).
 * ps_adj_backward takes dL/dphi (device, n_fields*N) and dL/dlnQ for the
 * last forward and returns dL/dw (device, n_fields*N), dL/dL_d for the three
 * box lengths L_d = n_d * cell_d (host, 3) and dL/d(ds_b) for each block's
 * contour step (host, n_blocks).  Slices are checkpointed every
 * checkpoint_interval contour steps (1: full storage; 0: ceil(sqrt(steps)));
 * the results do not depend on the interval.  ps_adj_info reports the steps
 * per sweep, the interval and the bytes of slice storage. */
typedef struct ps_adj ps_adj;
int ps_adj_create(const ps_config* cfg, int checkpoint_interval, ps_adj** out);
int ps_adj_create_polymer(const ps_config* cfg, int polymer, int chain, int checkpoint_interval,
                          ps_adj** out);
int ps_adj_species(const ps_adj* a, double* f_weight, double* length_ratio, double* dens_avg);
/* Charged systems (chargeFlexPseudoSpec blocks): the potential psi (device,
 * n_charges*N doubles) enters a charged block's Boltzmann factor next to w
 * and is held fixed by the adjoint; ps_adj_set_potential sets it (zero at
 * creation) and ps_adj_potential_grad returns dL/dpsi (device, n_charges*N)
 * for the last ps_adj_backward. */
int ps_adj_set_potential(ps_adj* a, const double* psi);
int ps_adj_potential_grad(ps_adj* a, double* g_psi);
int ps_adj_destroy(ps_adj* a);
int ps_adj_forward(ps_adj* a, const double* w, double* phi, double* log_q);
int ps_adj_backward(ps_adj* a, const double* g_phi, double g_log_q, double* g_w, double* g_box,
                    double* g_ds);
int ps_adj_info(const ps_adj* a, int* contour_steps, int* checkpoint_interval, size_t* slice_bytes);
void* ps_adj_stream(const ps_adj* a);
/* Message for the last error of an adjoint (or of the calling thread when a is NULL). */
const char* ps_adj_last_error(const ps_adj* a);

/* --- Fault injection for the bounded waits --------------------------------
 * No counterpart in the reference.  Every wait of a kernel on a bulk copy is
 * bounded; when a plane pass's wait runs out, the pass sets error bit 2 of the
 * handle's status word, drains the copy still in flight (full bound) and
 * returns, and the handle reports PS_GPU_ERR with the context still usable.
 * This sets the poll limit of that first wait on the current device (default
 * 2^22 polls; 0 gives up at once, 0xFFFFFFFF restores the default), so a test
 * can drive the timeout path without a fault.  Not for production runs. */
int ps_gpu_set_bulk_wait_limit(unsigned int polls);

/* --- FFT plugin: PsFFTBase<T,3> with host pointers ------------------------
 * The transforms are unnormalised and follow the reference's FFTW c2c calls on
 * real data (forward sign -1, backward +1).  Inputs and outputs are host arrays
 * of n[0]*n[1]*n[2] doubles in row-major order; each call copies them over
 * PCIe (a correct plugin, not the fast path) and returns when res is written.
 * Errors: PS_ATTRIB_ERR (null argument), PS_GPU_ERR (CUDA).
 *   ps_fft_scaled_pair     res = Re(IFFT(kdata * FFT(data)))
 *   ps_fft_scaled_pair_im  res = Re(IFFT(kdata * FFT(i*data)))  (data is the imaginary part)
 *   ps_fft_convolve_re     res = Re(IFFT(FFT(data1) * FFT(data2)))
 *   ps_fft_forward_abs     res = |FFT(data)|^2  (re^2 + im^2, as the reference computes it)
 *   ps_fft_forward         res = Re(FFT(data))
 *   ps_fft_backward        res = Re(IFFT(data)) for real data (the spectrum's imaginary part is 0)
 *   ps_fft_size            n[0]*n[1]*n[2];  ps_fft_get_grid  the extents n[3] */
int ps_fft_create(const int n[3], int precision, int device, ps_fft** out);
int ps_fft_destroy(ps_fft* f);
int ps_fft_size(const ps_fft* f, size_t* n_total);
int ps_fft_get_grid(const ps_fft* f, int n[3]);
int ps_fft_scaled_pair(ps_fft* f, const double* data, const double* kdata, double* res);
int ps_fft_scaled_pair_im(ps_fft* f, const double* data, const double* kdata, double* res);
int ps_fft_convolve_re(ps_fft* f, const double* data1, const double* data2, double* res);
int ps_fft_forward_abs(ps_fft* f, const double* data, double* res);
int ps_fft_forward(ps_fft* f, const double* data, double* res);
int ps_fft_backward(ps_fft* f, const double* data, double* res);
/* Message for the last FFT-plugin error of the calling thread. */
const char* ps_fft_last_error(void);

/* --- scaledFFTPair without any allocation ---------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need the transform: a host whose device memory is all owned by
 * another allocator (a framework's caching allocator or a pool that reserved
 * the GPU at start-up), or a solver loop that must not allocate once running.
 * Same result as ps_fft_scaled_pair, but data, kdata and res are the caller's
 * DEVICE arrays (n[0]*n[1]*n[2] doubles on the current device; data and res
 * 16-byte aligned) and the call is asynchronous on `stream` (a cudaStream_t;
 * NULL is the default stream).  The working storage is one fixed device array
 * of ps_fft_noalloc_scratch_bytes() bytes (4 MiB) per device, held until the
 * process exits: grids whose half spectrum nx*ny*(nz/2+1)*16 bytes plus
 * tables exceed it return PS_INPUT_ERR (64^3 fits, 96^3 does not).  All calls on a device
 * share that storage, so calls that overlap on the GPU (other streams or
 * threads) race.  The first call on each device resolves the storage's
 * address; make it before any stream capture (calls outside a capture resolve
 * it again, so a device reset by the host does not leave it stale).  A bulk
 * copy that times out inside the kernels leaves res unwritten and is not
 * reported.  Errors: PS_ATTRIB_ERR (null or misaligned pointer), PS_INPUT_ERR
 * (extent or size), PS_GPU_ERR (CUDA). */
int ps_fft_scaled_pair_noalloc(const int n[3], const double* data, const double* kdata,
                               double* res, void* stream);
size_t ps_fft_noalloc_scratch_bytes(void);
/* Message for the last error of ps_fft_scaled_pair_noalloc on the calling thread. */
const char* ps_fft_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PSWIFT_H */
