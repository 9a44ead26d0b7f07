/*
 * hhg_gpu.h -- C ABI of the B200 engine for HigherHarmonics' per-k-point
 * Bloch integration -> Brillouin-zone current sum -> trapezoidal FFT path.
 *
 * The reference has no FFI: its boundary is the C++ class
 * HHG::Dispatch::Dispatcher (sources/HHG/Dispatch/Dispatcher.hpp:14-50),
 * whose compute(rank, n_ranks, n_z) fills current_density_time through
 *   System::compute_current_density(Laser const*, TimeIntegrationConfig const&,
 *                                   int rank, int n_ranks[, int n_z])
 * (sources/HHG/Systems/PiFlux.hpp:92-93, Honeycomb.hpp:70-71,
 *  DiracSystem.hpp:58-59), after which main() runs the TrapezoidalFFT
 * (sources/hhg.cpp:264-292).  The entry points below replace those calls with
 * plain-C types: POD descriptors in, caller-owned host buffers out, status
 * codes instead of C++ exceptions.  No CUDA or torch type appears here; a
 * stream is passed as an opaque pointer where one is accepted.
 *
 * Units are the reference's (Laser.hpp:13-16): time in 1/omega_L, energies
 * in hbar*omega_L, momenta in inverse lattice units, hbar = e = 1.  Each
 * pulse carries an energy_scale that multiplies every model energy, so a
 * model given in other reduced units (e.g. the 2D Dirac model with omega =
 * 0.1) is integrated in the reference's units with energy_scale = 1/omega.
 *
 * Threading: one host thread per context.  Calls are synchronous unless
 * named *_async.  Several contexts may share a device.
 */
#ifndef HHG_GPU_H
#define HHG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HHG_ABI_VERSION 4

/* Errors: the reference throws std::invalid_argument / std::runtime_error
 * (sources/hhg.cpp:232, Dispatch/PiFluxDispatcher.cpp:104) and Boost.Odeint
 * throws when 500 consecutive steps fail; these map to status codes. */
typedef enum hhg_status {
    HHG_OK = 0,
    HHG_BAD_CONFIG = 1,   /* invalid descriptor / unknown system or laser type */
    HHG_STEP_LIMIT = 2,   /* a trajectory exceeded the failed-step / step limit */
    HHG_NONFINITE = 3,    /* a trajectory produced a non-finite Bloch vector */
    HHG_CUDA_ERROR = 4,   /* CUDA runtime / cuFFT failure */
    HHG_UNSUPPORTED = 5   /* valid request this build does not implement */
} hhg_status;

/* Model families (the reference's system_type, sources/hhg.cpp:224-233). */
typedef enum hhg_system_kind {
    HHG_SYS_DIRAC2D = 0,   /* gapped 2D Dirac: d = (v(kx-Ax), v(ky-Ay), mass) */
    HHG_SYS_PIFLUX2D = 1,  /* square-lattice pi-flux: d = -2t(cos(kx-Ax), cos(ky-Ay), 0) */
    HHG_SYS_PIFLUX3D = 2,  /* reference PiFlux: d = 2t(cos kx, cos ky, cos(kz-A)), field || z */
    HHG_SYS_HONEYCOMB = 3, /* reference Honeycomb, optional staggered mass */
    HHG_SYS_DIRAC3D = 4    /* reference DiracSystem sigma form, k = (k_z, kappa) */
} hhg_system_kind;

/* System: replaces the System ctor arguments (e.g. PiFlux.cpp:56-71).
 * hopping = t (PiFlux: band_width/sqrt(12), Honeycomb: band_width/6),
 * velocity = v (Dirac2D), mass = gap term, (pol_x, pol_y) = field
 * polarisation unit vector (Honeycomb's laser_theta, Honeycomb.hpp:93-95).
 *
 * Thermal initial state and relaxation (the reference models PiFlux-3D,
 * Honeycomb without mass and Dirac-3D only; the variant models take the
 * filled lower band and no relaxation):
 *   beta         = photon_energy / (k_B T) (PiFlux.cpp:63); 0 stands for
 *                  T = 0, the reference's is_zero(T) branch, whose Fermi
 *                  function is a step (GlobalDefinitions.hpp:36-41);
 *   fermi_energy = E_F / photon_energy (PiFlux.cpp:64);
 *   inv_diag_relax, inv_offdiag_relax = 1e15 hbar / (tau photon_energy)
 *                  (PiFlux.cpp:67-68); inv_diag_relax > 0 selects the
 *                  relaxation right-hand side as the reference's
 *                  __time_evolution__ does (PiFlux.cpp:509-516,
 *                  Honeycomb.cpp:214-223); the off-diagonal rate is read by
 *                  PiFlux-3D only (the dispatcher substitutes the diagonal
 *                  time when offdiagonal_relaxation_time <= 0,
 *                  PiFluxDispatcher.cpp:22-35).
 * All four are in the model's energy units: a pulse's energy_scale
 * multiplies fermi_energy and the rates and divides beta. */
typedef struct hhg_system_desc {
    int32_t kind;
    int32_t reserved;
    double hopping;
    double velocity;
    double mass;
    double pol_x, pol_y;
    double beta;
    double fermi_energy;
    double inv_diag_relax;
    double inv_offdiag_relax;
} hhg_system_desc;

typedef enum hhg_pulse_kind {
    HHG_PULSE_COSINE = 0,     /* CosineLaser, sources/HHG/Laser/CosineLaser.cpp:22-26 */
    HHG_PULSE_CONTINUOUS = 1, /* ContinuousLaser: envelope 1 (ContinuousLaser.cpp) */
    HHG_PULSE_GAUSS = 2,      /* GaussLaser (GaussLaser.cpp): envelope
                                 exp(-(t - c)^2 / (2 s^2)), c = t_begin + 3 pi n_cycles,
                                 s = pi n_cycles / sqrt(2 ln 20); no window cut */
    HHG_PULSE_SPLINE = 3      /* Laser::laser_function with use_spline (Laser.hpp:32-37):
                                 a cubic spline through caller samples, 0 after
                                 spline_cut -- the reference's PowerLawField,
                                 QuenchedField, DoubleLaser and ExperimentalLaser */
} hhg_pulse_kind;

/* One pulse instance plus its TimeIntegrationConfig
 * (sources/HHG/TimeIntegrationConfig.hpp:5-12).  A(t) =
 * amplitude * envelope(t) * sin(t + phase): for COSINE envelope = 0.5(1 -
 * cos((t - t_begin)/n_cycles)) on (t_begin, t_begin + 2 pi n_cycles), 0
 * elsewhere; CONTINUOUS and GAUSS as above; phase = 0 is the reference.  For
 * SPLINE, A(t) = amplitude * s(t) for t <= spline_cut and 0 after, where s is
 * the cubic spline through samples[k] at t_begin + k sample_dt (k <
 * n_samples) with s' = deriv_begin at the first and deriv_end at the last
 * sample (clamped ends, as boost::math cardinal_cubic_b_spline with given
 * endpoint derivatives; a NaN derivative is estimated by the one-sided
 * five-point difference), beyond the last sample the last piece continued.
 * The sampled window is [window_begin, window_end] in n_measurements
 * intervals of n_subdivisions initial RKF78 steps each (the reference uses
 * 50, e.g. PiFluxDispatcher.cpp:53). */
typedef struct hhg_pulse_desc {
    int32_t kind;
    int32_t n_measurements;
    int32_t n_subdivisions;
    int32_t reserved;
    double amplitude;     /* Laser::momentum_amplitude */
    double n_cycles;
    double t_begin;       /* Laser::t_begin */
    double phase;
    double window_begin;  /* TimeIntegrationConfig::t_begin */
    double window_end;    /* TimeIntegrationConfig::t_end */
    double energy_scale;  /* multiplies hopping, velocity and mass */
    const double *samples;  /* HHG_PULSE_SPLINE: n_samples values, host memory (read during the call) */
    int64_t n_samples;      /* >= 4 */
    double sample_dt;
    double deriv_begin, deriv_end;
    double spline_cut;      /* Laser::t_end of a spline laser */
} hhg_pulse_desc;

/* k-point quadrature. */
typedef enum hhg_grid_kind {
    HHG_GRID_TENSOR_GL = 0,        /* n1 x n2 Gauss-Legendre on [x_lo,x_hi]x[y_lo,y_hi] */
    HHG_GRID_RHOMBIC_GL = 1,       /* n1 x n2 GL in fractional coords of the honeycomb BZ */
    HHG_GRID_PIFLUX3D_REF = 2,     /* PiFlux::current_density_continuum_limit grid, n1 = z_range, n2 = N_coarse */
    HHG_GRID_HONEYCOMB_HEX_REF = 3,/* Honeycomb::compute_current_density grid, n1 = N_k */
    HHG_GRID_EXPLICIT = 4,         /* caller rows: kx, ky, kz, weight, S0x, S0y, S0z, 0 */
    HHG_GRID_PIFLUX3D_OCCUPATION = 5, /* PiFlux::compute_occupation_numbers grid (PiFlux.cpp:909-953):
                                         k = (x pi/N, pi/2, z pi/N), x, z < N = n1, row x N + z */
    HHG_GRID_PIFLUX3D_CUBE = 6,    /* PiFlux::current_per_energy grid (PiFlux.cpp:955-1035): k =
                                      (x, y, +-z) pi/N, x, y, z < N = n1, weight 1/N^3, rows
                                      2 (z N^2 + y N + x) + (0: +z, 1: -z) */
    HHG_GRID_PIFLUX3D_DEBUG = 7,   /* PiFlux::compute_current_density_debug momenta (PiFlux.cpp:320-371):
                                      k = (pi/2, pi/2 - 0.02 pi i, 0.49 pi), i < 25 (n_debug_points,
                                      GlobalDefinitions.hpp), weight 1; no size parameters */
    HHG_GRID_DIRAC3D_DEBUG = 8     /* DiracSystem::compute_current_density_debug (DiracSystem.cpp:333-363,
                                      427-457): n1 = n_z, x_hi = max_k; k_z = (n_z/10) 2 max_k / n_z,
                                      kappa_i = (i + 1) kappa_max / 26 with kappa_max =
                                      sqrt(max_k^2 - k_z^2), i < 25; weight k_z kappa / |k| */
} hhg_grid_kind;

typedef struct hhg_grid_desc {
    int32_t kind;
    int32_t n1, n2;
    int32_t reserved;
    double x_lo, x_hi, y_lo, y_hi;
    const double *rows; /* HHG_GRID_EXPLICIT: n_rows x 8 doubles, host memory */
    int64_t n_rows;
} hhg_grid_desc;

/* Steppers.  RKF78: the reference's controlled Fehlberg 7(8) (PiFlux.cpp:104-110).
 * MAGNUS4: two-point Gauss 4th-order Magnus, magnus_substeps per interval
 * (no reference counterpart).  DIRAC_MAGNUS: the reference's Dirac path,
 * DiracSystem::time_evolution_magnus (DiracSystem.cpp:176-211) -- one
 * closed-form step per interval, S <- exp(Omega) S, Omega from the first
 * four Legendre moments of A over the interval (30-point Gauss,
 * Laser.cpp:40-55) and the Magnus series of MagnusMatrix.cpp:25-76;
 * HHG_SYS_DIRAC3D only. */
typedef enum hhg_stepper {
    HHG_STEPPER_RKF78 = 0,
    HHG_STEPPER_MAGNUS4 = 1,
    HHG_STEPPER_DIRAC_MAGNUS = 2
} hhg_stepper;
typedef enum hhg_precision { HHG_PREC_FP64 = 0, HHG_PREC_MIXED = 1 } hhg_precision;
typedef enum hhg_proposer {
    HHG_PROPOSER_NONE = 0,    /* reference: every interval restarts at dt = measure_every / n_subdivisions */
    HHG_PROPOSER_CARRY = 1,   /* first step of an interval = last controller proposal */
    HHG_PROPOSER_LEARNED = 2, /* warp-synchronous dyadic steps, level proposed by a trained MLP */
    HHG_PROPOSER_LOCKSTEP = 3 /* warp-synchronous dyadic steps, level carried between intervals */
} hhg_proposer;

/* Solver options.  abs_tol / rel_tol: the reference uses 1e-12 / 1e-8
 * (PiFlux.cpp:20-21).  max_failed_steps: Boost.Odeint's failed_step_checker
 * limit (500).  max_attempts_per_interval bounds every device loop.
 * tile_k: k-points per work item in units of 32 (0 = auto).
 * block_threads: threads per CTA (0 = auto). */
typedef struct hhg_solver_opts {
    int32_t stepper;
    int32_t precision;
    int32_t proposer;
    int32_t magnus_substeps;
    double abs_tol, rel_tol;
    int32_t max_failed_steps;
    int32_t max_attempts_per_interval;
    int32_t tile_k;
    int32_t block_threads;
    const struct hhg_mlp *mlp; /* HHG_PROPOSER_LEARNED: the trained network (host memory) */
    int32_t mlp_every;         /* intervals between network proposals (>= 1, default 16) */
    int32_t coarsen_div;       /* lockstep / learned proposers: after an accepted step the warp
                                  halves its level when every lane's error norm is below
                                  1 / coarsen_div; 0 = the default: 600 in FP64 (the
                                  controller's growth rule, 0.9 err^(-1/8) >= 2), 64 in mixed
                                  precision (the FP32 right-hand side's rounding floor in the
                                  error estimate); 2 .. 65536 */
} hhg_solver_opts;

/* The learned step-size proposer (no counterpart in the reference, whose
 * controller restarts every interval at measure_every / n_subdivisions):
 * an MLP 8 -> 64 -> 64 -> 64 -> 1 with SiLU after the first three layers,
 * BF16 weights and activations, FP32 accumulation.  Inputs per k-point at the
 * start of a measurement interval: kx/pi, ky/pi, A(t0), E(t0) = -dA/dt, the
 * Bloch vector S(t0), log2(h / interval); output: the level
 * T = log2(interval / h*) of the largest step h* the RKF78 error norm accepts
 * (with a 0.9 safety factor).  A warp of 32 k-points steps at level
 * max ceil(T + level_margin).  params: w1[64][8], b1[64], w2[64][64], b2[64],
 * w3[64][64], b3[64], w4[64], b4 (row-major [out][in]); inputs are
 * standardised by (x - in_mu) * in_isig, the output de-standardised by
 * T = y * out_sigma + out_mu. */
#define HHG_MLP_INPUTS 8
#define HHG_MLP_HIDDEN 64
#define HHG_MLP_N_PARAMS (64 * 8 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1)
typedef struct hhg_mlp {
    float params[HHG_MLP_N_PARAMS];
    float in_mu[HHG_MLP_INPUTS];
    float in_isig[HHG_MLP_INPUTS];
    float out_mu, out_sigma;
    float level_margin;
    float reserved;
} hhg_mlp;

/* One training record (floats): the 8 raw inputs, the target level T,
 * h / interval of the recorded attempt, its error norm, 0. */
#define HHG_HIST_FIELDS 12

typedef struct hhg_train_opts {
    int32_t epochs;
    int32_t batch;      /* rows per Adam step (multiple of 128) */
    float lr;           /* Adam step size */
    float beta1, beta2, eps;
    float lr_final;     /* cosine decay from lr to lr_final over all steps */
    int32_t reserved;
    uint64_t seed;      /* batch order */
} hhg_train_opts;

typedef struct hhg_stats {
    int64_t k_points;
    int64_t trajectories;
    int64_t attempted_steps;  /* k.steps: attempted RKF78 steps (or Magnus sub-steps) */
    int64_t rejected_steps;
    int64_t failed_trajectories;
    int32_t poly_degree;      /* degree of the staged A(t) interpolants */
    int32_t items;            /* work items of the persistent launch */
    double kernel_ms;         /* device time of the integration kernel(s), CUDA events */
    double total_ms;          /* device time of the whole call */
} hhg_stats;

typedef struct hhg_ctx hhg_ctx;
typedef struct hhg_plan hhg_plan;

/* k-resolved observables (hhg_gpu_k_resolved). */
typedef enum hhg_kresolved {
    HHG_KOUT_BLOCH = 0,       /* the Bloch vector S: 3 doubles */
    HHG_KOUT_OCCUPATIONS = 1, /* lower and upper band amplitudes of S at k - A(t_i):
                                 sqrt((|S| -+ S.d_hat)/2), 2 doubles (PiFlux.cpp:227-235) */
    HHG_KOUT_CURRENT = 2      /* the trajectory's weighted current, weight x the
                                 system's time-evolution output: 1 double (Dirac-3D) */
} hhg_kresolved;

/* The Dirac system's momentum quadrature (DiracSystem::compute_current_density
 * and compute_current_density_diagonal_relaxation, DiracSystem.cpp:271-331,
 * 365-425, called by DiracDispatcher::compute, DiracDispatcher.cpp:66-79):
 *   k_z = (z - n_z/2) dz, dz = 2 max_k / n_z, z = 1 .. n_z - 1 without n_z/2
 *   (integer division; that slice has weight 0);
 *   kappa over [0, sqrt(max_k^2 - k_z^2)] with the integrand
 *   S_z(k_z, kappa, t_i) k_z kappa / |k| (0 at kappa = 0);
 *   j(t_i) = dz * sum_z (kappa integral).
 * The kappa integral is the adaptive trapezoidal rule the reference calls as
 * split_integrate<100>(f, 0, kappa_max, n_kappa, threshold, elementwise
 * error) from its author's library (not available; restated from the call):
 * [0, kappa_max] is cut into n_splits equal splits; each split starts as the
 * trapezoid of n_kappa panels and is halved (T <- T/2 + h sum f(midpoints))
 * until max_i |T_new(t_i) - T_old(t_i)| < threshold or max_halvings halvings
 * are done; the integral is the sum of the splits' last estimates. */
typedef struct hhg_kappa_quad {
    double max_k;          /* DiracSystem::max_k = band_width (DiracSystem.cpp:48, 62) */
    double threshold;      /* absolute elementwise change (DiracDispatcher.cpp:13: 1e-3) */
    int32_t n_z;           /* k_z slices + 1 (the config's n_z) */
    int32_t n_kappa;       /* panels of a split's first trapezoid (DiracDispatcher.cpp:14: 10) */
    int32_t n_splits;      /* equal splits of the kappa range (split_integrate<100>) */
    int32_t max_halvings;  /* refinement cap per split; 0 = 12 */
    int32_t z_first;       /* slices z_first .. z_first + z_count - 1 of z = 1 .. n_z - 1 only */
    int32_t z_count;       /* (one rank's block, DiracSystem.cpp:288-295); 0 = all slices */
} hhg_kappa_quad;

typedef struct hhg_kappa_stats {
    int64_t trajectories;  /* (k_z, kappa) nodes whose samples entered the estimates */
    int64_t speculative;   /* nodes integrated ahead of a convergence test and discarded */
    int32_t rounds;        /* refinement levels evaluated, the first trapezoids included */
    int32_t splits;        /* k_z slices x n_splits */
    int32_t unconverged;   /* splits still at or above the threshold after max_halvings */
    int32_t max_level;     /* most halvings any split took */
    int32_t launches;      /* integration launches (several levels and chunks of splits) */
    int32_t reserved;
} hhg_kappa_stats;

/* Library / context management. */
int hhg_abi_version(void);
hhg_status hhg_gpu_create(hhg_ctx **ctx, int device);
void hhg_gpu_destroy(hhg_ctx *ctx);
const char *hhg_last_error(const hhg_ctx *ctx);
void hhg_default_solver_opts(hhg_solver_opts *opts);

/* Gauss-Legendre nodes / weights on [-1,1], ascending (the reference's
 * gauss::container<n> tables, sources/HHG/thread_gauss.hpp, hold the positive
 * half of the same rule). */
hhg_status hhg_gauss_legendre(int n, double *x, double *w);

/* Number of k rows a grid descriptor expands to, and the rows themselves
 * (kx, ky, kz, weight, S0x, S0y, S0z, 0) for the given system.  rows may be
 * NULL to query the count only. */
hhg_status hhg_grid_rows(const hhg_system_desc *sys, const hhg_grid_desc *grid, double *rows,
                         int64_t *n_rows);

/* One-shot drop-in for System::compute_current_density over n_pulses pulse
 * instances: j_out (host, caller-owned) receives for pulse p the
 * n_measurements_p + 1 samples of j(t) at offset sum_{q<p}(n_measurements_q
 * + 1).  Synchronous.  The context keeps the plans (k table, pulse staging,
 * device buffers) of its last 4 distinct descriptor sets and reuses one when
 * a call repeats its descriptors byte for byte (explicit k rows and the
 * learned network compared by value); the integration runs every call. */
hhg_status hhg_gpu_current_density(hhg_ctx *ctx, const hhg_system_desc *sys,
                                   const hhg_pulse_desc *pulses, int n_pulses,
                                   const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                                   double *j_out, hhg_stats *stats);

/* TrapezoidalFFT::compute (sources/HHG/Fourier/TrapezoidalFFT.cpp:11-49) on
 * the x8 zero-padded j(t) (sources/hhg.cpp:36,277-285), on the device.
 * j has n_measurements + 1 samples on [t_begin, t_end]; re/im/freq receive
 * 4 (n_measurements + 1) + 1 values each (host, caller-owned). */
hhg_status hhg_gpu_spectrum(hhg_ctx *ctx, const double *j, int n_measurements, double t_begin,
                            double t_end, double *re_out, double *im_out, double *freq_out);

/* Plans: build the k table, pulse staging and work list once, then execute
 * on device-resident buffers.  Plans of one context built from the same
 * system and generated grid (not HHG_GRID_EXPLICIT rows, not the PiFlux-3D
 * cost-ordered tables of the NONE / CARRY proposers) share one read-only
 * device k table; the context keeps the last such table (n_k x 64 bytes)
 * until another system or grid replaces it or the context is destroyed. */
hhg_status hhg_plan_create(hhg_ctx *ctx, const hhg_system_desc *sys,
                           const hhg_pulse_desc *pulses, int n_pulses,
                           const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                           hhg_plan **plan);
void hhg_plan_destroy(hhg_plan *plan);
/* Total j samples over all pulses (length of a j buffer for this plan). */
int64_t hhg_plan_j_length(const hhg_plan *plan);
/* Launch the integration + reduction into the plan's device j buffer on
 * `stream` (a cudaStream_t, or NULL for the context stream).  Asynchronous. */
hhg_status hhg_plan_execute_async(hhg_plan *plan, void *stream);
/* Device pointer of the plan's j buffer (valid until hhg_plan_destroy). */
const double *hhg_plan_device_j(const hhg_plan *plan);
/* Synchronise, check the device status word and copy j to host. */
hhg_status hhg_plan_fetch(hhg_plan *plan, double *j_out, hhg_stats *stats);
/* TrapezoidalFFT of every pulse's device-resident j into plan-owned device
 * buffers (the device-side counterpart of hhg_gpu_spectrum).  Asynchronous. */
hhg_status hhg_plan_spectrum_async(hhg_plan *plan, void *stream);
/* Copy pulse `pulse`'s spectrum (4 (n_measurements + 1) + 1 values each) to
 * host.  Synchronous. */
hhg_status hhg_plan_fetch_spectrum(hhg_plan *plan, int pulse, double *re_out, double *im_out,
                                   double *freq_out);

/* The plan's execution (integration + reduction, and with with_spectrum != 0
 * the spectra) as one CUDA graph launch on `stream`.  The graph is captured
 * on the first call (and again after hhg_plan_autotune or when with_spectrum
 * changes) on the context's stream; it replaces hhg_plan_execute_async [+
 * hhg_plan_spectrum_async] and is read back with hhg_plan_fetch /
 * hhg_plan_fetch_spectrum (kernel_ms and total_ms: the whole graph launch).
 * No counterpart in the reference. */
hhg_status hhg_plan_execute_graph(hhg_plan *plan, void *stream, int with_spectrum);

/* Work-decomposition autotuner (no counterpart in the reference): times the
 * integration kernel over candidate k tiles per work item (32 k-points per
 * tile: 1, 2, 4, 8, 16) and persistent grid sizes (all resident CTAs, half),
 * `reps` timed runs each after one warm-up run, and keeps the fastest.  The
 * plan's results are unchanged by the choice (every candidate computes the
 * same trajectories; only the partial-row summation order changes). */
#define HHG_TUNE_MAX 16
typedef struct hhg_tune_report {
    int32_t n_candidates;
    int32_t best;
    int32_t tile_k[HHG_TUNE_MAX];
    int32_t grid[HHG_TUNE_MAX];
    double kernel_ms[HHG_TUNE_MAX];
} hhg_tune_report;
hhg_status hhg_plan_autotune(hhg_plan *plan, int reps, hhg_tune_report *report);

/* Diagnostic without a reference counterpart: measured FP64 FMA throughput
 * of the device (TFLOP/s, FMA = 2 flops), the denominator of the
 * integration kernel's roofline. */
hhg_status hhg_measure_fp64_peak(hhg_ctx *ctx, double *tflops);
/* The same for the FP32 pipe (the mixed-precision variant's denominator). */
hhg_status hhg_measure_fp32_peak(hhg_ctx *ctx, double *tflops);

/* Allocation-free variant of hhg_gpu_current_density for one pulse.  It has
 * no counterpart in the reference (which runs on the CPU).
 *
 * For callers that cannot allocate device memory during the call: code
 * running under another framework's memory pool or allocator hooks,
 * real-time loops where cudaMalloc's implicit synchronisation is not
 * acceptable, and jobs that budget every byte of a shared GPU.  The caller
 * passes the k table (n_rows x 8 doubles, the layout of hhg_grid_rows) and
 * receives j (n_measurements + 1 doubles), both in device memory.  The
 * integration scratch (pulse staging, partial current rows, counters) lives
 * in a fixed 64 MiB device array inside the library, so this call performs
 * no cudaMalloc/cudaFree and calls no allocating library routine; problems
 * whose scratch exceeds 64 MiB are rejected with HHG_BAD_CONFIG and a
 * message in err (e.g. 128x128 k rows over 8192 intervals fit).  Every GPU
 * on which the entry point is used holds the 64 MiB until the process exits.
 *
 * Runs asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) on the current device; it enqueues kernels only, so nothing it
 * enqueues reads host memory after it returns.  With stats != NULL it
 * synchronises the stream and reports HHG_STEP_LIMIT / HHG_NONFINITE like the
 * other entry points; with stats == NULL it returns after enqueueing, and
 * hhg_noalloc_status reports those conditions once the caller wants them.
 * The first call on a device looks up the scratch array's device address
 * (once per device, cached; the cache assumes the device's primary context
 * and no cudaDeviceReset for the life of the process); that first call must
 * come before any stream capture (HHG_UNSUPPORTED otherwise).  Later calls
 * may be captured into a CUDA graph with stats == NULL (they enqueue kernels
 * whose arguments are passed by value); with stats != NULL a capturing
 * stream is refused with HHG_UNSUPPORTED.  All calls share the one array, which keeps the
 * last call's contents: calls that overlap on the GPU race and must be
 * serialised by the caller.  Magnus-4 takes 1 to 4096 substeps, as in the
 * other entry points.  err (optional, err_cap bytes) receives a message on
 * failure. */
hhg_status hhg_gpu_current_density_noalloc(const hhg_system_desc *sys,
                                           const hhg_pulse_desc *pulse, const double *d_rows,
                                           int64_t n_rows, const hhg_solver_opts *opts,
                                           double *d_j_out, void *stream, hhg_stats *stats,
                                           char *err, size_t err_cap);
/* Outcome of the most recent hhg_gpu_current_density_noalloc call on the
 * current device, for callers that passed stats == NULL: synchronises
 * `stream` (the stream that call ran on), reads the counters and the status
 * word the call left in the shared scratch array, fills stats (optional) and
 * returns HHG_OK, HHG_STEP_LIMIT or HHG_NONFINITE as the call would have.
 * Another call on the device after it overwrites what this reads.  Not under
 * stream capture (HHG_UNSUPPORTED).  Allocates nothing; no counterpart in the
 * reference. */
hhg_status hhg_noalloc_status(void *stream, hhg_stats *stats, char *err, size_t err_cap);

/* Learned step-size proposer: collection, training and inference.  None has
 * a counterpart in the reference.
 *
 * hhg_learned_collect runs the integration with the carry controller in FP64
 * (opts' tolerances and limits; its proposer and precision are ignored) and
 * records, for every hist_every-th interval of each lane (staggered across
 * lanes), the interval's first attempt as one HHG_HIST_FIELDS record:
 * inputs, and T = log2(interval / h) - log2(0.9 / err) / 8 clamped to
 * [-1, 12].  Up to cap records go to `records` (host); n_records receives
 * the number written. */
hhg_status hhg_learned_collect(hhg_ctx *ctx, const hhg_system_desc *sys,
                               const hhg_pulse_desc *pulses, int n_pulses,
                               const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                               int hist_every, float *records, int64_t cap, int64_t *n_records,
                               hhg_stats *stats);
void hhg_default_train_opts(hhg_train_opts *opts);
/* Deterministic initial weights (uniform +-1/sqrt(fan_in), from `seed`) and,
 * when records != NULL, the input / output standardisation fitted to them
 * (mean and 1 / standard deviation per input; mean and standard deviation of
 * T).  level_margin is set to -0.5: a warp takes the largest of 32 lanes'
 * proposals, and the maximum of 32 noisy predictions sits above the largest
 * true level; at -0.5 the learned proposer takes the carried-level
 * heuristic's steps (at +0.25 it over-refined, 1.2-1.5x more steps). */
hhg_status hhg_mlp_init(uint64_t seed, const float *records, int64_t n_records, hhg_mlp *net);
/* Adam on the mean squared error of the standardised level, on the GPU: the
 * forward and backward GEMMs run on the tensor cores (tcgen05, BF16 inputs,
 * FP32 accumulation in tensor memory), Adam on FP32 master weights.  net
 * holds the initial weights and the standardisation on entry and the trained
 * weights on return.  epoch_loss (optional, epochs entries) receives the mean
 * batch loss of each epoch; train_ms (optional) the device time. */
hhg_status hhg_mlp_train(hhg_ctx *ctx, const float *records, int64_t n_records,
                         const hhg_train_opts *opts, hhg_mlp *net, float *epoch_loss,
                         double *train_ms);
/* Loss and its gradient with respect to params (HHG_MLP_N_PARAMS floats) over
 * n_records records (<= 1 << 20) as one batch, by the training kernels. */
hhg_status hhg_mlp_gradients(hhg_ctx *ctx, const float *records, int64_t n_records,
                             const hhg_mlp *net, float *grad_out, float *loss_out);
/* Predicted level T for n_records records: path 0 = the warp-level inference
 * used inside the integration kernel (mma.sync), path 1 = the training
 * forward pass (tcgen05). */
hhg_status hhg_mlp_predict(hhg_ctx *ctx, const float *records, int64_t n_records,
                           const hhg_mlp *net, int path, float *level_out);

/* k-resolved samples of one pulse: out[(i n_k + k) width + c] for every sample i
 * <= n_measurements and k-point k (host memory, (n_measurements + 1) n_k width
 * doubles), width 3 (HHG_KOUT_BLOCH), 2 (HHG_KOUT_OCCUPATIONS) or 1
 * (HHG_KOUT_CURRENT).  HHG_KOUT_CURRENT is the Dirac-3D system's: its debug
 * traces (DiracSystem::compute_current_density_debug and the relaxation twin,
 * DiracSystem.cpp:333-363, 427-457) are HHG_KOUT_CURRENT on
 * HHG_GRID_DIRAC3D_DEBUG, with the closed-form Magnus stepper (coherent) or FP64
 * RKF78 (relaxation), proposer NONE; a trajectory that failed reads 0.  The
 * reference's occupation tracking (PiFlux::evolve_occupation_numbers and
 * compute_occupation_numbers, PiFlux.cpp:222-318 and 909-953; the occupations
 * mode of hhg.cpp:120-168) is HHG_KOUT_OCCUPATIONS on
 * HHG_GRID_PIFLUX3D_OCCUPATION, with the z index of sample i shifted by
 * round(A(t_i) / dz) on the host.  PiFlux-3D only, FP64 RKF78, proposer NONE
 * or CARRY; a trajectory that failed reads NaN. */
hhg_status hhg_gpu_k_resolved(hhg_ctx *ctx, const hhg_system_desc *sys,
                              const hhg_pulse_desc *pulse, const hhg_grid_desc *grid,
                              const hhg_solver_opts *opts, int kind, double *out,
                              hhg_stats *stats);

/* The current split by the instantaneous band energy |d(k - A(t_i))| / 2t <
 * energy_cut (PiFlux::current_per_energy, PiFlux.cpp:955-1035; the
 * split_current mode of hhg.cpp:170-219, cut sqrt(3)/2): j_low and j_high,
 * n_measurements + 1 doubles each (host).  PiFlux-3D only, FP64 RKF78,
 * proposer NONE or CARRY. */
hhg_status hhg_gpu_split_current(hhg_ctx *ctx, const hhg_system_desc *sys,
                                 const hhg_pulse_desc *pulse, const hhg_grid_desc *grid,
                                 const hhg_solver_opts *opts, double energy_cut, double *j_low,
                                 double *j_high, hhg_stats *stats);

/* Drop-in for DiracSystem::compute_current_density (DiracSystem.cpp:271-331;
 * with sys->inv_diag_relax > 0 compute_current_density_diagonal_relaxation,
 * DiracSystem.cpp:365-425): j_out receives n_measurements + 1 doubles (host).
 * HHG_SYS_DIRAC3D only; opts->stepper HHG_STEPPER_DIRAC_MAGNUS (the
 * reference's coherent path, time_evolution_magnus) or HHG_STEPPER_RKF78 (the
 * sigma equation, time_evolution_sigma, and the relaxation path), FP64,
 * proposer NONE.  The new nodes of a level (of several levels, when they are
 * few) are integrated in one launch; the splits' estimates stay on the device
 * and take the levels one by one with the convergence test in between.  The
 * context keeps the plan and grow-only buffers for the next call with the same
 * system, pulse and options.  qstats and stats may be NULL; stats sums the
 * launches. */
hhg_status hhg_gpu_dirac_current_density(hhg_ctx *ctx, const hhg_system_desc *sys,
                                         const hhg_pulse_desc *pulse, const hhg_kappa_quad *quad,
                                         const hhg_solver_opts *opts, double *j_out,
                                         hhg_kappa_stats *qstats, hhg_stats *stats);

/* The continuous laser's spectrum (hhg.cpp:264-275): the first n_measurements
 * samples of j times the Welch window 1 - (i - N/2)^2 / (N^2/4)
 * (WelchWindow.hpp:11-13), an N-point r2c FFT (Fourier/FFT.cpp:8-42), and the
 * frequencies i / measure_every; N/2 + 1 values each (host). */
hhg_status hhg_gpu_spectrum_welch(hhg_ctx *ctx, const double *j, int n_measurements,
                                  double t_begin, double t_end, double *re_out, double *im_out,
                                  double *freq_out);

/* TrapezoidalFFT::compute (TrapezoidalFFT.cpp:11-49) of n_input samples as
 * given, without padding: delta_t = measure_every, [t_begin, t_end] the
 * TimeIntegrationConfig window, input[0] and input[n_input - 1] the end-point
 * samples.  This is the call hhg.cpp:287-290 makes on each debug trace
 * (n_input = n_measurements + 1).  re/im/freq receive n_input / 2 + 1 values
 * each (host, caller-owned). */
hhg_status hhg_gpu_trapezoidal_fft(hhg_ctx *ctx, const double *input, int64_t n_input,
                                   double delta_t, double t_begin, double t_end, double *re_out,
                                   double *im_out, double *freq_out);

/* A(t) of a pulse at n times (host only; Laser::laser_function as the engine
 * stages it, e.g. for the reference's laser_function output, hhg.cpp:301-305). */
hhg_status hhg_pulse_values(const hhg_pulse_desc *pulse, const double *t, int64_t n, double *A);

#ifdef __cplusplus
}
#endif
#endif
