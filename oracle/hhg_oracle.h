/*
 * hhg_oracle.h -- CPU FP64 restatement of the HigherHarmonics per-k-point
 * Bloch-integration path.  TEST INFRASTRUCTURE ONLY: the pytest suite, the
 * smoke check and the CPU-baseline leg of bench.py call it as the checker.
 * The product (libhhg_gpu.so) never links, loads or calls anything here.
 *
 * Parity status: the reference's time stepping lives in Boost.Odeint
 * (runge_kutta_fehlberg78 + controlled_runge_kutta + integrate_adaptive,
 * Boost 1.78 per cmake/user_settings.cmake:3), which is not present on this
 * machine and cannot be compiled with the reference.  The stepper here is
 * restated from Fehlberg's published 7(8) tableau (NASA TR R-287, 1968) and
 * the documented Boost.Odeint controller semantics.  The Gauss-Legendre
 * tables are pinned against the reference's own tables
 * (sources/HHG/thread_gauss.hpp) and the Magnus generator against the
 * reference's sympy derivation (helper/magnus_dirac.py); the RKF78 j(t) of
 * the reference itself is unpinned (no reference output exists).
 *
 * Units follow the reference (sources/HHG/Laser/Laser.hpp:13-16): time in
 * 1/omega_L, energies in hbar*omega_L, hbar = e = 1.
 */
#ifndef HHG_ORACLE_H
#define HHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_DIRAC2D = 0,       /* gapped 2D Dirac cone, d = (v(k-A)_x, v(k-A)_y, mass) */
    ORC_PIFLUX2D = 1,      /* square-lattice pi-flux, d = -2t(cos(kx-Ax), cos(ky-Ay), 0) */
    ORC_PIFLUX3D = 2,      /* reference PiFlux, d = 2t(cos kx, cos ky, cos(kz-A)) */
    ORC_HONEYCOMB = 3,     /* reference Honeycomb (+ optional staggered mass) */
    ORC_DIRAC3D = 4        /* reference DiracSystem sigma form, k = (k_z, kappa) */
};

enum { ORC_OK = 0, ORC_BAD_CONFIG = 1, ORC_STEP_LIMIT = 2, ORC_NONFINITE = 3 };

typedef struct {
    int kind;
    double hopping;      /* t in hbar*omega_L (PiFlux, Honeycomb) */
    double velocity;     /* v in hbar*omega_L per unit k (Dirac2D) */
    double mass;         /* staggered mass / gap term (Dirac2D, Honeycomb) */
    double pol_x, pol_y; /* field polarisation unit vector (cos theta, sin theta) */
    /* Thermal state and relaxation (PiFlux-3D, Honeycomb, Dirac-3D):
     * beta = photon_energy / (k_B T) with 0 standing for T = 0 (the
     * reference's beta = DBL_MAX sentinel, PiFlux.cpp:63), fermi_energy =
     * E_F / photon_energy, inv_*_relax = 1e15 hbar / (tau photon_energy)
     * (PiFlux.cpp:67-68); inv_diag_relax > 0 selects the relaxation
     * right-hand side (PiFlux.cpp:509-516, Honeycomb.cpp:214-223). */
    double beta;
    double fermi_energy;
    double inv_diag_relax;
    double inv_offdiag_relax;
} orc_model;

enum { ORC_PULSE_COSINE = 0, ORC_PULSE_CONTINUOUS = 1, ORC_PULSE_GAUSS = 2, ORC_PULSE_SPLINE = 3 };

typedef struct {
    double amplitude;    /* A0 = Laser::momentum_amplitude */
    double t_begin;      /* Laser::t_begin */
    double t_end;        /* Laser::t_end */
    double inv_n_cycles; /* CosineLaser::envelope_omega = 1/n_cycles */
    double phase;        /* carrier phase phi (0 in the reference) */
    int kind;            /* ORC_PULSE_*; 0 = the CosineLaser above */
    double gauss_center, gauss_sigma; /* GaussLaser (GaussLaser.cpp) */
    /* spline pulse: A = amplitude * s(t) for t <= t_end, 0 after; s through
     * spline_y[k] at t_begin + k spline_h with second derivatives spline_m
     * (orc_spline_moments) */
    const double *spline_y, *spline_m;
    int spline_n;
    double spline_h;
} orc_pulse;

typedef struct {
    double t_begin, t_end;
    int n_measurements, n_subdivisions;
} orc_time_config;

typedef struct {
    double abs_tol, rel_tol;
    int max_failed; /* Boost.Odeint failed_step_checker limit (500) */
    int stepper;    /* 0 = controlled RKF78, 1 = Magnus-4 (one step per sub-interval),
                     * 2 = the reference's Dirac-3D closed-form Magnus step per interval */
    int magnus_substeps;
} orc_solver;

typedef struct {
    uint64_t attempted, accepted, rejected, failed_k;
} orc_stats;

/* k table row: kx, ky, kz, weight, S0x, S0y, S0z, pad (8 doubles) */
#define ORC_KROW 8

/* Second derivatives M_k of the clamped cubic spline through y[0..n) at
 * spacing h with end slopes d0, dn (NaN: the one-sided five-point
 * difference): the moment equations of the interpolating cubic spline. */
void orc_spline_moments(const double *y, int n, double h, double d0, double dn, double *m);

double orc_laser(const orc_pulse *p, double t);
double orc_raw_laser(const orc_pulse *p, double t);

/* Gauss-Legendre: n nodes on [-1,1], ascending, and weights. */
void orc_gauss_legendre(int n, double *x, double *w);

/* Grids (write n rows of ORC_KROW doubles; return the row count).  A NULL
 * output pointer only returns the count. */
int orc_grid_tensor(const orc_model *m, int nx, int ny, double x_lo, double x_hi, double y_lo,
                    double y_hi, double *out);
int orc_grid_rhombic(const orc_model *m, int n1, int n2, double *out);
int orc_grid_piflux3d_ref(const orc_model *m, int z_range, int n_coarse, double *out);
int orc_grid_honeycomb_hex_ref(const orc_model *m, int n_k, double *out);

/* Initial Bloch vector: the reference's ic_sigma / Fermi-occupied state of
 * the reference models (T = 0, E_F = 0: the filled lower band, S0 = -d_hat);
 * the variant models take the filled lower band. */
void orc_initial_state(const orc_model *m, double kx, double ky, double kz, double *s0);

/* One k-point: Bloch vector at every sample (n_measurements+1 rows of 3). */
int orc_evolve_k(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                 const orc_solver *s, const double *krow, double *states, orc_stats *st);

/* Observable j contribution of one Bloch vector at sample time t (weight excluded). */
double orc_vertex(const orc_model *m, const orc_pulse *p, const double *krow, double t,
                  const double *S);

/* BZ sum j(t_i) = sum_k w_k vertex(k, A(t_i)) S(k, t_i), i = 0..n.  Fixed
 * reduction order (chunks of n_k/1024 in [1, 64] k-points, summed in
 * order), the same for any thread count. */
int orc_current_density(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                        const orc_solver *s, int n_k, const double *ktab, double *j_out,
                        orc_stats *st, int n_threads);

/* Step-size history of one k-point under the plain controller: for every
 * attempted step (t, dt, err, accepted).  Returns the count written (<= cap). */
int orc_step_history(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                     const orc_solver *s, const double *krow, int cap, double *hist);

/* k-resolved samples: kind 0 the Bloch vector (3 doubles), kind 1 the
 * reference's compute_occupations (PiFlux.cpp:227-235) at the shifted momentum
 * of update_equilibrium_state (PiFlux.cpp:252-258): (lower, upper).  out[(i n_k
 * + k) width + c].  PiFlux-3D rows. */
int orc_k_resolved(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                   const orc_solver *s, int n_k, const double *ktab, int kind, double *out,
                   int n_threads);

/* PiFlux::current_per_energy (PiFlux.cpp:955-1035): j split by the
 * instantaneous energy dispersion(k.shift_z(A(t_i))) < cut; weights from the
 * rows.  Fixed reduction order as orc_current_density. */
int orc_split_current(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                      const orc_solver *s, int n_k, const double *ktab, double cut,
                      double *j_low, double *j_high, int n_threads);

/* Reference Laser::magnus_coefficients (sources/HHG/Laser/Laser.cpp:40-55). */
void orc_magnus_coefficients(const orc_pulse *p, double delta_t, double t0, double *coeffs4);

/* Reference Magnus::Omega (sources/HHG/Systems/DiracDetail/MagnusMatrix.cpp:25-76):
 * returns the 3x3 row-major propagator U for the Dirac-3D sigma equation. */
void orc_dirac_magnus_U(double k, double kappa, double k_z, double delta_t,
                        const double *coeffs4, double *U9);

/* Reference DiracSystem::time_evolution_magnus (DiracSystem.cpp:176-211): S_z
 * at every sample for one (k_z, kappa). */
void orc_dirac3d_magnus_k(const orc_pulse *p, const orc_time_config *tc, double k_z,
                          double kappa, double *rhos);

/* Reference DiracSystem::time_evolution_sigma (DiracSystem.cpp:138-174). */
int orc_dirac3d_sigma_k(const orc_pulse *p, const orc_time_config *tc, const orc_solver *s,
                        double k_z, double kappa, double *rhos, orc_stats *st);

/* RKF78 tableau accessors (for the order-condition tests). */
void orc_rkf78_tableau(double *c13, double *a169, double *b13, double *db13);

#ifdef __cplusplus
}
#endif
#endif
