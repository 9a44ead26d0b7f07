/*
 * hhg_oracle.c -- CPU FP64 restatement of the reference's per-k-point Bloch
 * integration, Brillouin-zone current sum and Magnus propagators.
 *
 * TEST INFRASTRUCTURE ONLY (see hhg_oracle.h): used as the checker by the
 * tests, the smoke check and the CPU-baseline leg of bench.py; the product
 * never links it.
 *
 * Every routine cites the reference file:line whose behaviour it restates.
 * Reference paths are relative to the HigherHarmonics source tree.
 */
#include "hhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* Fehlberg 7(8) tableau (E. Fehlberg, NASA TR R-287, 1968).  This is the
 * tableau Boost.Odeint's runge_kutta_fehlberg78 implements; the propagated
 * solution is the 8th-order one, the error estimate is b8 - b7.            */
/* ------------------------------------------------------------------------ */
static const double RK_C[13] = {0.0,       2.0 / 27.0, 1.0 / 9.0, 1.0 / 6.0, 5.0 / 12.0,
                                1.0 / 2.0, 5.0 / 6.0,  1.0 / 6.0, 2.0 / 3.0, 1.0 / 3.0,
                                1.0,       0.0,        1.0};

/* Strictly lower triangular a_ij (row i = stage i, columns 0..i-1). */
static const double RK_A[13][12] = {
    {0},
    {2.0 / 27.0},
    {1.0 / 36.0, 1.0 / 12.0},
    {1.0 / 24.0, 0.0, 1.0 / 8.0},
    {5.0 / 12.0, 0.0, -25.0 / 16.0, 25.0 / 16.0},
    {1.0 / 20.0, 0.0, 0.0, 1.0 / 4.0, 1.0 / 5.0},
    {-25.0 / 108.0, 0.0, 0.0, 125.0 / 108.0, -65.0 / 27.0, 125.0 / 54.0},
    {31.0 / 300.0, 0.0, 0.0, 0.0, 61.0 / 225.0, -2.0 / 9.0, 13.0 / 900.0},
    {2.0, 0.0, 0.0, -53.0 / 6.0, 704.0 / 45.0, -107.0 / 9.0, 67.0 / 90.0, 3.0},
    {-91.0 / 108.0, 0.0, 0.0, 23.0 / 108.0, -976.0 / 135.0, 311.0 / 54.0, -19.0 / 60.0,
     17.0 / 6.0, -1.0 / 12.0},
    {2383.0 / 4100.0, 0.0, 0.0, -341.0 / 164.0, 4496.0 / 1025.0, -301.0 / 82.0,
     2133.0 / 4100.0, 45.0 / 82.0, 45.0 / 164.0, 18.0 / 41.0},
    {3.0 / 205.0, 0.0, 0.0, 0.0, 0.0, -6.0 / 41.0, -3.0 / 205.0, -3.0 / 41.0, 3.0 / 41.0,
     6.0 / 41.0, 0.0},
    {-1777.0 / 4100.0, 0.0, 0.0, -341.0 / 164.0, 4496.0 / 1025.0, -289.0 / 82.0,
     2193.0 / 4100.0, 51.0 / 82.0, 33.0 / 164.0, 12.0 / 41.0, 0.0, 1.0},
};

static const double RK_B[13] = {0.0,         0.0,        0.0,         0.0,         0.0,
                                34.0 / 105.0, 9.0 / 35.0, 9.0 / 35.0,  9.0 / 280.0, 9.0 / 280.0,
                                0.0,         41.0 / 840.0, 41.0 / 840.0};

static const double RK_DB[13] = {-41.0 / 840.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                                 -41.0 / 840.0, 41.0 / 840.0, 41.0 / 840.0};

void orc_rkf78_tableau(double *c13, double *a169, double *b13, double *db13) {
    for (int i = 0; i < 13; ++i) {
        c13[i] = RK_C[i];
        b13[i] = RK_B[i];
        db13[i] = RK_DB[i];
        for (int j = 0; j < 13; ++j) a169[13 * i + j] = (j < i) ? RK_A[i][j] : 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* Pulse: CosineLaser (sources/HHG/Laser/CosineLaser.cpp:22-26) inside
 * Laser::laser_function (sources/HHG/Laser/Laser.hpp:32-37, 51-53).  The
 * carrier phase is an addition for the synthetic pulse tables; 0 reproduces
 * the reference bit for bit.                                               */
/* ------------------------------------------------------------------------ */
static inline double cosine_envelope(const orc_pulse *p, double t) {
    if (t <= p->t_begin || t >= p->t_end) return 0.0;
    return 0.5 * (1. - cos(p->inv_n_cycles * (t - p->t_begin)));
}

void orc_spline_moments(const double *y, int n, double h, double d0, double dn, double *m) {
    if (isnan(d0)) d0 = (-25.0 * y[0] + 48.0 * y[1] - 36.0 * y[2] + 16.0 * y[3] - 3.0 * y[4]) / (12.0 * h);
    if (isnan(dn))
        dn = (25.0 * y[n - 1] - 48.0 * y[n - 2] + 36.0 * y[n - 3] - 16.0 * y[n - 4] + 3.0 * y[n - 5]) / (12.0 * h);
    /* 2 M_0 + M_1 = 6 ((y_1 - y_0)/h - d0)/h; M_(k-1) + 4 M_k + M_(k+1) =
     * 6 (y_(k+1) - 2 y_k + y_(k-1))/h^2; M_(n-2) + 2 M_(n-1) = 6 (dn - (y_(n-1)
     * - y_(n-2))/h)/h; solved by Gaussian elimination of the tridiagonal */
    double *cp = malloc(sizeof(double) * n), *dp = malloc(sizeof(double) * n);
    for (int k = 0; k < n; ++k) {
        double a = 1.0, b = 4.0, c = 1.0, r;
        if (k == 0) {
            a = 0.0, b = 2.0;
            r = 6.0 * ((y[1] - y[0]) / h - d0) / h;
        } else if (k == n - 1) {
            b = 2.0, c = 0.0;
            r = 6.0 * (dn - (y[n - 1] - y[n - 2]) / h) / h;
        } else {
            r = 6.0 * (y[k + 1] - 2.0 * y[k] + y[k - 1]) / (h * h);
        }
        const double den = k == 0 ? b : b - a * cp[k - 1];
        cp[k] = c / den;
        dp[k] = (k == 0 ? r : r - a * dp[k - 1]) / den;
    }
    m[n - 1] = dp[n - 1];
    for (int k = n - 2; k >= 0; --k) m[k] = dp[k] - cp[k] * m[k + 1];
    free(cp), free(dp);
}

/* s(t) on the piece of t (the first / last piece continued outside) */
static double spline_eval(const orc_pulse *p, double t) {
    const double h = p->spline_h;
    int k = (int)floor((t - p->t_begin) / h);
    if (k < 0) k = 0;
    if (k > p->spline_n - 2) k = p->spline_n - 2;
    const double a = (p->t_begin + (k + 1) * h) - t, b = t - (p->t_begin + k * h);
    const double *y = p->spline_y, *m = p->spline_m;
    return m[k] * a * a * a / (6.0 * h) + m[k + 1] * b * b * b / (6.0 * h) +
           (y[k] - m[k] * h * h / 6.0) * a / h + (y[k + 1] - m[k + 1] * h * h / 6.0) * b / h;
}

/* Laser::raw_laser_function (Laser.hpp:38-42): the CosineLaser, the
 * ContinuousLaser (envelope 1), the GaussLaser envelope
 * exp(-((t - c)(t - c)) / (2 s s)) (GaussLaser.cpp:36-38) or the spline,
 * which is 0 after t_end (Laser.hpp:35). */
double orc_raw_laser(const orc_pulse *p, double t) {
    switch (p->kind) {
    case ORC_PULSE_CONTINUOUS:
        return sin(t + p->phase);
    case ORC_PULSE_GAUSS: {
        const double x = t - p->gauss_center;
        return exp(-(x * x) / (2.0 * p->gauss_sigma * p->gauss_sigma)) * sin(t + p->phase);
    }
    case ORC_PULSE_SPLINE:
        return t > p->t_end ? 0.0 : spline_eval(p, t);
    default:
        return cosine_envelope(p, t) * sin(t + p->phase);
    }
}

double orc_laser(const orc_pulse *p, double t) { return p->amplitude * orc_raw_laser(p, t); }

/* ------------------------------------------------------------------------ */
/* Gauss-Legendre nodes by Newton iteration on P_n in long double.  The
 * reference ships Boost-generated tables (sources/HHG/thread_gauss.hpp:9-19
 * is the generator); the tests pin this routine against those tables.      */
/* ------------------------------------------------------------------------ */
void orc_gauss_legendre(int n, double *x, double *w) {
    const long double pi = 3.141592653589793238462643383279502884L;
    int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        long double z = cosl(pi * (i + 0.75L) / (n + 0.5L));
        long double pp = 0.0L;
        for (int it = 0; it < 100; ++it) {
            long double p1 = 1.0L, p2 = 0.0L;
            for (int j = 1; j <= n; ++j) {
                long double p3 = p2;
                p2 = p1;
                p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0L);
            long double dz = p1 / pp;
            z -= dz;
            if (fabsl(dz) < 1e-19L * (1.0L + fabsl(z))) {
                /* one more evaluation of the derivative at the converged node */
                p1 = 1.0L;
                p2 = 0.0L;
                for (int j = 1; j <= n; ++j) {
                    long double p3 = p2;
                    p2 = p1;
                    p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / j;
                }
                pp = n * (z * p1 - p2) / (z * z - 1.0L);
                break;
            }
        }
        long double wi = 2.0L / ((1.0L - z * z) * pp * pp);
        /* z is the i-th largest node */
        x[n - 1 - i] = (double)z;
        x[i] = (double)(-z);
        w[n - 1 - i] = (double)wi;
        w[i] = (double)wi;
    }
    if (n & 1) x[n / 2] = 0.0;
}

/* Positive half of a GL rule of order n, ascending: the reference's
 * gauss::container<n>::abscissa / weights layout (thread_gauss.hpp:24-311). */
static void gauss_half(int n, double *xa, double *wa) {
    double *x = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * n);
    orc_gauss_legendre(n, x, w);
    for (int i = 0; i < n / 2; ++i) {
        xa[i] = x[n / 2 + i];
        wa[i] = w[n / 2 + i];
    }
    free(x);
    free(w);
}

/* is_zero (sources/HHG/GlobalDefinitions.hpp:61-71): biased exponent below
 * 0b01111010011, i.e. |x| < 2^-44. */
static int ref_is_zero(double v) {
    uint64_t bits;
    memcpy(&bits, &v, sizeof bits);
    return (int)((bits >> 52) & 0x7FF) < 0x3D3;
}

/* ------------------------------------------------------------------------ */
/* Models: right-hand sides, initial states and current vertices.           */
/* ------------------------------------------------------------------------ */
static const double NN[3][2] = {{1.0, 0.0}, {-0.5, 0.5 * 1.732050807568877293527446341},
                                {-0.5, -0.5 * 1.732050807568877293527446341}};

typedef struct {
    double kx, ky, kz, cx, cy; /* cx/cy cache cos(kx), cos(ky) for the PiFlux-3D form */
    double s0[3];              /* initial Bloch vector (Dirac-3D relaxation target) */
} kctx;

static inline void cross(const double *m, const double *s, double *o) {
    /* cross_product (sources/HHG/GlobalDefinitions.hpp:49-55) */
    o[0] = m[1] * s[2] - m[2] * s[1];
    o[1] = m[2] * s[0] - m[0] * s[2];
    o[2] = m[0] * s[1] - m[1] * s[0];
}

/* fermi_function (sources/HHG/GlobalDefinitions.hpp:36-41); beta == 0
 * stands for the reference's T = 0 sentinel beta = numeric_limits::max(),
 * for which the function is a step with 1/2 at zero energy. */
static double fermi(double energy, double beta) {
    if (beta == 0.0) return energy != 0 ? (energy < 0 ? 1.0 : 0.0) : 0.5;
    return 1. / (1. + exp(beta * energy));
}

/* PiFlux::ic_sigma (PiFlux.cpp:519-549) with alpha^2 = occupation_a and
 * beta^2 = occupation_b (PiFlux.cpp:420-426) of the momentum (cx, cy, cz). */
static void piflux_ic(const orc_model *m, double cx, double cy, double cz, double *s0) {
    const double disp = sqrt(cx * cx + cy * cy + cz * cz);
    const double a2 = fermi(-m->fermi_energy + 2 * m->hopping * disp, m->beta);
    const double b2 = fermi(-m->fermi_energy - 2 * m->hopping * disp, m->beta);
    const double diff = a2 - b2;
    const double prod = 2 * sqrt(a2 * b2);
    const double zeps = cz + disp;
    s0[0] = (diff * cx * zeps + prod * (cy * cy + cz * zeps)) / (disp * zeps);
    s0[1] = (diff * cy * zeps - prod * cx * cy) / (disp * zeps);
    s0[2] = (diff * cz * zeps - prod * cx * zeps) / (disp * zeps);
}

/* Honeycomb::ic_sigma (Honeycomb.cpp:355-361) with occupation_a/b
 * (Honeycomb.cpp:347-353) at gamma = gre + i gim. */
static void honeycomb_ic(const orc_model *m, double gre, double gim, double *s0) {
    const double ag = hypot(gre, gim);
    const double a2 = fermi(m->fermi_energy - m->hopping * ag, m->beta);
    const double b2 = fermi(m->fermi_energy + m->hopping * ag, m->beta);
    const double diff = a2 - b2;
    const double prod = 2 * sqrt(a2 * b2);
    s0[0] = -diff * gre / ag;
    s0[1] = diff * gim / ag;
    s0[2] = -prod;
}

/* PiFlux::time_evolution_diagonal_relaxation right_side with its
 * update_equilibrium_state (PiFlux.cpp:113-186).  The equilibrium's
 * off-diagonal direction is taken from diagonal_sigma (PiFlux.cpp:1037-1048)
 * of the lambda's captured current_state, which Boost.Odeint's
 * controlled_runge_kutta::try_step holds at the step's start state while it
 * evaluates the stages (the new state is copied in only on acceptance): X. */
static void piflux_relax_rhs(const orc_model *m, const kctx *k, double A, const double *S,
                             const double *X, double *dS) {
    const double pf = 4 * m->hopping;
    double cx = k->cx, cy = k->cy, cz = cos(k->kz - A); /* shifted_k.update_z(k.z - A) */
    const double mv[3] = {k->cx, k->cy, cos(k->kz - A)};
    if (ref_is_zero(cx) && ref_is_zero(cy) && cz < 0.0) {
        cx = fabs(cz) * 1e-4; /* RESCUE_TRAFO (PiFlux.cpp:51, 136-139) */
        cz *= (1. - 0.5 * 1e-4 * 1e-4);
    }
    const double disp = sqrt(cx * cx + cy * cy + cz * cz);
    const double a2 = fermi(-m->fermi_energy + 2 * m->hopping * disp, m->beta);
    const double b2 = fermi(-m->fermi_energy - 2 * m->hopping * disp, m->beta);
    const double diff = a2 - b2;
    /* diagonal_sigma(current_state, shifted_k), components x and y */
    const double z = cz + disp;
    const double nrm = 2 * disp * z;
    const double xz = 2 * cx * z, yz = 2 * cy * z, xy = 2 * cx * cy;
    const double sg0 = (X[0] * (z * z - cx * cx + cy * cy) - xy * X[1] - xz * X[2]) / nrm;
    const double sg1 = (X[1] * (z * z + cx * cx - cy * cy) - xy * X[0] - yz * X[2]) / nrm;
    const double xyl = sqrt(sg0 * sg0 + sg1 * sg1);
    const double prod = 2 * sqrt(a2 * b2) * (ref_is_zero(xyl) ? 1.0 : sg0 / xyl);
    const double imag = 2 * sqrt(a2 * b2) * (ref_is_zero(xyl) ? 0.0 : sg1 / xyl);
    const double zeps = cz + disp;
    const double norm = disp * zeps;
    const double fd = diff * zeps / norm;
    const double rd[3] = {cx * fd, cy * fd, cz * fd};
    double ro[3];
    ro[0] = prod * (cy * cy + cz * zeps);
    ro[1] = prod * (-cx * cy);
    ro[2] = prod * (-cx * zeps);
    ro[0] += imag * (-cx * cy);
    ro[1] += imag * (cx * cx + cz * zeps);
    ro[2] += imag * (-cy * zeps);
    for (int i = 0; i < 3; ++i) ro[i] /= norm;
    cross(mv, S, dS);
    for (int i = 0; i < 3; ++i) {
        dS[i] *= pf;
        dS[i] -= m->inv_diag_relax * (S[i] / 3.0 - rd[i]) +
                 m->inv_offdiag_relax * (S[i] * (2. / 3.) - ro[i]);
    }
}

/* X: the step's start state (read by the PiFlux-3D relaxation form only). */
static void model_rhs(const orc_model *m, const kctx *k, const orc_pulse *p, double t,
                      const double *S, const double *X, double *dS) {
    const double A = orc_laser(p, t);
    const int relax = m->inv_diag_relax > 0.0;
    switch (m->kind) {
    case ORC_PIFLUX3D: {
        if (relax) {
            piflux_relax_rhs(m, k, A, S, X, dS);
            break;
        }
        /* PiFlux::time_evolution_sigma right_side (PiFlux.cpp:89-94) */
        const double pf = 4 * m->hopping;
        const double mv[3] = {k->cx, k->cy, cos(k->kz - A)};
        cross(mv, S, dS);
        for (int i = 0; i < 3; ++i) dS[i] *= pf;
        break;
    }
    case ORC_PIFLUX2D: {
        /* 2D pi-flux, d = -2t(cos(kx - A px), cos(ky - A py), 0): same
         * structure as PiFlux.cpp:89-94 with prefactor 2*(-2t). */
        const double pf = -4 * m->hopping;
        const double mv[3] = {cos(k->kx - m->pol_x * A), cos(k->ky - m->pol_y * A), 0.0};
        cross(mv, S, dS);
        for (int i = 0; i < 3; ++i) dS[i] *= pf;
        break;
    }
    case ORC_DIRAC2D: {
        /* gapped 2D Dirac: dS/dt = 2 d(k - A) x S */
        const double d[3] = {m->velocity * (k->kx - m->pol_x * A),
                             m->velocity * (k->ky - m->pol_y * A), m->mass};
        cross(d, S, dS);
        for (int i = 0; i < 3; ++i) dS[i] *= 2.0;
        break;
    }
    case ORC_HONEYCOMB: {
        /* Honeycomb::time_evolution_sigma right_side (Honeycomb.cpp:131-138)
         * with shifted_gamma (Honeycomb.cpp:41-47); the staggered-mass term
         * 2*mass*(-S_y, S_x, 0) is the gapped variant of the 512x512 rhombic
         * workload (mass 0 = the reference model). */
        const double pf = 2 * m->hopping;
        const double xs = m->pol_x * A, ys = m->pol_y * A;
        double gre = 0.0, gim = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double ph = NN[j][0] * (k->kx - xs) + NN[j][1] * (k->ky - ys);
            gre += cos(ph);
            gim += sin(ph);
        }
        dS[0] = -pf * (S[2] * gim);
        dS[1] = -pf * (S[2] * gre);
        dS[2] = pf * (S[0] * gim + S[1] * gre);
        if (m->mass != 0.0) {
            dS[0] -= 2.0 * m->mass * S[1];
            dS[1] += 2.0 * m->mass * S[0];
        }
        if (relax) {
            /* Honeycomb::time_evolution_diagonal_relaxation (Honeycomb.cpp:160-212):
             * dxdt -= 1/tau (state - ic_sigma(k - A)) */
            double eq[3];
            honeycomb_ic(m, gre, gim, eq);
            for (int i = 0; i < 3; ++i) dS[i] -= m->inv_diag_relax * (S[i] - eq[i]);
        }
        break;
    }
    case ORC_DIRAC3D: {
        /* DiracSystem::time_evolution_sigma right_side (DiracSystem.cpp:144-153);
         * kx = k_z, ky = kappa, kz = |k| */
        const double mx = A * 2.0 * k->ky / k->kz;
        const double mz = 2.0 * (k->kz - A * k->kx / k->kz);
        if (relax) {
            /* DiracSystem::time_evolution_diagonal_relaxation (DiracSystem.cpp:213-251):
             * relaxation towards the initial state */
            const double g = m->inv_diag_relax;
            dS[0] = mz * S[1] - (S[0] - k->s0[0]) * g;
            dS[1] = mx * S[2] - S[0] * mz - (S[1] - k->s0[1]) * g;
            dS[2] = -mx * S[1] - (S[2] - k->s0[2]) * g;
            break;
        }
        dS[0] = mz * S[1];
        dS[1] = mx * S[2] - S[0] * mz;
        dS[2] = -mx * S[1];
        break;
    }
    default:
        dS[0] = dS[1] = dS[2] = 0.0;
    }
}

double orc_vertex(const orc_model *m, const orc_pulse *p, const double *krow, double t,
                  const double *S) {
    const double A = orc_laser(p, t);
    switch (m->kind) {
    case ORC_PIFLUX3D:
        /* x_buffer[i] *= w_z * sin(k.z - A(t_i)) (PiFlux.cpp:832-838) */
        return sin(krow[2] - A) * S[2];
    case ORC_PIFLUX2D:
        return m->pol_x * sin(krow[0] - m->pol_x * A) * S[0] +
               m->pol_y * sin(krow[1] - m->pol_y * A) * S[1];
    case ORC_DIRAC2D:
        return m->pol_x * S[0] + m->pol_y * S[1];
    case ORC_HONEYCOMB: {
        /* shifted_grad_gamma + projection (Honeycomb.cpp:49-61, 273-279, 328-330) */
        const double xs = m->pol_x * A, ys = m->pol_y * A;
        double g0r = 0, g0i = 0, g1r = 0, g1i = 0;
        for (int j = 0; j < 3; ++j) {
            const double ph = NN[j][0] * (krow[0] - xs) + NN[j][1] * (krow[1] - ys);
            const double c = cos(ph), s = sin(ph);
            g0r += NN[j][0] * c;
            g0i += NN[j][0] * s;
            g1r += NN[j][1] * c;
            g1i += NN[j][1] * s;
        }
        const double bx = g0r * S[0] + g0i * S[1];
        const double by = g1r * S[0] + g1i * S[1];
        return bx * m->pol_x + by * m->pol_y;
    }
    case ORC_DIRAC3D:
        /* rhos = S_z; the k_z*kappa/|k| weight is folded into krow[3] */
        return S[2];
    }
    return 0.0;
}

void orc_initial_state(const orc_model *m, double kx, double ky, double kz, double *s0) {
    switch (m->kind) {
    case ORC_PIFLUX3D:
        /* ic_sigma (PiFlux.cpp:519-549); T = 0, E_F = 0: -(cx, cy, cz)/|d| */
        piflux_ic(m, cos(kx), cos(ky), cos(kz), s0);
        break;
    case ORC_PIFLUX2D: {
        const double cx = cos(kx), cy = cos(ky);
        const double n = sqrt(cx * cx + cy * cy);
        s0[0] = cx / n;
        s0[1] = cy / n;
        s0[2] = 0.0;
        break;
    }
    case ORC_DIRAC2D: {
        const double d0 = m->velocity * kx, d1 = m->velocity * ky, d2 = m->mass;
        const double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        s0[0] = -d0 / n;
        s0[1] = -d1 / n;
        s0[2] = -d2 / n;
        break;
    }
    case ORC_HONEYCOMB: {
        /* Honeycomb::ic_sigma at T = 0 (Honeycomb.cpp:355-361) */
        double gre = 0.0, gim = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double ph = NN[j][0] * kx + NN[j][1] * ky;
            gre += cos(ph);
            gim += sin(ph);
        }
        if (m->mass == 0.0) {
            honeycomb_ic(m, gre, gim, s0);
        } else {
            const double d0 = m->hopping * gre, d1 = -m->hopping * gim, d2 = m->mass;
            const double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            s0[0] = -d0 / n;
            s0[1] = -d1 / n;
            s0[2] = -d2 / n;
        }
        break;
    }
    case ORC_DIRAC3D: {
        /* (2 a0 b0, 0, a0^2 - b0^2), a0 = f(E_F + |k|), b0 = f(E_F - |k|)
         * (DiracSystem.cpp:155-158, dispersion :253-255); kx = k_z, ky = kappa */
        const double disp = sqrt(ky * ky + kx * kx);
        const double a0 = fermi(m->fermi_energy + disp, m->beta);
        const double b0 = fermi(m->fermi_energy - disp, m->beta);
        s0[0] = 2. * a0 * b0;
        s0[1] = 0.0;
        s0[2] = a0 * a0 - b0 * b0;
        break;
    }
    default:
        s0[0] = s0[1] = s0[2] = 0.0;
    }
}

static void fill_row(const orc_model *m, double kx, double ky, double kz, double w, double *row) {
    row[0] = kx;
    row[1] = ky;
    row[2] = kz;
    row[3] = w;
    orc_initial_state(m, kx, ky, kz, row + 4);
    row[7] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Grids                                                                    */
/* ------------------------------------------------------------------------ */
int orc_grid_tensor(const orc_model *m, int nx, int ny, double x_lo, double x_hi, double y_lo,
                    double y_hi, double *out) {
    const int n = nx * ny;
    if (!out) return n;
    double *gx = malloc(sizeof(double) * nx), *wx = malloc(sizeof(double) * nx);
    double *gy = malloc(sizeof(double) * ny), *wy = malloc(sizeof(double) * ny);
    orc_gauss_legendre(nx, gx, wx);
    orc_gauss_legendre(ny, gy, wy);
    const double hx = 0.5 * (x_hi - x_lo), mx = 0.5 * (x_hi + x_lo);
    const double hy = 0.5 * (y_hi - y_lo), my = 0.5 * (y_hi + y_lo);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            fill_row(m, hx * gx[i] + mx, hy * gy[j] + my, 0.0, hx * hy * wx[i] * wy[j],
                     out + (size_t)ORC_KROW * (i * ny + j));
    free(gx), free(wx), free(gy), free(wy);
    return n;
}

/* Rhombic BZ k = f1 b1 + f2 b2, f in [-1/2, 1/2]^2, b1 = 2pi/3 (1, -sqrt3),
 * b2 = 2pi/3 (1, sqrt3) for the reference's bond vectors (Honeycomb.hpp:23-27). */
int orc_grid_rhombic(const orc_model *m, int n1, int n2, double *out) {
    const int n = n1 * n2;
    if (!out) return n;
    const double s3 = 1.732050807568877293527446341;
    const double b1x = 2.0 * M_PI / 3.0, b1y = -2.0 * M_PI / 3.0 * s3;
    const double b2x = 2.0 * M_PI / 3.0, b2y = 2.0 * M_PI / 3.0 * s3;
    const double area = fabs(b1x * b2y - b1y * b2x);
    double *g1 = malloc(sizeof(double) * n1), *w1 = malloc(sizeof(double) * n1);
    double *g2 = malloc(sizeof(double) * n2), *w2 = malloc(sizeof(double) * n2);
    orc_gauss_legendre(n1, g1, w1);
    orc_gauss_legendre(n2, g2, w2);
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j) {
            const double f1 = 0.5 * g1[i], f2 = 0.5 * g2[j];
            fill_row(m, f1 * b1x + f2 * b2x, f1 * b1y + f2 * b2y, 0.0,
                     0.25 * area * w1[i] * w2[j], out + (size_t)ORC_KROW * (i * n2 + j));
        }
    free(g1), free(w1), free(g2), free(w2);
    return n;
}

/* PiFlux::current_density_continuum_limit + improved_xy_integral
 * (PiFlux.cpp:665-863).  The row weight is (w_x * transform_weight) * w_y * w_z.
 * The reference rescues the initial state of +k_z slices with cos k_z < 0
 * (PiFlux.cpp:812-816): the IC then uses cos k_z * (1 - 0.5e-8). */
typedef struct {
    double lo, hi;
    int nh;
} seg;

int orc_grid_piflux3d_ref(const orc_model *m, int z_range, int n_coarse, double *out) {
    const int n_fine = 8 * n_coarse;
    const int per_z = (2 * n_fine) * n_fine + (2 * 3 * n_coarse) * (2 * n_coarse) +
                      2 * (2 * n_coarse) * (2 * n_coarse);
    const int n = 2 * z_range * per_z;
    if (!out) return n;
    const double pi = M_PI;
    const double edge = 0.35 * pi;
    /* regions: x segment + its half order, y segment + its half order */
    const seg rx[4] = {{edge, pi - edge, n_fine}, {0.0, pi, 3 * n_coarse}, {0.0, edge, n_coarse},
                       {pi - edge, pi, n_coarse}};
    const seg ry[4] = {{edge, 0.5 * pi, n_fine / 2}, {0.0, edge, n_coarse},
                       {edge, 0.5 * pi, n_coarse}, {edge, 0.5 * pi, n_coarse}};
    double *za = malloc(sizeof(double) * z_range), *zw = malloc(sizeof(double) * z_range);
    gauss_half(2 * z_range, za, zw);
    size_t row = 0;
    double last_cx = 0.0, last_cy = 0.0;
    for (int z = 0; z < z_range; ++z) {
        for (int sgn = 0; sgn < 2; ++sgn) {
            const double kz = (sgn == 0 ? pi : -pi) * za[z];
            double cz = cos(kz);
            /* +z: fresh momentum_type (cos_x = cos_y = 0); -z: leftovers */
            const double chk_x = (sgn == 0) ? 0.0 : last_cx;
            const double chk_y = (sgn == 0) ? 0.0 : last_cy;
            if (ref_is_zero(chk_x) && ref_is_zero(chk_y) && cz < 0.0) cz *= (1. - 0.5 * 1e-4 * 1e-4);
            for (int r = 0; r < 4; ++r) {
                const int nxh = rx[r].nh, nyh = ry[r].nh;
                double *xa = malloc(sizeof(double) * nxh), *xw = malloc(sizeof(double) * nxh);
                double *ya = malloc(sizeof(double) * nyh), *yw = malloc(sizeof(double) * nyh);
                gauss_half(2 * nxh, xa, xw);
                gauss_half(2 * nyh, ya, yw);
                const double xh = 0.5 * (rx[r].hi - rx[r].lo), xm = 0.5 * (rx[r].hi + rx[r].lo);
                const double yh = 0.5 * (ry[r].hi - ry[r].lo), ym = 0.5 * (ry[r].hi + ry[r].lo);
                const double tw = xh * yh;
                for (int i = 0; i < nxh; ++i)
                    for (int sx = 0; sx < 2; ++sx) {
                        const double kx = xh * (sx ? -xa[i] : xa[i]) + xm;
                        const double mw = xw[i] * tw;
                        for (int j = 0; j < nyh; ++j)
                            for (int sy = 0; sy < 2; ++sy) {
                                const double ky = yh * (sy ? -ya[j] : ya[j]) + ym;
                                double *o = out + ORC_KROW * row++;
                                o[0] = kx;
                                o[1] = ky;
                                o[2] = kz;
                                o[3] = mw * yw[j] * zw[z];
                                /* ic_sigma with the (possibly rescued) cos_z */
                                const double cx = cos(kx), cy = cos(ky);
                                piflux_ic(m, cx, cy, cz, o + 4);
                                o[7] = 0.0;
                                last_cx = cx;
                                last_cy = cy;
                            }
                    }
                free(xa), free(xw), free(ya), free(yw);
            }
        }
    }
    free(za), free(zw);
    return (int)row;
}

/* Honeycomb::compute_current_density grid (Honeycomb.cpp:225-323). */
int orc_grid_honeycomb_hex_ref(const orc_model *m, int n_k, double *out) {
    const int n = 4 * n_k * n_k;
    if (!out) return n;
    const double pi = M_PI, s3 = 1.732050807568877293527446341;
    const double min_x = -2 * pi / 3, max_x = 2 * pi / 3;
    double *a = malloc(sizeof(double) * n_k), *w = malloc(sizeof(double) * n_k);
    gauss_half(2 * n_k, a, w);
    size_t row = 0;
    for (int x = 0; x < n_k; ++x) {
        const double kx0 = 0.5 * (max_x - min_x) * a[x] + 0.5 * (max_x + min_x);
        const double ymax = (4 * pi / (3 * s3)) - (fabs(kx0) / s3);
        for (int sx = 0; sx < 2; ++sx) {
            const double kx = sx ? (0.5 * (max_x - min_x) * (-a[x]) + 0.5 * (max_x + min_x)) : kx0;
            for (int y = 0; y < n_k; ++y) {
                const double tw = 0.5 * (max_x - min_x) * (0.5 * (ymax - (-ymax))) * w[x] * w[y];
                for (int sy = 0; sy < 2; ++sy) {
                    const double ay = sy ? -a[y] : a[y];
                    const double ky = 0.5 * (ymax - (-ymax)) * ay + 0.5 * (ymax + (-ymax));
                    fill_row(m, kx, ky, 0.0, tw, out + ORC_KROW * row++);
                }
            }
        }
    }
    free(a), free(w);
    return (int)row;
}

/* ------------------------------------------------------------------------ */
/* Controlled RKF78 over one output interval: the semantics of
 * integrate_adaptive(make_controlled<runge_kutta_fehlberg78>(abs, rel), ...)
 * as called at PiFlux.cpp:104-110 / Honeycomb.cpp:150-157 /
 * DiracSystem.cpp:166-172.
 *  - every attempt evaluates dxdt at (x, t) and 12 further stages;
 *  - err = max_i |xerr_i| / (abs + rel (|x_i| + dt |dxdt_i|));
 *  - err > 1: reject, dt *= max(0.9 err^(-1/6), 0.2);
 *  - else accept, and if err < 0.5: dt *= 0.9 max(err, 5^-8)^(-1/8);
 *  - the step is clipped to land on t_end; the loop runs while
 *    t_end - t > DBL_EPSILON (absolute, as Boost's less_with_sign);
 *  - 500 consecutive rejections abort (failed_step_checker).              */
/* ------------------------------------------------------------------------ */
typedef struct {
    const orc_model *m;
    const kctx *k;
    const orc_pulse *p;
} rhs_ctx;

static int rkf78_try(const rhs_ctx *c, double *x, double *t, double *dt, double abs_tol,
                     double rel_tol, double *err_out) {
    double K[13][3];
    double xt[3];
    model_rhs(c->m, c->k, c->p, *t, x, x, K[0]);
    const double h = *dt;
    for (int s = 1; s < 13; ++s) {
        for (int i = 0; i < 3; ++i) {
            double acc = 1.0 * x[i];
            for (int j = 0; j < s; ++j)
                if (RK_A[s][j] != 0.0) acc += (RK_A[s][j] * h) * K[j][i];
            xt[i] = acc;
        }
        model_rhs(c->m, c->k, c->p, *t + RK_C[s] * h, xt, x, K[s]);
    }
    double xn[3], err = 0.0;
    for (int i = 0; i < 3; ++i) {
        double acc = 1.0 * x[i];
        double e = 0.0;
        int first = 1;
        for (int j = 0; j < 13; ++j) {
            if (RK_B[j] != 0.0) acc += (RK_B[j] * h) * K[j][i];
            if (RK_DB[j] != 0.0) {
                if (first) {
                    e = (RK_DB[j] * h) * K[j][i];
                    first = 0;
                } else
                    e += (RK_DB[j] * h) * K[j][i];
            }
        }
        xn[i] = acc;
        const double r = fabs(e) / (abs_tol + rel_tol * (1.0 * fabs(x[i]) + (1.0 * h) * fabs(K[0][i])));
        if (r > err) err = r;
    }
    *err_out = err;
    if (err > 1.0) {
        double f = 9.0 / 10.0 * pow(err, -1.0 / (7 - 1));
        if (f < 1.0 / 5.0) f = 1.0 / 5.0;
        *dt = h * f;
        return 0;
    }
    *t += h;
    for (int i = 0; i < 3; ++i) x[i] = xn[i];
    if (err < 0.5) {
        double e2 = pow(5.0, -8.0);
        if (err > e2) e2 = err;
        *dt = h * (9.0 / 10.0 * pow(e2, -1.0 / 8));
    }
    return 1;
}

static int integrate_interval(const rhs_ctx *c, double *x, double t0, double t1, double dt,
                              const orc_solver *s, orc_stats *st, double *hist, int *nh,
                              int cap) {
    const double eps = 2.220446049250313080847e-16;
    double t = t0;
    while (t1 - t > eps) {
        if ((t + dt) - t1 > eps) dt = t1 - t;
        int fails = 0;
        for (;;) {
            double err;
            const double t_before = t, dt_before = dt;
            const int ok = rkf78_try(c, x, &t, &dt, s->abs_tol, s->rel_tol, &err);
            st->attempted++;
            if (hist && *nh < cap) {
                double *hrow = hist + 4 * (*nh);
                hrow[0] = t_before;
                hrow[1] = dt_before;
                hrow[2] = err;
                hrow[3] = ok;
                (*nh)++;
            }
            if (ok) {
                st->accepted++;
                break;
            }
            st->rejected++;
            if (++fails >= s->max_failed) return ORC_STEP_LIMIT;
        }
        if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]))) return ORC_NONFINITE;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Magnus-4 (two-point Gauss, one step per sub-interval) for dS/dt = 2 d x S:
 * omega = h (d1 + d2) + (sqrt3/3) h^2 (d2 x d1), S <- exp([omega]_x) S.
 * Not a reference path: the 4th-order Magnus variant of the honeycomb
 * workload; the
 * reference's general so(3) Magnus (GeneralMagnus.cpp) is its design source. */
/* ------------------------------------------------------------------------ */
static void dvec(const orc_model *m, const kctx *k, const orc_pulse *p, double t, double *d) {
    const double A = orc_laser(p, t);
    switch (m->kind) {
    case ORC_DIRAC2D:
        d[0] = m->velocity * (k->kx - m->pol_x * A);
        d[1] = m->velocity * (k->ky - m->pol_y * A);
        d[2] = m->mass;
        break;
    case ORC_PIFLUX2D:
        d[0] = -2 * m->hopping * cos(k->kx - m->pol_x * A);
        d[1] = -2 * m->hopping * cos(k->ky - m->pol_y * A);
        d[2] = 0.0;
        break;
    case ORC_PIFLUX3D:
        d[0] = 2 * m->hopping * k->cx;
        d[1] = 2 * m->hopping * k->cy;
        d[2] = 2 * m->hopping * cos(k->kz - A);
        break;
    case ORC_HONEYCOMB: {
        const double xs = m->pol_x * A, ys = m->pol_y * A;
        double gre = 0.0, gim = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double ph = NN[j][0] * (k->kx - xs) + NN[j][1] * (k->ky - ys);
            gre += cos(ph);
            gim += sin(ph);
        }
        d[0] = m->hopping * gre;
        d[1] = -m->hopping * gim;
        d[2] = m->mass;
        break;
    }
    default:
        d[0] = d[1] = d[2] = 0.0;
    }
}

static void rotate(const double *w, double *S) {
    const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double th = sqrt(th2);
    double sa, ca; /* sin(th)/th, (1-cos th)/th^2 */
    if (th < 1e-4) {
        sa = 1.0 - th2 / 6.0 + th2 * th2 / 120.0;
        ca = 0.5 - th2 / 24.0 + th2 * th2 / 720.0;
    } else {
        sa = sin(th) / th;
        ca = (1.0 - cos(th)) / th2;
    }
    double wx[3];
    cross(w, S, wx);
    double wwx[3];
    cross(w, wx, wwx);
    for (int i = 0; i < 3; ++i) S[i] += sa * wx[i] + ca * wwx[i];
}

static void magnus4_interval(const orc_model *m, const kctx *k, const orc_pulse *p, double t0,
                             double t1, int nsub, double *S) {
    const double h = (t1 - t0) / nsub;
    const double g = 0.5 - 0.28867513459481288225; /* 1/2 - sqrt3/6 */
    for (int s = 0; s < nsub; ++s) {
        const double ts = t0 + s * h;
        double d1[3], d2[3], c[3], w[3];
        dvec(m, k, p, ts + g * h, d1);
        dvec(m, k, p, ts + (1.0 - g) * h, d2);
        cross(d2, d1, c);
        const double q = 0.57735026918962576451 * h * h; /* sqrt3/3 h^2 */
        for (int i = 0; i < 3; ++i) w[i] = h * (d1[i] + d2[i]) + q * c[i];
        rotate(w, S);
    }
}

/* ------------------------------------------------------------------------ */
/* Per-k evolution over the reference's measurement loop                    */
/* (PiFlux.cpp:96-110): t_begin, t_end = t_begin + measure_every, ...        */
/* ------------------------------------------------------------------------ */
static void make_kctx(const double *krow, kctx *k) {
    k->kx = krow[0];
    k->ky = krow[1];
    k->kz = krow[2];
    k->cx = cos(krow[0]);
    k->cy = cos(krow[1]);
    k->s0[0] = krow[4];
    k->s0[1] = krow[5];
    k->s0[2] = krow[6];
}

typedef void (*sample_fn)(void *user, int i, const double *S);

static int evolve_generic(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                          const orc_solver *s, const double *krow, orc_stats *st, sample_fn fn,
                          void *user, double *hist, int *nh, int cap) {
    kctx k;
    make_kctx(krow, &k);
    const rhs_ctx c = {m, &k, p};
    double S[3] = {krow[4], krow[5], krow[6]};
    const double measure_every = (tc->t_end - tc->t_begin) / tc->n_measurements;
    const double dt = measure_every / tc->n_subdivisions;
    double t_begin = tc->t_begin;
    double t_end = t_begin + measure_every;
    fn(user, 0, S);
    if (s->stepper == 2 && m->kind != ORC_DIRAC3D) return ORC_BAD_CONFIG;
    for (int i = 1; i <= tc->n_measurements; ++i) {
        if (s->stepper == 1) {
            magnus4_interval(m, &k, p, t_begin, t_end, s->magnus_substeps, S);
            st->attempted += s->magnus_substeps;
            st->accepted += s->magnus_substeps;
        } else if (s->stepper == 2) {
            /* DiracSystem::time_evolution_magnus (DiracSystem.cpp:190-210) on the
             * row's (k_z, kappa, |k|) and initial state */
            double cf[4], U[9];
            orc_magnus_coefficients(p, measure_every, t_begin, cf);
            for (int q = 0; q < 4; ++q) cf[q] /= k.kz;
            orc_dirac_magnus_U(2 * k.kz, 2 * k.ky, 2 * k.kx, measure_every, cf, U);
            const double s0 = U[0] * S[0] + U[1] * S[1] + U[2] * S[2];
            const double s1 = U[3] * S[0] + U[4] * S[1] + U[5] * S[2];
            const double s2 = U[6] * S[0] + U[7] * S[1] + U[8] * S[2];
            S[0] = s0, S[1] = s1, S[2] = s2;
            st->attempted++;
            st->accepted++;
        } else {
            const int rc = integrate_interval(&c, S, t_begin, t_end, dt, s, st, hist, nh, cap);
            if (rc != ORC_OK) return rc;
        }
        fn(user, i, S);
        t_begin = t_end;
        t_end += measure_every;
    }
    return ORC_OK;
}

typedef struct {
    double *states;
} store_user;

static void store_states(void *u, int i, const double *S) {
    double *o = ((store_user *)u)->states + 3 * (size_t)i;
    o[0] = S[0];
    o[1] = S[1];
    o[2] = S[2];
}

int orc_evolve_k(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                 const orc_solver *s, const double *krow, double *states, orc_stats *st) {
    store_user u = {states};
    return evolve_generic(m, p, tc, s, krow, st, store_states, &u, NULL, NULL, 0);
}

static void no_store(void *u, int i, const double *S) {
    (void)u, (void)i, (void)S;
}

int orc_step_history(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                     const orc_solver *s, const double *krow, int cap, double *hist) {
    orc_stats st = {0, 0, 0, 0};
    int nh = 0;
    const int rc = evolve_generic(m, p, tc, s, krow, &st, no_store, NULL, hist, &nh, cap);
    return rc == ORC_OK ? nh : -rc;
}

typedef struct {
    const orc_model *m;
    const orc_pulse *p;
    const double *krow;
    const double *t_samples;
    double *acc;
} acc_user;

static void accumulate(void *u, int i, const double *S) {
    acc_user *a = (acc_user *)u;
    a->acc[i] += a->krow[3] * orc_vertex(a->m, a->p, a->krow, a->t_samples[i], S);
}

int orc_current_density(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                        const orc_solver *s, int n_k, const double *ktab, double *j_out,
                        orc_stats *st, int n_threads) {
    const int ns = tc->n_measurements + 1;
    /* chunk size depends on n_k only (so the sum is the same for any thread
     * count) and keeps >= 1024 chunks for load balance on many cores */
    int chunk = n_k / 1024;
    if (chunk < 1) chunk = 1;
    if (chunk > 64) chunk = 64;
    const int n_chunks = (n_k + chunk - 1) / chunk;
    const double measure_every = (tc->t_end - tc->t_begin) / tc->n_measurements;
    double *t_samples = malloc(sizeof(double) * ns);
    /* sample times i * time_step + t_begin (PiFlux.cpp:834-836) */
    for (int i = 0; i < ns; ++i) t_samples[i] = i * measure_every + tc->t_begin;
    double *part = calloc((size_t)n_chunks * ns, sizeof(double));
    int status = ORC_OK;
    uint64_t att = 0, acc_n = 0, rej = 0, failed = 0;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads) reduction(+ : att, acc_n, rej, failed)
#endif
    for (int c = 0; c < n_chunks; ++c) {
        double *buf = part + (size_t)c * ns;
        for (int q = c * chunk; q < n_k && q < (c + 1) * chunk; ++q) {
            orc_stats ls = {0, 0, 0, 0};
            acc_user u = {m, p, ktab + (size_t)ORC_KROW * q, t_samples, buf};
            const int rc = evolve_generic(m, p, tc, s, u.krow, &ls, accumulate, &u, NULL, NULL, 0);
            att += ls.attempted;
            acc_n += ls.accepted;
            rej += ls.rejected;
            if (rc != ORC_OK) {
                failed++;
#ifdef _OPENMP
#pragma omp critical
#endif
                status = rc;
            }
        }
    }
    for (int i = 0; i < ns; ++i) j_out[i] = 0.0;
    for (int c = 0; c < n_chunks; ++c)
        for (int i = 0; i < ns; ++i) j_out[i] += part[(size_t)c * ns + i];
    free(part);
    free(t_samples);
    if (st) {
        st->attempted += att;
        st->accepted += acc_n;
        st->rejected += rej;
        st->failed_k += failed;
    }
    (void)n_threads;
    return status;
}

/* ------------------------------------------------------------------------ */
/* k-resolved samples and the energy-split current (PiFlux)                  */
/* ------------------------------------------------------------------------ */
/* diagonal_sigma (PiFlux.cpp:1037-1048) at the momentum cosines (cx, cy, cz) */
static void diagonal_sigma(const double *in, double cx, double cy, double cz, double *o) {
    const double disp = sqrt(cx * cx + cy * cy + cz * cz);
    const double z = cz + disp;
    const double norm = 2 * disp * z;
    const double xz = 2 * cx * z, yz = 2 * cy * z, xy = 2 * cx * cy;
    o[0] = (in[0] * (z * z - cx * cx + cy * cy) - xy * in[1] - xz * in[2]) / norm;
    o[1] = (in[1] * (z * z + cx * cx - cy * cy) - xy * in[0] - yz * in[2]) / norm;
    o[2] = (in[2] * (z * z - cx * cx - cy * cy) + xz * in[0] + yz * in[1]) / norm;
}

int orc_k_resolved(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                   const orc_solver *s, int n_k, const double *ktab, int kind, double *out,
                   int n_threads) {
    const int ns = tc->n_measurements + 1;
    const int width = kind == 0 ? 3 : 2;
    const double me = (tc->t_end - tc->t_begin) / tc->n_measurements;
    int status = ORC_OK;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int q = 0; q < n_k; ++q) {
        const double *krow = ktab + (size_t)ORC_KROW * q;
        double *states = malloc(sizeof(double) * 3 * ns);
        orc_stats st = {0, 0, 0, 0};
        const int rc = orc_evolve_k(m, p, tc, s, krow, states, &st);
        if (rc != ORC_OK) {
#ifdef _OPENMP
#pragma omp critical
#endif
            status = rc;
        }
        for (int i = 0; i < ns; ++i) {
            const double *S = states + 3 * i;
            double *o = out + ((size_t)i * n_k + q) * width;
            if (kind == 0) {
                o[0] = S[0], o[1] = S[1], o[2] = S[2];
                continue;
            }
            /* shifted_k.update_z(k.z - A) with the rescue of update_equilibrium_state */
            const double A = orc_laser(p, i * me + tc->t_begin);
            double cx = cos(krow[0]), cy = cos(krow[1]), cz = cos(krow[2] - A);
            if (ref_is_zero(cx) && ref_is_zero(cy) && cz < 0.0) {
                cx = fabs(cz) * 1e-4;
                cz *= (1. - 0.5 * 1e-4 * 1e-4);
            }
            double d[3];
            diagonal_sigma(S, cx, cy, cz, d);
            const double n = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            o[0] = sqrt(0.5 * (-d[2] + n));
            o[1] = sqrt(0.5 * (d[2] + n));
        }
        free(states);
    }
    (void)n_threads;
    return status;
}

typedef struct {
    const orc_pulse *p;
    const double *krow;
    const double *t_samples;
    double cut;
    double *lo, *hi;
} split_user;

static void accumulate_split(void *u, int i, const double *S) {
    split_user *a = (split_user *)u;
    const double A = orc_laser(a->p, a->t_samples[i]);
    const double cx = cos(a->krow[0]), cy = cos(a->krow[1]), cz = cos(a->krow[2] - A);
    const double energy = sqrt(cx * cx + cy * cy + cz * cz); /* dispersion(k.shift_z(A)) */
    const double v = a->krow[3] * (S[2] * sin(a->krow[2] - A));
    if (energy < a->cut) a->lo[i] += v;
    else a->hi[i] += v;
}

int orc_split_current(const orc_model *m, const orc_pulse *p, const orc_time_config *tc,
                      const orc_solver *s, int n_k, const double *ktab, double cut,
                      double *j_low, double *j_high, int n_threads) {
    const int ns = tc->n_measurements + 1;
    int chunk = n_k / 1024;
    if (chunk < 1) chunk = 1;
    if (chunk > 64) chunk = 64;
    const int n_chunks = (n_k + chunk - 1) / chunk;
    const double me = (tc->t_end - tc->t_begin) / tc->n_measurements;
    double *t_samples = malloc(sizeof(double) * ns);
    for (int i = 0; i < ns; ++i) t_samples[i] = i * me + tc->t_begin;
    double *part = calloc((size_t)2 * n_chunks * ns, sizeof(double));
    int status = ORC_OK;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int c = 0; c < n_chunks; ++c) {
        for (int q = c * chunk; q < n_k && q < (c + 1) * chunk; ++q) {
            orc_stats ls = {0, 0, 0, 0};
            split_user u = {p, ktab + (size_t)ORC_KROW * q, t_samples, cut,
                            part + (size_t)(2 * c) * ns, part + (size_t)(2 * c + 1) * ns};
            const int rc = evolve_generic(m, p, tc, s, u.krow, &ls, accumulate_split, &u, NULL, NULL, 0);
            if (rc != ORC_OK) {
#ifdef _OPENMP
#pragma omp critical
#endif
                status = rc;
            }
        }
    }
    for (int i = 0; i < ns; ++i) j_low[i] = j_high[i] = 0.0;
    for (int c = 0; c < n_chunks; ++c)
        for (int i = 0; i < ns; ++i) {
            j_low[i] += part[(size_t)(2 * c) * ns + i];
            j_high[i] += part[(size_t)(2 * c + 1) * ns + i];
        }
    free(part);
    free(t_samples);
    (void)n_threads;
    return status;
}

/* ------------------------------------------------------------------------ */
/* Reference Dirac-3D Magnus path                                           */
/* ------------------------------------------------------------------------ */
/* 30-point Gauss-Legendre on [0,1] in the reference's node order
 * (sources/HHG/Laser/gauss.hpp:14-80): negative nodes by increasing |x|,
 * then positive nodes increasing; shifted Legendre values as gauss.hpp:82-101
 * computes them, including its legendre_4 = 20x^3 - 30x^2 + 12x + 1. */
/* The 30-point rule on [0, 1] in the reference's order (gauss.hpp:14-80:
 * negative nodes by increasing |x|, then the positive ones), computed once at
 * load time as the reference's tables are compile-time constants. */
static double gl30_ab[30], gl30_wt[30];

__attribute__((constructor)) static void gl30_init(void) {
    double x[30], w[30];
    orc_gauss_legendre(30, x, w);
    for (int i = 0; i < 15; ++i) {
        const double xi = x[15 + i]; /* i-th positive node, ascending */
        gl30_ab[i] = 0.5 * (-xi + 1.);
        gl30_ab[15 + i] = 0.5 * (xi + 1.);
        gl30_wt[i] = 0.5 * w[15 + i];
        gl30_wt[15 + i] = 0.5 * w[15 + i];
    }
}

void orc_magnus_coefficients(const orc_pulse *p, double delta_t, double t0, double *coeffs) {
    const double *ab = gl30_ab, *wt = gl30_wt;
    double c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (int i = 0; i < 30; ++i) {
        const double a = ab[i];
        const double l2 = 2. * a - 1.;
        const double l3 = 6. * a * (a - 1.) + 1.;
        const double l4 = 20. * a * a * a - 30. * a * a + 12. * a + 1.;
        const double lv = orc_raw_laser(p, t0 + delta_t * a);
        c0 += wt[i] * lv;
        c1 += wt[i] * l2 * lv;
        c2 += wt[i] * l3 * lv;
        c3 += wt[i] * l4 * lv;
    }
    coeffs[0] = c0 * p->amplitude;
    coeffs[1] = c1 * (3. * p->amplitude);
    coeffs[2] = c2 * (5. * p->amplitude);
    coeffs[3] = c3 * (7. * p->amplitude);
}

/* Magnus generator of helper/magnus_dirac.py evaluated on axial vectors: for
 * 3x3 skew matrices [x]_x, the commutator [[x]_x, [y]_x] = [x cross y]_x, so
 * every nested commutator of the series is a nested cross product.  With
 * H <-> h = (0, 0, k), A <-> a = (kappa, 0, -k_z) and M1 = H + alpha A,
 * M2..M4 = (beta, gamma, delta) A, the reference's Omega is [omega]_x and its
 * (a, b, c) entries (MagnusMatrix.cpp:35-57) are (-omega_2, omega_1,
 * -omega_0).  U = exp(Omega) as MagnusMatrix.cpp:59-75. */
static void cr(const double *a, const double *b, double *o) { cross(a, b, o); }

void orc_dirac_magnus_U(double k, double kappa, double k_z, double delta_t, const double *cf,
                        double *U) {
    const double ks = k * delta_t, kap = kappa * delta_t, kzs = k_z * delta_t;
    const double h[3] = {0.0, 0.0, ks};
    const double av[3] = {kap, 0.0, -kzs};
    double m1[3], m2[3], m3[3], m4[3];
    for (int i = 0; i < 3; ++i) {
        m1[i] = h[i] + cf[0] * av[i];
        m2[i] = cf[1] * av[i];
        m3[i] = cf[2] * av[i];
        m4[i] = cf[3] * av[i];
    }
    double c12[3], c13[3], c14[3], c112[3], c113[3];
    cr(m1, m2, c12);
    cr(m1, m3, c13);
    cr(m1, m4, c14);
    cr(m1, c12, c112);
    cr(m1, c13, c113);
    double t1[3], t2[3], t3[3], om[3];
    for (int i = 0; i < 3; ++i) om[i] = m1[i] - c12[i] / 6.0;
#define ADD(coef, v)                                           \
    for (int i = 0; i < 3; ++i) om[i] += (coef) * (v)[i];
    cr(m2, c12, t1);
    ADD(-1.0 / 60.0, t1);
    cr(m1, c112, t1);
    ADD(1.0 / 360.0, t1);
    cr(m2, c14, t1);
    ADD(1.0 / 140.0, t1);
    cr(m3, c13, t1);
    ADD(-1.0 / 420.0, t1);
    cr(m4, c12, t1);
    ADD(-1.0 / 210.0, t1);
    cr(m1, c14, t2);
    cr(m1, t2, t1);
    ADD(-1.0 / 840.0, t1);
    cr(m2, c113, t1);
    ADD(1.0 / 504.0, t1);
    cr(m2, c12, t2);
    cr(m2, t2, t1);
    ADD(-1.0 / 840.0, t1);
    cr(m3, c112, t1);
    ADD(1.0 / 2520.0, t1);
    cr(m1, c113, t2);
    cr(m1, t2, t1);
    ADD(-1.0 / 2520.0, t1);
    cr(c12, c112, t1);
    ADD(-1.0 / 7560.0, t1);
    cr(m1, c112, t2);
    cr(m2, t2, t1);
    ADD(1.0 / 2520.0, t1);
    cr(m1, c112, t3);
    cr(m1, t3, t2);
    cr(m1, t2, t1);
    ADD(-1.0 / 15120.0, t1);
#undef ADD
    const double a = -om[2], b = om[1], c = -om[0];
    const double n2 = a * a + b * b + c * c;
    const double ev = sqrt(n2);
    const double x = cos(ev), y = sin(ev);
    U[0] = ((a * a + b * b) * x + c * c) / n2;
    U[1] = (b * c * (x - 1) + a * ev * y) / n2;
    U[2] = (-a * c * (x - 1) + b * ev * y) / n2;
    U[3] = (b * c * (x - 1) - a * ev * y) / n2;
    U[4] = ((a * a + c * c) * x + b * b) / n2;
    U[5] = (a * b * (x - 1) + c * ev * y) / n2;
    U[6] = (-a * c * (x - 1) - b * ev * y) / n2;
    U[7] = (a * b * (x - 1) - c * ev * y) / n2;
    U[8] = ((b * b + c * c) * x + a * a) / n2;
}

void orc_dirac3d_magnus_k(const orc_pulse *p, const orc_time_config *tc, double k_z,
                          double kappa, double *rhos) {
    const double mk = sqrt(k_z * k_z + kappa * kappa);
    double S[3] = {0.0, 0.0, -1.0};
    const double me = (tc->t_end - tc->t_begin) / tc->n_measurements;
    double t_begin = tc->t_begin, t_end = t_begin + me;
    rhos[0] = S[2];
    for (int i = 1; i <= tc->n_measurements; ++i) {
        double cf[4], U[9];
        orc_magnus_coefficients(p, me, t_begin, cf);
        for (int q = 0; q < 4; ++q) cf[q] /= mk;
        orc_dirac_magnus_U(2 * mk, 2 * kappa, 2 * k_z, me, cf, U);
        const double s0 = U[0] * S[0] + U[1] * S[1] + U[2] * S[2];
        const double s1 = U[3] * S[0] + U[4] * S[1] + U[5] * S[2];
        const double s2 = U[6] * S[0] + U[7] * S[1] + U[8] * S[2];
        S[0] = s0, S[1] = s1, S[2] = s2;
        rhos[i] = S[2];
        t_begin = t_end;
        t_end += me;
    }
}

int orc_dirac3d_sigma_k(const orc_pulse *p, const orc_time_config *tc, const orc_solver *s,
                        double k_z, double kappa, double *rhos, orc_stats *st) {
    const orc_model m = {ORC_DIRAC3D, 0, 0, 0, 1, 0};
    const double krow[8] = {k_z, kappa, sqrt(k_z * k_z + kappa * kappa), 1.0, 0.0, 0.0, -1.0, 0.0};
    double *states = malloc(sizeof(double) * 3 * (tc->n_measurements + 1));
    const int rc = orc_evolve_k(&m, p, tc, s, krow, states, st);
    for (int i = 0; i <= tc->n_measurements; ++i) rhos[i] = states[3 * i + 2];
    free(states);
    return rc;
}
