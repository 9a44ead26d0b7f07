// hhg_gpu.cu -- host side of the C ABI declared in include/hhg_gpu.h:
// contexts, Gauss-Legendre rules, k grids with their initial Bloch vectors,
// plans (device-resident k table, per-interval pulse staging, work list,
// partial buffer), launches, status checking and the trapezoidal FFT.
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hhg_gpu.h"
#include "hhg_launch.cuh"
#include "hhg_pulse_prep.hpp"

using hhg::PulseDev;

struct hhg_ctx {
    int device = 0;
    // plans of the one-shot entry point, most recently used first (key: the
    // serialised descriptors)
    std::vector<std::pair<std::string, hhg_plan *>> plan_cache;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string last_error;
    std::map<int, cufftHandle> fft_plans;
    // spectrum scratch
    double *d_x = nullptr, *d_out = nullptr;
    double2 *d_F = nullptr;
    size_t x_cap = 0, f_cap = 0;
    // the Dirac quadrature's state, kept between calls: the plan (pulse
    // staging, launch state) of the last (system, pulse, options), the rows
    // its k table and sample buffer hold, and grow-only device buffers
    hhg_plan *kappa_plan = nullptr;
    // the device k table of the last plan built from a generated grid (key:
    // the system and grid descriptors), shared with the plans that use it: a
    // new batch of pulses on the same grid skips building and uploading rows
    std::shared_ptr<double> ktab_shared;
    std::string ktab_key;
    std::string kappa_key;
    long long kappa_cap = 0;
    int kappa_occ = 1;
    struct Grow {
        void *p = nullptr;
        size_t bytes = 0;
    } kappa_T, kappa_items, kappa_change, kappa_j, kappa_slice;
};

struct hhg_plan {
    hhg_ctx *ctx = nullptr;
    std::shared_ptr<double> ktab_owner;  // set when d_ktab is the context's shared table
    int model = 0, degree = 7;
    hhg_solver_opts opts{};
    int n_pulses = 0;
    int64_t n_k = 0;
    int tiles_per_item = 1, items_per_pulse = 0;
    long long n_items = 0;
    long long j_len = 0, part_len = 0, coef_len = 0, n_intervals = 0;
    std::vector<PulseDev> pulses;
    std::vector<double> window_end;
    int grid = 0;
    // device buffers
    double *d_ktab = nullptr, *d_coef = nullptr, *d_part = nullptr, *d_j = nullptr,
           *d_tgrid = nullptr;
    PulseDev *d_pulses = nullptr;
    long long *d_ioff = nullptr;
    unsigned long long *d_counters = nullptr;
    int *d_status = nullptr;
    bool timed = false;
    // spectra (allocated on first hhg_plan_spectrum_async)
    double *d_spec = nullptr, *d_x = nullptr;
    double2 *d_F = nullptr;
    std::vector<long long> spec_off;  // per pulse offset (in n_fft units) into d_spec
    long long spec_len = 0;
    // learned proposer: packed network
    hhg::MlpPacked *d_mlp = nullptr;
    // step-history recording (hhg_learned_collect)
    bool record = false;
    int hist_every = 1;
    long long hist_cap = 0;
    float *d_hist = nullptr;
    unsigned long long *d_hist_count = nullptr;
    long long part_cap = 0;  // doubles allocated for d_part
    int occupancy = 1;       // resident CTAs per SM of the selected kernel variant
    // CUDA graph of one execution (integration + reduction [+ spectra])
    cudaGraphExec_t gexec = nullptr;
    int graph_spec = -1;
    // output mode (bz_integrate_kernel's OUT): 1 split current (two partial
    // channels, j of 2 j_len), 2/3 k-resolved samples into d_kout
    int out_mode = 0;
    double energy_cut = 0.0;
    double *d_kout = nullptr;
    long long kout_len = 0;
};

namespace hhg {
void pack_mlp(const hhg_mlp &net, MlpPacked *out);
hhg_status mlp_train_impl(cudaStream_t s, const float *records, int64_t n, const hhg_train_opts &o,
                          hhg_mlp *net, float *epoch_loss, double *train_ms, std::string *msg);
hhg_status mlp_gradients_impl(cudaStream_t s, const float *records, int64_t n, const hhg_mlp *net,
                              float *grad_out, float *loss_out, std::string *msg);
hhg_status mlp_predict_impl(cudaStream_t s, const float *records, int64_t n, const hhg_mlp *net,
                            int path, float *out, std::string *msg);
}  // namespace hhg

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kSqrt3 = 1.732050807568877293527446341;

hhg_status set_err(hhg_ctx *ctx, hhg_status st, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

#define HHG_CUDA(ctx, call)                                                              \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess)                                                          \
            return set_err(ctx, HHG_CUDA_ERROR,                                          \
                           std::string(#call) + ": " + cudaGetErrorString(e__));         \
    } while (0)

// Gauss-Legendre nodes by Newton iteration on P_n in long double.
void gauss_legendre_compute(int n, double *x, double *w) {
    const long double pi = 3.141592653589793238462643383279502884L;
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        long double z = cosl(pi * (i + 0.75L) / (n + 0.5L));
        long double dp = 0.0L;
        for (int it = 0; it < 100; ++it) {
            long double p1 = 1.0L, p2 = 0.0L;
            for (int j = 1; j <= n; ++j) {
                const long double p3 = p2;
                p2 = p1;
                p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / j;
            }
            dp = n * (z * p1 - p2) / (z * z - 1.0L);
            const long double dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-19L * (1.0L + fabsl(z))) {
                p1 = 1.0L;
                p2 = 0.0L;
                for (int j = 1; j <= n; ++j) {
                    const long double p3 = p2;
                    p2 = p1;
                    p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / j;
                }
                dp = n * (z * p1 - p2) / (z * z - 1.0L);
                break;
            }
        }
        const long double wi = 2.0L / ((1.0L - z * z) * dp * dp);
        x[n - 1 - i] = (double)z;
        x[i] = (double)(-z);
        w[n - 1 - i] = (double)wi;
        w[i] = (double)wi;
    }
    if (n & 1) x[n / 2] = 0.0;
}

// The same, remembered per n for the life of the process (a 1024-point rule
// costs ~10 ms of long-double Newton steps, and every plan on a grid needs it).
void gauss_legendre(int n, double *x, double *w) {
    static std::mutex mu;
    static std::map<int, std::vector<double>> rules;  // n nodes, then n weights
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = rules.find(n);
        if (it != rules.end()) {
            std::memcpy(x, it->second.data(), sizeof(double) * n);
            std::memcpy(w, it->second.data() + n, sizeof(double) * n);
            return;
        }
    }
    std::vector<double> r(2 * (size_t)n);
    gauss_legendre_compute(n, r.data(), r.data() + n);
    std::memcpy(x, r.data(), sizeof(double) * n);
    std::memcpy(w, r.data() + n, sizeof(double) * n);
    std::lock_guard<std::mutex> lock(mu);
    rules.emplace(n, std::move(r));
}

// Positive half, ascending: gauss::container<n> (thread_gauss.hpp).
void gauss_half(int n, std::vector<double> &xa, std::vector<double> &wa) {
    std::vector<double> x(n), w(n);
    gauss_legendre(n, x.data(), w.data());
    xa.assign(x.begin() + n / 2, x.end());
    wa.assign(w.begin() + n / 2, w.end());
}

bool ref_is_zero(double v) {
    uint64_t bits;
    std::memcpy(&bits, &v, sizeof bits);
    return (int)((bits >> 52) & 0x7FF) < 0x3D3;
}

// fermi_function (GlobalDefinitions.hpp:36-41); beta == 0 stands for the
// reference's T = 0 sentinel (a step with 1/2 at zero energy).
double fermi_occ(double e, double beta) {
    if (beta == 0.0) return e != 0 ? (e < 0 ? 1.0 : 0.0) : 0.5;
    return 1. / (1. + exp(beta * e));
}

// PiFlux::ic_sigma (PiFlux.cpp:519-549) with alpha^2 = occupation_a, beta^2 =
// occupation_b (PiFlux.cpp:420-426) at the momentum cosines (cx, cy, cz).
void piflux_ic(const hhg_system_desc &s, double cx, double cy, double cz, double *s0) {
    const double disp = sqrt(cx * cx + cy * cy + cz * cz);
    const double a2 = fermi_occ(-s.fermi_energy + 2 * s.hopping * disp, s.beta);
    const double b2 = fermi_occ(-s.fermi_energy - 2 * s.hopping * disp, s.beta);
    const double diff = a2 - b2;
    const double prod = 2 * sqrt(a2 * b2);
    const double zeps = cz + disp;
    s0[0] = (diff * cx * zeps + prod * (cy * cy + cz * zeps)) / (disp * zeps);
    s0[1] = (diff * cy * zeps - prod * cx * cy) / (disp * zeps);
    s0[2] = (diff * cz * zeps - prod * cx * zeps) / (disp * zeps);
}

// Initial Bloch vector: the reference models' ic_sigma / Fermi-occupied state
// (T = 0, E_F = 0: the filled lower band), the variants' filled lower band
// S0 = -d_hat(k).
void initial_state(const hhg_system_desc &s, double kx, double ky, double kz, double *s0) {
    switch (s.kind) {
    case HHG_SYS_PIFLUX3D:
        piflux_ic(s, cos(kx), cos(ky), cos(kz), s0);
        break;
    case HHG_SYS_PIFLUX2D: {
        const double cx = cos(kx), cy = cos(ky);
        const double n = sqrt(cx * cx + cy * cy);
        s0[0] = cx / n;
        s0[1] = cy / n;
        s0[2] = 0.0;
        break;
    }
    case HHG_SYS_DIRAC2D: {
        const double d0 = s.velocity * kx, d1 = s.velocity * ky, d2 = s.mass;
        const double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        s0[0] = -d0 / n;
        s0[1] = -d1 / n;
        s0[2] = -d2 / n;
        break;
    }
    case HHG_SYS_HONEYCOMB: {
        // Honeycomb::ic_sigma at T = 0 (Honeycomb.cpp:355-361)
        double gre = 0.0, gim = 0.0;
        const double nn[3][2] = {{1.0, 0.0}, {-0.5, 0.5 * kSqrt3}, {-0.5, -0.5 * kSqrt3}};
        for (int j = 0; j < 3; ++j) {
            const double ph = nn[j][0] * kx + nn[j][1] * ky;
            gre += cos(ph);
            gim += sin(ph);
        }
        if (s.mass == 0.0) {
            // Honeycomb::ic_sigma with occupation_a/b (Honeycomb.cpp:347-361)
            const double ag = hypot(gre, gim);
            const double a2 = fermi_occ(s.fermi_energy - s.hopping * ag, s.beta);
            const double b2 = fermi_occ(s.fermi_energy + s.hopping * ag, s.beta);
            const double diff = a2 - b2;
            s0[0] = -diff * gre / ag;
            s0[1] = diff * gim / ag;
            s0[2] = -(2 * sqrt(a2 * b2));
        } else {
            const double d0 = s.hopping * gre, d1 = -s.hopping * gim, d2 = s.mass;
            const double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            s0[0] = -d0 / n;
            s0[1] = -d1 / n;
            s0[2] = -d2 / n;
        }
        break;
    }
    case HHG_SYS_DIRAC3D: {
        // (2 a0 b0, 0, a0^2 - b0^2), a0 = f(E_F + |k|), b0 = f(E_F - |k|)
        // (DiracSystem.cpp:155-158, 253-255); kx = k_z, ky = kappa
        const double disp = sqrt(ky * ky + kx * kx);
        const double a0 = fermi_occ(s.fermi_energy + disp, s.beta);
        const double b0 = fermi_occ(s.fermi_energy - disp, s.beta);
        s0[0] = 2. * a0 * b0;
        s0[1] = 0.0;
        s0[2] = a0 * a0 - b0 * b0;
        break;
    }
    default:
        s0[0] = s0[1] = s0[2] = 0.0;
    }
}

void push_row(const hhg_system_desc &s, double kx, double ky, double kz, double w, double *o) {
    o[0] = kx;
    o[1] = ky;
    o[2] = kz;
    o[3] = w;
    initial_state(s, kx, ky, kz, o + 4);
    o[7] = 0.0;
}

// n_debug_points (GlobalDefinitions.hpp): the momenta of the debug traces
constexpr int kDebugPoints = 25;

int64_t grid_count(const hhg_grid_desc &g) {
    switch (g.kind) {
    case HHG_GRID_TENSOR_GL:
    case HHG_GRID_RHOMBIC_GL:
        return (int64_t)g.n1 * g.n2;
    case HHG_GRID_PIFLUX3D_REF: {
        const int64_t c = g.n2, f = 8 * c;
        return 2 * (int64_t)g.n1 * ((2 * f) * f + (6 * c) * (2 * c) + 2 * (2 * c) * (2 * c));
    }
    case HHG_GRID_HONEYCOMB_HEX_REF:
        return 4 * (int64_t)g.n1 * g.n1;
    case HHG_GRID_EXPLICIT:
        return g.n_rows;
    case HHG_GRID_PIFLUX3D_OCCUPATION:
        return (int64_t)g.n1 * g.n1;
    case HHG_GRID_PIFLUX3D_CUBE:
        return 2 * (int64_t)g.n1 * g.n1 * g.n1;
    case HHG_GRID_PIFLUX3D_DEBUG:
    case HHG_GRID_DIRAC3D_DEBUG:
        return kDebugPoints;
    }
    return -1;
}

// A PiFlux row of a momentum_type built from (x, y, z) with the reference's
// construction-time rescue (PiFlux.cpp:934-938, 983-988): when cos x and cos y
// vanish (is_zero) and cos z < 0, cos x becomes |cos z| 1e-4 and cos z is
// scaled by 1 - 0.5e-8.  Unlike the continuum-limit grid the rescued cos x
// stays in the momentum that is evolved, so the row carries it as kx =
// acos(|cos z| 1e-4); the initial state uses the rescued cosines.
void piflux_rescued_row(const hhg_system_desc &s, double x, double y, double z, double w, double *o) {
    double cx = cos(x), cy = cos(y), cz = cos(z);
    double kx = x;
    if (ref_is_zero(cx) && ref_is_zero(cy) && cz < 0.0) {
        cx = std::fabs(cz) * 1e-4;
        cz *= (1. - 0.5 * 1e-4 * 1e-4);
        kx = std::acos(cx);
    }
    o[0] = kx;
    o[1] = y;
    o[2] = z;
    o[3] = w;
    piflux_ic(s, cx, cy, cz, o + 4);
    o[7] = 0.0;
}

// body(i) for i in [0, n) on up to 32 host threads (each i writes its own
// outputs, so the result is the same whatever the schedule); serial below
// min_n items.
template <class F> void parallel_for(int n, F body, int min_n = 64) {
    const unsigned hc = std::thread::hardware_concurrency();
    const int nt = (int)std::min<unsigned>(std::max(hc, 1u), 32u);
    if (nt <= 1 || n < min_n) {
        for (int i = 0; i < n; ++i) body(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (int i; (i = next.fetch_add(1)) < n;) body(i);
        });
    for (auto &th : pool) th.join();
}

// Row builders; see the oracle for the same restatements.
void build_rows(const hhg_system_desc &s, const hhg_grid_desc &g, double *out) {
    size_t r = 0;
    switch (g.kind) {
    case HHG_GRID_TENSOR_GL: {
        std::vector<double> gx(g.n1), wx(g.n1), gy(g.n2), wy(g.n2);
        gauss_legendre(g.n1, gx.data(), wx.data());
        gauss_legendre(g.n2, gy.data(), wy.data());
        const double hx = 0.5 * (g.x_hi - g.x_lo), mx = 0.5 * (g.x_hi + g.x_lo);
        const double hy = 0.5 * (g.y_hi - g.y_lo), my = 0.5 * (g.y_hi + g.y_lo);
        parallel_for(g.n1, [&](int i) {
            for (int j = 0; j < g.n2; ++j)
                push_row(s, hx * gx[i] + mx, hy * gy[j] + my, 0.0, hx * hy * wx[i] * wy[j],
                         out + 8 * ((size_t)i * g.n2 + j));
        });
        break;
    }
    case HHG_GRID_RHOMBIC_GL: {
        // k = f1 b1 + f2 b2, f in [-1/2, 1/2]^2, b1 = 2pi/3 (1, -sqrt3), b2 = 2pi/3 (1, sqrt3)
        const double b1x = 2.0 * kPi / 3.0, b1y = -2.0 * kPi / 3.0 * kSqrt3;
        const double b2x = 2.0 * kPi / 3.0, b2y = 2.0 * kPi / 3.0 * kSqrt3;
        const double area = fabs(b1x * b2y - b1y * b2x);
        std::vector<double> g1(g.n1), w1(g.n1), g2(g.n2), w2(g.n2);
        gauss_legendre(g.n1, g1.data(), w1.data());
        gauss_legendre(g.n2, g2.data(), w2.data());
        parallel_for(g.n1, [&](int i) {
            for (int j = 0; j < g.n2; ++j) {
                const double f1 = 0.5 * g1[i], f2 = 0.5 * g2[j];
                push_row(s, f1 * b1x + f2 * b2x, f1 * b1y + f2 * b2y, 0.0,
                         0.25 * area * w1[i] * w2[j], out + 8 * ((size_t)i * g.n2 + j));
            }
        });
        break;
    }
    case HHG_GRID_PIFLUX3D_REF: {
        // PiFlux::current_density_continuum_limit / improved_xy_integral
        // (PiFlux.cpp:665-863), including the initial-state rescue of +k_z
        // slices with cos k_z < 0 (PiFlux.cpp:812-816).
        const int zr = g.n1, nc = g.n2, nf = 8 * nc;
        const double pi = kPi, edge = 0.35 * pi;
        struct Seg { double lo, hi; int nh; };
        const Seg rx[4] = {{edge, pi - edge, nf}, {0.0, pi, 3 * nc}, {0.0, edge, nc}, {pi - edge, pi, nc}};
        const Seg ry[4] = {{edge, 0.5 * pi, nf / 2}, {0.0, edge, nc}, {edge, 0.5 * pi, nc}, {edge, 0.5 * pi, nc}};
        std::vector<double> za, zw;
        gauss_half(2 * zr, za, zw);
        std::vector<double> xa[4], xw[4], ya[4], yw[4];
        for (int q = 0; q < 4; ++q) {
            gauss_half(2 * rx[q].nh, xa[q], xw[q]);
            gauss_half(2 * ry[q].nh, ya[q], yw[q]);
        }
        double last_cx = 0.0, last_cy = 0.0;
        for (int z = 0; z < zr; ++z)
            for (int sg = 0; sg < 2; ++sg) {
                const double kz = (sg == 0 ? pi : -pi) * za[z];
                double cz = cos(kz);
                const double chx = sg == 0 ? 0.0 : last_cx, chy = sg == 0 ? 0.0 : last_cy;
                if (ref_is_zero(chx) && ref_is_zero(chy) && cz < 0.0) cz *= (1. - 0.5 * 1e-4 * 1e-4);
                for (int q = 0; q < 4; ++q) {
                    const double xh = 0.5 * (rx[q].hi - rx[q].lo), xm = 0.5 * (rx[q].hi + rx[q].lo);
                    const double yh = 0.5 * (ry[q].hi - ry[q].lo), ym = 0.5 * (ry[q].hi + ry[q].lo);
                    const double tw = xh * yh;
                    for (int i = 0; i < rx[q].nh; ++i)
                        for (int sx = 0; sx < 2; ++sx) {
                            const double kx = xh * (sx ? -xa[q][i] : xa[q][i]) + xm;
                            const double mw = xw[q][i] * tw;
                            for (int j = 0; j < ry[q].nh; ++j)
                                for (int sy = 0; sy < 2; ++sy) {
                                    const double ky = yh * (sy ? -ya[q][j] : ya[q][j]) + ym;
                                    double *o = out + 8 * r++;
                                    o[0] = kx;
                                    o[1] = ky;
                                    o[2] = kz;
                                    o[3] = mw * yw[q][j] * zw[z];
                                    const double cx = cos(kx), cy = cos(ky);
                                    piflux_ic(s, cx, cy, cz, o + 4);
                                    o[7] = 0.0;
                                    last_cx = cx;
                                    last_cy = cy;
                                }
                        }
                }
            }
        break;
    }
    case HHG_GRID_HONEYCOMB_HEX_REF: {
        // Honeycomb::compute_current_density (Honeycomb.cpp:225-323)
        const int nk = g.n1;
        const double min_x = -2 * kPi / 3, max_x = 2 * kPi / 3;
        std::vector<double> a, w;
        gauss_half(2 * nk, a, w);
        for (int x = 0; x < nk; ++x) {
            const double kx0 = 0.5 * (max_x - min_x) * a[x] + 0.5 * (max_x + min_x);
            const double ymax = (4 * kPi / (3 * kSqrt3)) - (fabs(kx0) / kSqrt3);
            for (int sx = 0; sx < 2; ++sx) {
                const double kx = sx ? (0.5 * (max_x - min_x) * (-a[x]) + 0.5 * (max_x + min_x)) : kx0;
                for (int y = 0; y < nk; ++y) {
                    const double tw = 0.5 * (max_x - min_x) * (0.5 * (ymax - (-ymax))) * w[x] * w[y];
                    for (int sy = 0; sy < 2; ++sy) {
                        const double ay = sy ? -a[y] : a[y];
                        const double ky = 0.5 * (ymax - (-ymax)) * ay + 0.5 * (ymax + (-ymax));
                        push_row(s, kx, ky, 0.0, tw, out + 8 * r++);
                    }
                }
            }
        }
        break;
    }
    case HHG_GRID_EXPLICIT:
        std::memcpy(out, g.rows, sizeof(double) * 8 * (size_t)g.n_rows);
        break;
    case HHG_GRID_PIFLUX3D_OCCUPATION: {
        // PiFlux::compute_occupation_numbers (PiFlux.cpp:909-953): i = x N + z,
        // k = (x dx, pi/2, dz z)
        const int N = g.n1;
        const double dx = kPi / N, dz = kPi / N;
        for (int i = 0; i < N * N; ++i) {
            const int x = i / N, z = i % N;
            piflux_rescued_row(s, x * dx, 0.5 * kPi, dz * z, 1.0, out + 8 * r++);
        }
        break;
    }
    case HHG_GRID_PIFLUX3D_CUBE: {
        // PiFlux::current_per_energy (PiFlux.cpp:955-1035): i = z N^2 + y N + x,
        // k = (x, y, z) dxy and its -z mirror (k.invert()), both weighted 1/N^3
        const int N = g.n1;
        const double d = kPi / N;
        const double w = 1.0 / ((double)N * N * N);
        for (int64_t i = 0; i < (int64_t)N * N * N; ++i) {
            const int z = (int)(i / ((int64_t)N * N)), y = (int)((i / N) % N), x = (int)(i % N);
            piflux_rescued_row(s, x * d, y * d, d * z, w, out + 8 * r);
            double *m = out + 8 * (r + 1);
            std::memcpy(m, out + 8 * r, 8 * sizeof(double));
            m[2] = -m[2];
            r += 2;
        }
        break;
    }
    case HHG_GRID_PIFLUX3D_DEBUG:
        // PiFlux::compute_current_density_debug (PiFlux.cpp:320-371): momentum_type
        // (picked_x, picked[i], picked_z) as constructed, no rescue
        for (int i = 0; i < kDebugPoints; ++i)
            push_row(s, 0.5 * kPi, 0.5 * kPi - (i * 0.02 * kPi), 0.49 * kPi, 1.0, out + 8 * r++);
        break;
    case HHG_GRID_DIRAC3D_DEBUG: {
        // DiracSystem::compute_current_density_debug (DiracSystem.cpp:333-363):
        // picked_z = n_z/2 + n_z/10, delta_z = 2 max_k / n_z, kappa_max from
        // kappa_integration_upper_limit (DiracSystem.cpp:257-261), rows
        // (k_z, kappa, |k|) weighted by integration_weight k_z kappa / |k|
        const int n_z = g.n1;
        const double max_k = g.x_hi;
        const double delta_z = 2 * max_k / n_z;
        const double k_z = (n_z / 2 + n_z / 10 - n_z / 2) * delta_z;
        const double kappa_max = std::sqrt(max_k * max_k - k_z * k_z);
        for (int i = 0; i < kDebugPoints; ++i) {
            const double kappa = (i + 1) * kappa_max / (kDebugPoints + 1);
            const double mk = std::sqrt(k_z * k_z + kappa * kappa);
            push_row(s, k_z, kappa, mk, k_z * kappa / mk, out + 8 * r++);
        }
        break;
    }
    }
}

hhg_status check_system(hhg_ctx *ctx, const hhg_system_desc *s) {
    if (!s) return set_err(ctx, HHG_BAD_CONFIG, "null system descriptor");
    if (s->kind < HHG_SYS_DIRAC2D || s->kind > HHG_SYS_DIRAC3D)
        return set_err(ctx, HHG_BAD_CONFIG, "System type not recognized");
    if (!std::isfinite(s->hopping) || !std::isfinite(s->velocity) || !std::isfinite(s->mass) ||
        !std::isfinite(s->pol_x) || !std::isfinite(s->pol_y) || !std::isfinite(s->beta) ||
        !std::isfinite(s->fermi_energy) || !std::isfinite(s->inv_diag_relax) ||
        !std::isfinite(s->inv_offdiag_relax))
        return set_err(ctx, HHG_BAD_CONFIG, "non-finite system parameter");
    if (s->beta < 0.0 || s->inv_diag_relax < 0.0 || s->inv_offdiag_relax < 0.0)
        return set_err(ctx, HHG_BAD_CONFIG, "beta and the relaxation rates must be >= 0");
    const bool thermal = s->beta != 0.0 || s->fermi_energy != 0.0 || s->inv_diag_relax > 0.0;
    const bool reference_model = s->kind == HHG_SYS_PIFLUX3D || s->kind == HHG_SYS_DIRAC3D ||
                                 (s->kind == HHG_SYS_HONEYCOMB && s->mass == 0.0);
    if (thermal && !reference_model)
        return set_err(ctx, HHG_UNSUPPORTED,
                       "temperature, Fermi energy and relaxation are defined for the reference "
                       "models (PiFlux-3D, Honeycomb without mass, Dirac-3D) only");
    return HHG_OK;
}

hhg_status check_grid(hhg_ctx *ctx, const hhg_grid_desc *g) {
    if (!g) return set_err(ctx, HHG_BAD_CONFIG, "null grid descriptor");
    switch (g->kind) {
    case HHG_GRID_TENSOR_GL:
    case HHG_GRID_RHOMBIC_GL:
        if (g->n1 < 1 || g->n2 < 1 || g->n1 > 65536 || g->n2 > 65536)
            return set_err(ctx, HHG_BAD_CONFIG, "grid order out of range");
        break;
    case HHG_GRID_PIFLUX3D_REF:
        if (g->n1 < 1 || g->n2 < 1 || g->n1 > 4096 || g->n2 > 256)
            return set_err(ctx, HHG_BAD_CONFIG, "PiFlux reference grid size out of range");
        break;
    case HHG_GRID_HONEYCOMB_HEX_REF:
        if (g->n1 < 1 || g->n1 > 8192) return set_err(ctx, HHG_BAD_CONFIG, "N_k out of range");
        break;
    case HHG_GRID_EXPLICIT:
        if (!g->rows || g->n_rows < 1) return set_err(ctx, HHG_BAD_CONFIG, "explicit grid without rows");
        break;
    case HHG_GRID_PIFLUX3D_OCCUPATION:
        if (g->n1 < 1 || g->n1 > 16384) return set_err(ctx, HHG_BAD_CONFIG, "occupation grid N out of range");
        break;
    case HHG_GRID_PIFLUX3D_CUBE:
        if (g->n1 < 1 || g->n1 > 1024) return set_err(ctx, HHG_BAD_CONFIG, "cube grid N out of range");
        break;
    case HHG_GRID_PIFLUX3D_DEBUG:
        break;
    case HHG_GRID_DIRAC3D_DEBUG:
        if (g->n1 < 1 || g->n1 > (1 << 24) || !(g->x_hi > 0.0) || !std::isfinite(g->x_hi))
            return set_err(ctx, HHG_BAD_CONFIG, "Dirac debug grid needs n_z >= 1 and max_k > 0");
        break;
    default:
        return set_err(ctx, HHG_BAD_CONFIG, "grid type not recognized");
    }
    const int64_t n = grid_count(*g);
    if (n < 1 || n > (int64_t)1 << 31) return set_err(ctx, HHG_BAD_CONFIG, "k grid too large");
    return HHG_OK;
}

hhg_status check_pulse(hhg_ctx *ctx, const hhg_pulse_desc &p) {
    if (p.kind < HHG_PULSE_COSINE || p.kind > HHG_PULSE_SPLINE)
        return set_err(ctx, HHG_BAD_CONFIG, "Laser type not recognized");
    if (p.n_measurements < 1 || p.n_measurements > (1 << 24))
        return set_err(ctx, HHG_BAD_CONFIG, "n_measurements out of range");
    if (p.n_subdivisions < 1) return set_err(ctx, HHG_BAD_CONFIG, "n_subdivisions must be >= 1");
    if ((p.kind == HHG_PULSE_COSINE || p.kind == HHG_PULSE_GAUSS) &&
        (!(p.n_cycles > 0.0) || !std::isfinite(p.n_cycles)))
        return set_err(ctx, HHG_BAD_CONFIG, "n_cycles must be > 0");
    if (p.kind == HHG_PULSE_SPLINE) {
        if (!p.samples || p.n_samples < 5 || p.n_samples > (1 << 24))
            return set_err(ctx, HHG_BAD_CONFIG, "a spline pulse needs 5 <= n_samples <= 2^24 samples");
        if (!(p.sample_dt > 0.0) || !std::isfinite(p.sample_dt) || !std::isfinite(p.spline_cut) ||
            std::isinf(p.deriv_begin) || std::isinf(p.deriv_end))
            return set_err(ctx, HHG_BAD_CONFIG, "spline pulse: sample_dt > 0, finite cut and derivatives");
        for (int64_t k = 0; k < p.n_samples; ++k)
            if (!std::isfinite(p.samples[k])) return set_err(ctx, HHG_BAD_CONFIG, "non-finite pulse sample");
    }
    if (!std::isfinite(p.amplitude) || !std::isfinite(p.t_begin) || !std::isfinite(p.phase) ||
        !std::isfinite(p.window_begin) || !std::isfinite(p.window_end) ||
        !std::isfinite(p.energy_scale))
        return set_err(ctx, HHG_BAD_CONFIG, "non-finite pulse parameter");
    if (!(p.window_end > p.window_begin)) return set_err(ctx, HHG_BAD_CONFIG, "empty time window");
    if (!(p.energy_scale > 0.0)) return set_err(ctx, HHG_BAD_CONFIG, "energy_scale must be > 0");
    return HHG_OK;
}

// Internal kernel model (hhg::Model): the ABI kind, or a variant with fewer
// distinct pulse projections when the polarisation allows it.
int kernel_model(const hhg_system_desc &s) {
    if (s.inv_diag_relax > 0.0) {
        // relaxation right-hand sides (PiFlux.cpp:509-516, Honeycomb.cpp:214-223)
        if (s.kind == HHG_SYS_PIFLUX3D) return hhg::PIFLUX3D_RELAX;
        if (s.kind == HHG_SYS_HONEYCOMB) return hhg::HONEYCOMB_RELAX;
        if (s.kind == HHG_SYS_DIRAC3D) return hhg::DIRAC3D_RELAX;
    }
    if (s.kind == HHG_SYS_PIFLUX2D && s.pol_x == s.pol_y) return hhg::PIFLUX2D_SYM;
    if (s.kind == HHG_SYS_HONEYCOMB && s.pol_y == 0.0) return hhg::HONEYCOMB_X;
    return s.kind;
}

constexpr size_t kPlanCacheSize = 4;

// Byte key of the k table a generated grid gives for a system.
std::string ktab_key(const hhg_system_desc *sys, const hhg_grid_desc *grid) {
    std::string k;
    auto put = [&k](const void *p, size_t n) { k.append(static_cast<const char *>(p), n); };
    put(sys, sizeof *sys);
    put(&grid->kind, 4 * 3);
    put(&grid->x_lo, 8 * 4);
    return k;
}

// Byte key of the descriptors of one one-shot call: every field that changes
// the computation (explicit k rows and the learned network by value).
std::string plan_key(const hhg_system_desc *sys, const hhg_pulse_desc *pulses, int n_pulses,
                     const hhg_grid_desc *grid, const hhg_solver_opts *opts) {
    std::string k;
    auto put = [&k](const void *p, size_t n) { k.append(static_cast<const char *>(p), n); };
    put(&sys->kind, 4);
    put(&sys->hopping, 8 * 9);
    put(&n_pulses, 4);
    for (int i = 0; i < n_pulses; ++i) {
        const hhg_pulse_desc &q = pulses[i];
        put(&q.kind, 4 * 3);
        put(&q.amplitude, 8 * 7);
        if (q.kind == HHG_PULSE_SPLINE && q.samples && q.n_samples > 0) {
            put(&q.n_samples, 8 * 5);
            put(q.samples, sizeof(double) * (size_t)q.n_samples);
        }
    }
    put(&grid->kind, 4 * 3);
    put(&grid->x_lo, 8 * 4);
    put(&grid->n_rows, 8);
    if (grid->kind == HHG_GRID_EXPLICIT && grid->rows && grid->n_rows > 0)
        put(grid->rows, sizeof(double) * 8 * (size_t)grid->n_rows);
    if (opts) {
        put(&opts->stepper, 4 * 4);
        put(&opts->abs_tol, 8 * 2);
        put(&opts->max_failed_steps, 4 * 4);
        put(&opts->mlp_every, 4);
        put(&opts->coarsen_div, 4);
        const bool learned = opts->proposer == HHG_PROPOSER_LEARNED && opts->mlp;
        put(&learned, 1);
        if (learned) put(opts->mlp, sizeof(hhg_mlp));
    } else {
        put("default", 7);
    }
    return k;
}

// Kernel step-control mode for an ABI proposer: 0 restart, 1 carry, 2 dyadic,
// 3 learned dyadic.
int kernel_proposer(int abi) {
    switch (abi) {
    case HHG_PROPOSER_CARRY: return 1;
    case HHG_PROPOSER_LOCKSTEP: return 2;
    case HHG_PROPOSER_LEARNED: return 3;
    default: return 0;
    }
}

int model_nf(int m) {
    switch (hhg::base_model(m)) {
    case hhg::DIRAC2D: return 1;
    case hhg::DIRAC3D: return 1;
    case hhg::PIFLUX3D: return 2;
    case hhg::PIFLUX2D: return 4;
    case hhg::HONEYCOMB: return 6;
    case hhg::PIFLUX2D_SYM: return 2;
    case hhg::HONEYCOMB_X: return 4;
    }
    return 0;
}

// Chebyshev-tail test of the staged interpolants, in long double so the
// fit's own rounding (~1e-19) sits below the threshold: the smallest degree in
// {5, 7, 11} whose Chebyshev tail beyond it is below 2^-56 of the function scale
// on sampled intervals, or -1 if even degree 11 is not enough.
// ---------------------------------------------------------------------------
// Pulses on the host: the spline coefficients, A(t) for the sample-0 record
// and the window checks, the continued A(t) in long double for the degree test.
// ---------------------------------------------------------------------------
// Clamped cubic spline through y[0..n) at spacing h as cardinal cubic
// B-spline coefficients c_(-1..n) (n + 2 values): interpolation (c_(k-1) +
// 4 c_k + c_(k+1)) / 6 = y_k, end slopes (c_1 - c_(-1)) / 2h = d0 and (c_n -
// c_(n-2)) / 2h = dn, eliminated into a tridiagonal system solved in long
// double.  A NaN slope takes the one-sided five-point difference.
std::vector<double> spline_coefficients(const double *y, int64_t n, double h, double d0, double dn) {
    if (std::isnan(d0)) d0 = (-25.0 * y[0] + 48.0 * y[1] - 36.0 * y[2] + 16.0 * y[3] - 3.0 * y[4]) / (12.0 * h);
    if (std::isnan(dn))
        dn = (25.0 * y[n - 1] - 48.0 * y[n - 2] + 36.0 * y[n - 3] - 16.0 * y[n - 4] + 3.0 * y[n - 5]) / (12.0 * h);
    std::vector<long double> sub(n), diag(n), sup(n), rhs(n), c(n);
    for (int64_t k = 0; k < n; ++k) {
        sub[k] = 1.0L;
        diag[k] = 4.0L;
        sup[k] = 1.0L;
        rhs[k] = 6.0L * y[k];
    }
    sup[0] = 2.0L;
    rhs[0] += 2.0L * h * d0;
    sub[n - 1] = 2.0L;
    rhs[n - 1] -= 2.0L * h * dn;
    for (int64_t k = 1; k < n; ++k) {  // Thomas elimination (diagonally dominant)
        const long double m = sub[k] / diag[k - 1];
        diag[k] -= m * sup[k - 1];
        rhs[k] -= m * rhs[k - 1];
    }
    c[n - 1] = rhs[n - 1] / diag[n - 1];
    for (int64_t k = n - 2; k >= 0; --k) c[k] = (rhs[k] - sup[k] * c[k + 1]) / diag[k];
    std::vector<double> out(n + 2);
    out[0] = (double)(c[1] - 2.0L * h * d0);
    for (int64_t k = 0; k < n; ++k) out[k + 1] = (double)c[k];
    out[n + 1] = (double)(c[n - 2] + 2.0L * h * dn);
    return out;
}

struct HostPulse {
    const hhg_pulse_desc &q;
    std::vector<double> coef;  // SPLINE
    explicit HostPulse(const hhg_pulse_desc &p) : q(p) {
        if (q.kind == HHG_PULSE_SPLINE)
            coef = spline_coefficients(q.samples, q.n_samples, q.sample_dt, q.deriv_begin, q.deriv_end);
    }
    // GaussLaser (GaussLaser.cpp): centre and 2 sigma^2
    long double gauss_c() const { return q.t_begin + 3.0L * kPi * q.n_cycles; }
    double gauss_2s2() const {
        const double sigma = kPi * q.n_cycles / std::sqrt(2.0 * std::log(1.0 / 0.05));
        return 2.0 * sigma * sigma;
    }
    long double spline_ld(long double t) const {
        const int64_t n = q.n_samples;
        const long double u = (t - q.t_begin) / q.sample_dt;
        int64_t k = (int64_t)floorl(u);
        k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
        const long double x = u - k, y = 1.0L - x;
        const double *c = coef.data() + k;
        return (y * y * y * c[0] + (3 * x * x * x - 6 * x * x + 4) * c[1] +
                (-3 * x * x * x + 3 * x * x + 3 * x + 1) * c[2] + x * x * x * c[3]) / 6.0L;
    }
    // A(t) without the window cut
    long double continued_ld(long double t) const {
        switch (q.kind) {
        case HHG_PULSE_CONTINUOUS: return (long double)q.amplitude * sinl(t + q.phase);
        case HHG_PULSE_GAUSS: {
            const long double x = t - gauss_c();
            return (long double)q.amplitude * expl(-(x * x) / gauss_2s2()) * sinl(t + q.phase);
        }
        case HHG_PULSE_SPLINE: return (long double)q.amplitude * spline_ld(t);
        default: {
            const long double inv = 1.0L / q.n_cycles;
            return (long double)q.amplitude * ((0.5L * (1.0L - cosl(inv * (t - q.t_begin)))) * sinl(t + q.phase));
        }
        }
    }
    // the open window outside which A = 0
    void window(double &tb, double &te) const {
        tb = -INFINITY;
        te = INFINITY;
        if (q.kind == HHG_PULSE_COSINE) {
            tb = q.t_begin;
            te = q.t_begin + 2 * kPi * q.n_cycles;  // CosineLaser::base_duration (CosineLaser.hpp:13-15)
        } else if (q.kind == HHG_PULSE_SPLINE) {
            te = std::nextafter(q.spline_cut, INFINITY);  // A(t) = 0 for t > t_end (Laser.hpp:35)
        }
    }
    // A(t) as the device's laser_exact
    double value(double t) const {
        if (q.kind == HHG_PULSE_COSINE) {
            const double te = q.t_begin + 2 * kPi * q.n_cycles;
            double env = 0.0;
            if (!(t <= q.t_begin || t >= te)) env = 0.5 * (1. - cos((1. / q.n_cycles) * (t - q.t_begin)));
            return q.amplitude * (env * sin(t + q.phase));
        }
        double tb, te;
        window(tb, te);
        if (t <= tb || t >= te) return 0.0;
        return (double)continued_ld(t);
    }
};

// Everything of a device pulse record that depends on the pulse alone; the
// spline coefficient pointer is set by the caller once the device copy exists.
void fill_pulse_dev(const hhg_pulse_desc &q, const HostPulse &hp, PulseDev &d) {
    d.amplitude = q.amplitude;
    hp.window(d.t_begin, d.t_end);
    d.inv_n_cycles = q.kind == HHG_PULSE_COSINE ? 1. / q.n_cycles : 0.0;
    d.phase = q.phase;
    d.window_begin = q.window_begin;
    d.measure_every = (q.window_end - q.window_begin) / q.n_measurements;
    d.dt0 = d.measure_every / q.n_subdivisions;
    d.kind = q.kind;
    if (q.kind == HHG_PULSE_GAUSS) {
        d.gauss_c = (double)hp.gauss_c();
        d.gauss_2s2 = hp.gauss_2s2();
    }
    if (q.kind == HHG_PULSE_SPLINE) {
        d.spline_n = (int)q.n_samples;
        d.spline_t0 = q.t_begin;
        d.spline_inv_h = 1.0 / q.sample_dt;
    }
    d.n_meas = q.n_measurements;
}

// Chebyshev-tail threshold of the staged interpolants: 2^-56 of the function
// scale, tested on up to 257 evenly spread intervals (the analytic pulses
// are uniformly smooth).  A spline pulse is only C2 at its knots: at the
// reference's sampling (1024 intervals per cycle, DoubleLaser's 1000 knots
// over 1.5 pulse durations) the tail of an interval holding a knot is ~4e-16
// of the scale in the median and up to 3e-12 where the sampled sub-pulse has a
// kink (the CosineLaser's window edge) or its steepest curvature, so the
// spline threshold is 2^-36 and every interval is tested; knots denser than
// the intervals, or a spline that turns within a knot or two (QuenchedField's
// step, 4e-9), are refused.
// Chebyshev nodes cos(pi (k + 1/2) / 16) and the DCT matrix cos(pi j (k + 1/2) / 16)
// of the degree test, in long double, computed once.
struct ChebTables {
    static constexpr int NN = 16;
    long double node[NN], dct[NN][NN];
    ChebTables() {
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int k = 0; k < NN; ++k) node[k] = cosl(pi * (k + 0.5L) / NN);
        for (int j = 0; j < NN; ++j)
            for (int k = 0; k < NN; ++k) dct[j][k] = cosl(pi * j * (k + 0.5L) / NN);
    }
};

int choose_degree(const hhg_pulse_desc &p, const double *proj, int nf) {
    static const ChebTables tab;
    const HostPulse hp(p);
    const int NN = ChebTables::NN;
    const long double me = ((long double)p.window_end - p.window_begin) / p.n_measurements;
    const int samples = p.kind == HHG_PULSE_SPLINE ? p.n_measurements : std::min(p.n_measurements, 257);
    long double tail5 = 0.0L, tail7 = 0.0L, tail11 = 0.0L, scale = 1.0L;
    for (int q = 0; q < samples; ++q) {
        const int i = (int)((long long)q * p.n_measurements / samples);
        const long double ctr = p.window_begin + (i + 0.5L) * me, half = 0.5L * me;
        const int groups = nf == 1 ? 1 : nf / 2;
        for (int n = 0; n < groups; ++n) {
            for (int part = 0; part < (nf == 1 ? 1 : 2); ++part) {
                long double fv[NN];
                for (int k = 0; k < NN; ++k) {
                    const long double A = hp.continued_ld(ctr + half * tab.node[k]);
                    if (nf == 1) fv[k] = A;
                    else fv[k] = part == 0 ? cosl(proj[n] * A) : sinl(proj[n] * A);
                }
                for (int j = 0; j < NN; ++j) {
                    long double acc = 0.0L;
                    for (int k = 0; k < NN; ++k) acc += fv[k] * tab.dct[j][k];
                    acc = fabsl(acc * 2.0L / NN);
                    if (j == 0) scale = std::max(scale, acc);
                    if (j > 5) tail5 = std::max(tail5, acc);
                    if (j > 7) tail7 = std::max(tail7, acc);
                    if (j > 11) tail11 = std::max(tail11, acc);
                }
            }
        }
    }
    const long double thr = ldexpl(1.0L, p.kind == HHG_PULSE_SPLINE ? -36 : -56) * scale;
    if (tail5 <= thr) return 5;
    if (tail7 <= thr) return 7;
    if (tail11 <= thr) return 11;
    return -1;
}

// Thermal and relaxation constants of the *_RELAX kernel models, in the
// pulse's energy units (energy_scale es multiplies energies and rates,
// divides beta): [1] 2t (PiFlux occupation energies), [4] E_F, [5] beta,
// [6] diagonal rate, [7] off-diagonal rate.
void set_relax_params(const hhg_system_desc &s, double es, double *mp) {
    if (s.inv_diag_relax <= 0.0) return;
    if (s.kind == HHG_SYS_PIFLUX3D) mp[1] = 2.0 * s.hopping * es;
    mp[4] = s.fermi_energy * es;
    mp[5] = s.beta / es;
    mp[6] = s.inv_diag_relax * es;
    mp[7] = s.inv_offdiag_relax * es;
}

// A(t) of one pulse on the host, as the device's laser_exact.
double host_laser(const hhg_pulse_desc &q, double t) { return HostPulse(q).value(t); }

// Requests the relaxation kernels do not cover.
hhg_status check_relax(hhg_ctx *ctx, const hhg_system_desc &s, const hhg_pulse_desc *pulses,
                       int n_pulses, const hhg_solver_opts &o) {
    if (s.inv_diag_relax <= 0.0) return HHG_OK;
    if (o.stepper != HHG_STEPPER_RKF78 || o.precision != HHG_PREC_FP64)
        return set_err(ctx, HHG_UNSUPPORTED, "relaxation right-hand sides run with FP64 RKF78 only");
    if (s.kind == HHG_SYS_PIFLUX3D && s.beta != 0.0 && s.inv_offdiag_relax > 0.0 &&
        o.proposer != HHG_PROPOSER_NONE)
        // the off-diagonal equilibrium reads the step's start state
        // (PiFlux.cpp:145), so j(t) is a first-order function of the step
        // sequence: only the reference schedule reproduces the reference
        return set_err(ctx, HHG_UNSUPPORTED,
                       "PiFlux relaxation at T > 0 depends on the step sequence; use the reference "
                       "step schedule (HHG_PROPOSER_NONE)");
    if (s.kind == HHG_SYS_HONEYCOMB)
        for (int p = 0; p < n_pulses; ++p)
            if (host_laser(pulses[p], pulses[p].window_begin) != 0.0)
                // the reference starts from the equilibrium at k - A(t_begin)
                // (Honeycomb.cpp:193-194); the k table holds the one at A = 0
                return set_err(ctx, HHG_UNSUPPORTED,
                               "honeycomb relaxation needs A(window_begin) = 0 (window starting "
                               "at or before the pulse)");
    return HHG_OK;
}

hhg_status launch_variant(const hhg_plan *pl, hhg::LaunchReq &r) {
    cudaError_t e = cudaErrorInvalidValue;
    switch (pl->model) {
    case HHG_SYS_DIRAC2D: e = hhg::launch_dirac2d(r); break;
    case HHG_SYS_PIFLUX2D: e = hhg::launch_piflux2d(r); break;
    case HHG_SYS_PIFLUX3D: e = hhg::launch_piflux3d(r); break;
    case HHG_SYS_HONEYCOMB: e = hhg::launch_honeycomb(r); break;
    case HHG_SYS_DIRAC3D: e = hhg::launch_dirac3d(r); break;
    case hhg::PIFLUX2D_SYM: e = hhg::launch_piflux2d_sym(r); break;
    case hhg::HONEYCOMB_X: e = hhg::launch_honeycomb_x(r); break;
    case hhg::PIFLUX3D_RELAX: e = hhg::launch_piflux3d_relax(r); break;
    case hhg::HONEYCOMB_RELAX: e = hhg::launch_honeycomb_relax(r); break;
    case hhg::DIRAC3D_RELAX: e = hhg::launch_dirac3d_relax(r); break;
    }
    if (e != cudaSuccess)
        return set_err(pl->ctx, HHG_CUDA_ERROR, std::string("integration launch: ") + cudaGetErrorString(e));
    return HHG_OK;
}

hhg_status stage_variant(const hhg_plan *pl, hhg::StageReq &s) {
    cudaError_t e = cudaErrorInvalidValue;
    switch (pl->model) {
    case HHG_SYS_DIRAC2D: e = hhg::stage_dirac2d(s); break;
    case HHG_SYS_PIFLUX2D: e = hhg::stage_piflux2d(s); break;
    case HHG_SYS_PIFLUX3D: e = hhg::stage_piflux3d(s); break;
    case HHG_SYS_HONEYCOMB: e = hhg::stage_honeycomb(s); break;
    case HHG_SYS_DIRAC3D: e = hhg::stage_dirac3d(s); break;
    case hhg::PIFLUX2D_SYM: e = hhg::stage_piflux2d_sym(s); break;
    case hhg::HONEYCOMB_X: e = hhg::stage_honeycomb_x(s); break;
    case hhg::PIFLUX3D_RELAX: e = hhg::stage_piflux3d_relax(s); break;
    case hhg::HONEYCOMB_RELAX: e = hhg::stage_honeycomb_relax(s); break;
    case hhg::DIRAC3D_RELAX: e = hhg::stage_dirac3d_relax(s); break;
    }
    if (e != cudaSuccess)
        return set_err(pl->ctx, HHG_CUDA_ERROR, std::string("staging launch: ") + cudaGetErrorString(e));
    return HHG_OK;
}

}  // namespace

extern "C" {

int hhg_abi_version(void) { return HHG_ABI_VERSION; }

void hhg_default_solver_opts(hhg_solver_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->stepper = HHG_STEPPER_RKF78;
    o->precision = HHG_PREC_FP64;
    o->proposer = HHG_PROPOSER_NONE;
    o->magnus_substeps = 1;
    o->abs_tol = 1.0e-12;  // PiFlux.cpp:20-21
    o->rel_tol = 1.0e-8;
    o->max_failed_steps = 500;
    o->max_attempts_per_interval = 100000;
    o->tile_k = 0;
    o->block_threads = 128;
    o->mlp = nullptr;
    o->mlp_every = 16;
    o->coarsen_div = 0;
}

hhg_status hhg_gpu_create(hhg_ctx **out, int device) {
    if (!out) return HHG_BAD_CONFIG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return HHG_CUDA_ERROR;
    if (device < 0 || device >= n) return HHG_BAD_CONFIG;
    hhg_ctx *c = new hhg_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return HHG_CUDA_ERROR;
    }
    for (auto &e : c->ev) cudaEventCreate(&e);
    *out = c;
    return HHG_OK;
}

void hhg_gpu_destroy(hhg_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    for (auto &kv : c->plan_cache) hhg_plan_destroy(kv.second);
    c->plan_cache.clear();
    if (c->kappa_plan) hhg_plan_destroy(c->kappa_plan);
    c->ktab_shared.reset();
    for (hhg_ctx::Grow *g : {&c->kappa_T, &c->kappa_items, &c->kappa_change, &c->kappa_j, &c->kappa_slice})
        cudaFree(g->p);
    for (auto &kv : c->fft_plans) cufftDestroy(kv.second);
    cudaFree(c->d_x);
    cudaFree(c->d_F);
    cudaFree(c->d_out);
    for (auto &e : c->ev) cudaEventDestroy(e);
    cudaStreamDestroy(c->stream);
    delete c;
}

const char *hhg_last_error(const hhg_ctx *c) { return c ? c->last_error.c_str() : "null context"; }

hhg_status hhg_gauss_legendre(int n, double *x, double *w) {
    if (n < 1 || n > 1 << 20 || !x || !w) return HHG_BAD_CONFIG;
    gauss_legendre(n, x, w);
    return HHG_OK;
}

hhg_status hhg_grid_rows(const hhg_system_desc *sys, const hhg_grid_desc *grid, double *rows,
                         int64_t *n_rows) {
    hhg_status st = check_system(nullptr, sys);
    if (st != HHG_OK) return st;
    st = check_grid(nullptr, grid);
    if (st != HHG_OK) return st;
    const int64_t n = grid_count(*grid);
    if (n_rows) *n_rows = n;
    if (rows) build_rows(*sys, *grid, rows);
    return HHG_OK;
}

// cost_order: for the PiFlux-3D models, order the k rows by a cost
// proxy (below); plans whose outputs are indexed by k keep the caller's order.
static hhg_status plan_create_impl(hhg_ctx *ctx, const hhg_system_desc *sys,
                                   const hhg_pulse_desc *pulses, int n_pulses,
                                   const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                                   hhg_plan **out, bool cost_order) {
    if (!ctx || !out) return HHG_BAD_CONFIG;
    *out = nullptr;
    hhg_status st = check_system(ctx, sys);
    if (st != HHG_OK) return st;
    st = check_grid(ctx, grid);
    if (st != HHG_OK) return st;
    if (!pulses || n_pulses < 1 || n_pulses > (1 << 20))
        return set_err(ctx, HHG_BAD_CONFIG, "need at least one pulse");
    for (int p = 0; p < n_pulses; ++p)
        if ((st = check_pulse(ctx, pulses[p])) != HHG_OK) return st;
    hhg_solver_opts o;
    hhg_default_solver_opts(&o);
    if (opts) o = *opts;
    if (o.stepper != HHG_STEPPER_RKF78 && o.stepper != HHG_STEPPER_MAGNUS4 &&
        o.stepper != HHG_STEPPER_DIRAC_MAGNUS)
        return set_err(ctx, HHG_BAD_CONFIG, "unknown stepper");
    if (o.stepper == HHG_STEPPER_DIRAC_MAGNUS &&
        (sys->kind != HHG_SYS_DIRAC3D || o.precision != HHG_PREC_FP64 ||
         o.proposer != HHG_PROPOSER_NONE))
        return set_err(ctx, HHG_UNSUPPORTED,
                       "the closed-form Magnus step is the Dirac-3D model's, in FP64, one step per "
                       "interval (no step proposer)");
    if (o.stepper == HHG_STEPPER_MAGNUS4 && !hhg_prep::magnus_substeps_ok(o.magnus_substeps))
        return set_err(ctx, HHG_BAD_CONFIG, "magnus_substeps out of range");
    if (o.stepper == HHG_STEPPER_MAGNUS4 && o.precision != HHG_PREC_FP64)
        return set_err(ctx, HHG_UNSUPPORTED, "Magnus-4 runs in FP64 only");
    if (o.precision != HHG_PREC_FP64 && o.precision != HHG_PREC_MIXED)
        return set_err(ctx, HHG_BAD_CONFIG, "unknown precision");
    if (o.proposer != HHG_PROPOSER_NONE && o.proposer != HHG_PROPOSER_CARRY &&
        o.proposer != HHG_PROPOSER_LOCKSTEP && o.proposer != HHG_PROPOSER_LEARNED)
        return set_err(ctx, HHG_BAD_CONFIG, "unknown proposer");
    if (o.proposer == HHG_PROPOSER_LEARNED) {
        if (!o.mlp || !(o.mlp->out_sigma > 0.0f))
            return set_err(ctx, HHG_BAD_CONFIG,
                           "the learned proposer needs opts.mlp: a network from hhg_mlp_init + hhg_mlp_train");
        if (o.mlp_every < 1) return set_err(ctx, HHG_BAD_CONFIG, "mlp_every must be >= 1");
        if (o.stepper != HHG_STEPPER_RKF78)
            return set_err(ctx, HHG_UNSUPPORTED, "the learned proposer drives the RKF78 stepper");
    }
    if (!(o.abs_tol >= 0.0) || !(o.rel_tol >= 0.0) || !(o.abs_tol + o.rel_tol > 0.0))
        return set_err(ctx, HHG_BAD_CONFIG, "tolerances must be >= 0 and not both 0");
    if (o.coarsen_div != 0 && (o.coarsen_div < 2 || o.coarsen_div > 65536))
        return set_err(ctx, HHG_BAD_CONFIG, "coarsen_div must be 0 (default) or in 2 .. 65536");
    if (o.max_failed_steps < 1) o.max_failed_steps = 500;
    if (o.max_attempts_per_interval < 1) o.max_attempts_per_interval = 100000;
    if ((st = check_relax(ctx, *sys, pulses, n_pulses, o)) != HHG_OK) return st;

    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    hhg_plan *pl = new hhg_plan();
    pl->ctx = ctx;
    pl->model = kernel_model(*sys);
    pl->opts = o;
    pl->n_pulses = n_pulses;
    const int nf = model_nf(pl->model);

    // k table: built here, or the context's shared table of the same system
    // and generated grid (the cost-ordered tables depend on the pulse and
    // explicit rows are the caller's: neither is shared)
    pl->n_k = grid_count(*grid);
    const bool cost_sort = cost_order && hhg::base_model(pl->model) == hhg::PIFLUX3D && pl->n_k > 32 &&
                           (o.proposer == HHG_PROPOSER_NONE || o.proposer == HHG_PROPOSER_CARRY);
    const bool share_ktab = !cost_sort && grid->kind != HHG_GRID_EXPLICIT;
    const std::string kkey = share_ktab ? ktab_key(sys, grid) : std::string();
    const bool reuse_ktab = share_ktab && ctx->ktab_shared && ctx->ktab_key == kkey;
    std::vector<double> ktab;
    if (!reuse_ktab) {
        ktab.resize((size_t)pl->n_k * 8);
        build_rows(*sys, *grid, ktab.data());
    }
    if (cost_sort) {
        // With per-lane step control a warp's lanes finish together only if
        // their k-points need similar numbers of steps.  The step count
        // follows the time average of |d(k - A(t))| (correlation -0.43
        // measured on the oracle, relaxation path); a stable sort by it raised
        // the active lanes of a warp from 0.83 to 0.90 of 32.  Only the
        // (fixed) order of the Brillouin-zone sum changes.  Warp-synchronous
        // (dyadic) stepping is left in the grid's order: there a warp takes
        // its finest lane's level at every moment, and the grid's slices keep
        // lanes whose needs peak together (same k_z) in one warp (the sort
        // measured 7 % slower there).
        const hhg_pulse_desc &q0 = pulses[0];
        const HostPulse hp(q0);
        constexpr int kT = 256;
        double cA[kT], sA[kT];
        for (int i = 0; i < kT; ++i) {
            const double A = hp.value(q0.window_begin + (q0.window_end - q0.window_begin) * (i + 0.5) / kT);
            cA[i] = cos(A);
            sA[i] = sin(A);
        }
        std::vector<double> key((size_t)pl->n_k);
        for (int64_t r = 0; r < pl->n_k; ++r) {
            const double *row = ktab.data() + 8 * r;
            const double cx = cos(row[0]), cy = cos(row[1]), cz = cos(row[2]), sz = sin(row[2]);
            const double p2 = cx * cx + cy * cy;
            double acc = 0.0;
            for (int i = 0; i < kT; ++i) {
                const double u = cz * cA[i] + sz * sA[i];
                acc += sqrt(p2 + u * u);
            }
            key[(size_t)r] = acc;
        }
        std::vector<int64_t> order((size_t)pl->n_k);
        for (int64_t r = 0; r < pl->n_k; ++r) order[(size_t)r] = r;
        std::stable_sort(order.begin(), order.end(),
                         [&](int64_t a, int64_t b) { return key[(size_t)a] < key[(size_t)b]; });
        std::vector<double> sorted(ktab.size());
        for (int64_t r = 0; r < pl->n_k; ++r)
            std::memcpy(sorted.data() + 8 * r, ktab.data() + 8 * order[(size_t)r], 8 * sizeof(double));
        ktab.swap(sorted);
    }

    // per-pulse records, staged projections and degree
    const double nny = 0.5 * kSqrt3;
    double proj[3] = {0, 0, 0};
    switch (hhg::base_model(pl->model)) {
    case hhg::PIFLUX2D:
        proj[0] = sys->pol_x;
        proj[1] = sys->pol_y;
        break;
    case hhg::PIFLUX2D_SYM:
        proj[0] = sys->pol_x;
        break;
    case hhg::HONEYCOMB:
        proj[0] = 1.0 * sys->pol_x + 0.0 * sys->pol_y;
        proj[1] = -0.5 * sys->pol_x + nny * sys->pol_y;
        proj[2] = -0.5 * sys->pol_x - nny * sys->pol_y;
        break;
    case hhg::HONEYCOMB_X:
        proj[0] = sys->pol_x;
        proj[1] = -0.5 * sys->pol_x;
        break;
    case hhg::PIFLUX3D:
        proj[0] = 1.0;
        break;
    }
    // A spline pulse whose knots a per-interval polynomial cannot follow (a
    // step between two knots) is evaluated exactly at every stage time
    // (degree 0), in FP64 RKF78 with the reference schedule or the carried step.
    const bool exact_ok = o.stepper == HHG_STEPPER_RKF78 && o.precision == HHG_PREC_FP64 &&
                          (o.proposer == HHG_PROPOSER_NONE || o.proposer == HHG_PROPOSER_CARRY);
    int degree = 5;
    bool exact = false;
    // the degree test costs ~5 ms of long-double work per pulse: pulses in parallel
    std::vector<int> degs((size_t)n_pulses);
    parallel_for(n_pulses, [&](int p) { degs[(size_t)p] = choose_degree(pulses[p], proj, nf); }, 2);
    for (int p = 0; p < n_pulses; ++p) {
        const int d = degs[(size_t)p];
        if (d < 0 && pulses[p].kind == HHG_PULSE_SPLINE && exact_ok) {
            exact = true;
            continue;
        }
        if (d < 0) {
            delete pl;
            return set_err(ctx, HHG_UNSUPPORTED,
                           pulses[p].kind == HHG_PULSE_SPLINE
                               ? "spline pulse: knots too dense or too steep for the staged "
                                 "interpolants; exact evaluation runs FP64 RKF78 with the NONE or "
                                 "CARRY proposer"
                               : "measurement interval too coarse for the staged pulse interpolants");
        }
        degree = std::max(degree, d);
    }
    pl->degree = exact ? 0 : degree;
    degree = pl->degree;
    const bool dyadic = o.proposer == HHG_PROPOSER_LOCKSTEP || o.proposer == HHG_PROPOSER_LEARNED;
    const int slot = dyadic ? hhg::slot_doubles_dyadic(nf, degree) : hhg::slot_doubles(nf, degree);

    // work decomposition
    const int64_t tiles = (pl->n_k + 31) / 32;
    int tpi = o.tile_k > 0 ? o.tile_k : 1;
    if (o.tile_k <= 0) {
        // auto: keep at least ~8 items per resident warp when there is work
        // for that, and the partial buffer below 8 GB
        const long long resident = (long long)ctx->sm_count * hhg::kWarpsPerBlock * hhg::kMinBlocksPerSM;
        long long total_samples = 0;
        for (int p = 0; p < n_pulses; ++p) total_samples += pulses[p].n_measurements + 1;
        while (true) {
            const long long items = (long long)n_pulses * ((tiles + tpi - 1) / tpi);
            const double part_bytes = 8.0 * (double)((tiles + tpi - 1) / tpi) * (double)total_samples;
            if (part_bytes > 8e9 || items > 64 * resident) {
                if (tpi >= tiles) break;
                tpi *= 2;
                continue;
            }
            break;
        }
    }
    pl->tiles_per_item = tpi;
    pl->items_per_pulse = (int)((tiles + tpi - 1) / tpi);
    pl->n_items = (long long)pl->items_per_pulse * n_pulses;

    pl->pulses.resize(n_pulses);
    pl->window_end.resize(n_pulses);
    for (int p = 0; p < n_pulses; ++p) pl->window_end[p] = pulses[p].window_end;
    std::vector<long long> ioff(n_pulses + 1, 0);
    long long coef_len = 0, part_len = 0, j_len = 0;
    std::vector<double> spline_coef;  // spline pulses' coefficients, stored after the slots
    std::vector<long long> spline_off(n_pulses, -1);
    for (int p = 0; p < n_pulses; ++p) {
        const hhg_pulse_desc &q = pulses[p];
        PulseDev &d = pl->pulses[p];
        std::memset(&d, 0, sizeof d);
        const HostPulse hp(q);
        fill_pulse_dev(q, hp, d);
        if (q.kind == HHG_PULSE_SPLINE) {
            spline_off[p] = (long long)spline_coef.size();
            spline_coef.insert(spline_coef.end(), hp.coef.begin(), hp.coef.end());
        }
        const double es = q.energy_scale;
        switch (sys->kind) {
        case HHG_SYS_DIRAC2D:
            d.mp[0] = 2.0 * sys->velocity * es;
            d.mp[1] = 2.0 * sys->mass * es;
            break;
        case HHG_SYS_PIFLUX3D:
            d.mp[0] = 4.0 * sys->hopping * es;
            break;
        case HHG_SYS_PIFLUX2D:
            d.mp[0] = -4.0 * sys->hopping * es;
            break;
        case HHG_SYS_HONEYCOMB:
            d.mp[0] = 2.0 * sys->hopping * es;
            d.mp[1] = 2.0 * sys->mass * es;
            break;
        default:
            break;
        }
        d.mp[2] = sys->pol_x;
        d.mp[3] = sys->pol_y;
        set_relax_params(*sys, es, d.mp);
        for (int n = 0; n < 3; ++n) d.s[n] = proj[n];
        // sample-0 record, exact: A(t_0) and the staged functions at it
        const double A0 = hp.value(0 * d.measure_every + d.window_begin);
        d.s0rec[0] = A0;
        if (nf == 1) d.s0rec[1] = A0;
        else if (hhg::base_model(pl->model) == hhg::PIFLUX3D) {
            d.s0rec[1] = cos(A0);
            d.s0rec[2] = sin(A0);
        } else
            for (int n = 0; n < nf / 2; ++n) {
                d.s0rec[1 + 2 * n] = cos(proj[n] * A0);
                d.s0rec[2 + 2 * n] = sin(proj[n] * A0);
            }
        d.n_meas = q.n_measurements;
        d.items = pl->items_per_pulse;
        d.coef_off = coef_len;
        d.part_off = part_len;
        d.j_off = j_len;
        coef_len += (long long)q.n_measurements * slot;
        part_len += (long long)pl->items_per_pulse * (q.n_measurements + 1);
        j_len += q.n_measurements + 1;
        ioff[p + 1] = ioff[p] + q.n_measurements;
    }
    // the Dirac Magnus staging reads the reference's 30-point rule on [0, 1]
    // (gauss.hpp:14-80: negative nodes by increasing |x|, then positive ones),
    // stored after the staging slots
    const bool magnus_moments = o.stepper == HHG_STEPPER_DIRAC_MAGNUS;
    std::vector<double> gl30;
    if (magnus_moments) {
        double x[30], w[30];
        gauss_legendre(30, x, w);
        gl30.assign(60, 0.0);
        for (int i = 0; i < 15; ++i) {
            gl30[i] = 0.5 * (-x[15 + i] + 1.);
            gl30[15 + i] = 0.5 * (x[15 + i] + 1.);
            gl30[30 + i] = 0.5 * w[15 + i];
            gl30[45 + i] = 0.5 * w[15 + i];
        }
    }
    const long long gl_off = coef_len;
    if (magnus_moments) coef_len += 60;
    const long long spline_base = coef_len;
    coef_len += (long long)spline_coef.size();
    pl->coef_len = coef_len;
    pl->part_len = part_len;
    pl->j_len = j_len;
    pl->n_intervals = ioff[n_pulses];
    // accumulated interval ends (t_begin = t_end; t_end += measure_every, PiFlux.cpp:108-109)
    std::vector<double> tgrid((size_t)(pl->n_intervals + n_pulses));
    for (int p = 0; p < n_pulses; ++p) {
        double *tg = tgrid.data() + ioff[p] + p;
        double t_begin = pl->pulses[p].window_begin;
        double t_end = t_begin + pl->pulses[p].measure_every;
        tg[0] = t_begin;
        for (int i = 1; i <= pulses[p].n_measurements; ++i) {
            tg[i] = t_end;
            t_begin = t_end;
            t_end += pl->pulses[p].measure_every;
        }
    }

    auto fail = [&](const char *what, cudaError_t e) {
        hhg_plan_destroy(pl);
        return set_err(ctx, HHG_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    cudaStream_t s = ctx->stream;
    if (reuse_ktab) {
        pl->ktab_owner = ctx->ktab_shared;
        pl->d_ktab = pl->ktab_owner.get();
    } else if ((e = cudaMalloc(&pl->d_ktab, ktab.size() * sizeof(double))) != cudaSuccess) {
        return fail("alloc k table", e);
    } else if (share_ktab) {
        pl->ktab_owner = std::shared_ptr<double>(pl->d_ktab, [](double *p) { cudaFree(p); });
        ctx->ktab_shared = pl->ktab_owner;
        ctx->ktab_key = kkey;
    }
    if ((e = cudaMalloc(&pl->d_pulses, n_pulses * sizeof(PulseDev))) != cudaSuccess) return fail("alloc pulses", e);
    if ((e = cudaMalloc(&pl->d_coef, coef_len * sizeof(double))) != cudaSuccess) return fail("alloc staging", e);
    if ((e = cudaMalloc(&pl->d_part, part_len * sizeof(double))) != cudaSuccess) return fail("alloc partials", e);
    if ((e = cudaMalloc(&pl->d_j, j_len * sizeof(double))) != cudaSuccess) return fail("alloc j", e);
    if ((e = cudaMalloc(&pl->d_tgrid, tgrid.size() * sizeof(double))) != cudaSuccess) return fail("alloc tgrid", e);
    if ((e = cudaMalloc(&pl->d_ioff, ioff.size() * sizeof(long long))) != cudaSuccess) return fail("alloc offsets", e);
    if ((e = cudaMalloc(&pl->d_counters, 8 * sizeof(unsigned long long))) != cudaSuccess) return fail("alloc counters", e);
    if ((e = cudaMalloc(&pl->d_status, sizeof(int))) != cudaSuccess) return fail("alloc status", e);
    for (int p = 0; p < n_pulses; ++p)
        if (spline_off[p] >= 0) pl->pulses[p].spline = pl->d_coef + spline_base + spline_off[p];
    if (o.proposer == HHG_PROPOSER_LEARNED) {
        hhg::MlpPacked packed;
        hhg::pack_mlp(*o.mlp, &packed);
        if ((e = cudaMalloc(&pl->d_mlp, sizeof packed)) != cudaSuccess) return fail("alloc network", e);
        // synchronous: `packed` lives on this stack frame
        if ((e = cudaMemcpy(pl->d_mlp, &packed, sizeof packed, cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail("upload network", e);
        pl->opts.mlp = nullptr;  // the plan keeps its device copy only
    }
    if (!reuse_ktab &&
        (e = cudaMemcpyAsync(pl->d_ktab, ktab.data(), ktab.size() * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return fail("upload k table", e);
    if ((e = cudaMemcpyAsync(pl->d_pulses, pl->pulses.data(), n_pulses * sizeof(PulseDev), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail("upload pulses", e);
    if ((e = cudaMemcpyAsync(pl->d_tgrid, tgrid.data(), tgrid.size() * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail("upload tgrid", e);
    if ((e = cudaMemcpyAsync(pl->d_ioff, ioff.data(), ioff.size() * sizeof(long long), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail("upload offsets", e);
    if (magnus_moments &&
        (e = cudaMemcpyAsync(pl->d_coef + gl_off, gl30.data(), 60 * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return fail("upload quadrature", e);
    if (!spline_coef.empty() &&
        (e = cudaMemcpyAsync(pl->d_coef + spline_base, spline_coef.data(), spline_coef.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return fail("upload pulse splines", e);
    hhg::StageReq sr{pl->d_pulses, n_pulses, pl->d_tgrid, pl->d_ioff, pl->d_coef,
                     pl->n_intervals, degree, 9.0 / 10.0 * pow(pow(5.0, -8.0), -1.0 / 8), s};
    sr.layout = dyadic ? (o.precision == HHG_PREC_MIXED ? 2 : 1) : (magnus_moments ? 3 : 0);
    if (magnus_moments) sr.gl30 = pl->d_coef + gl_off;
    if ((st = stage_variant(pl, sr)) != HHG_OK) {
        hhg_plan_destroy(pl);
        return st;
    }
    // persistent grid: resident CTAs, but no more than the items need
    int occ = 0;
    hhg::LaunchReq lr{};
    lr.degree = degree;
    lr.precision = o.precision;
    lr.stepper = o.stepper;
    lr.proposer = kernel_proposer(o.proposer);
    lr.grid = 0;
    lr.occupancy_out = &occ;
    if ((st = launch_variant(pl, lr)) != HHG_OK) {
        hhg_plan_destroy(pl);
        return st;
    }
    pl->occupancy = std::max(occ, 1);
    pl->part_cap = part_len;
    const long long max_ctas = (long long)std::max(occ, 1) * ctx->sm_count;
    const long long need = (pl->n_items + hhg::kWarpsPerBlock - 1) / hhg::kWarpsPerBlock;
    pl->grid = (int)std::max(1LL, std::min(max_ctas, need));
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail("plan setup", e);
    *out = pl;
    return HHG_OK;
}

hhg_status hhg_plan_create(hhg_ctx *ctx, const hhg_system_desc *sys, const hhg_pulse_desc *pulses,
                           int n_pulses, const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                           hhg_plan **out) {
    return plan_create_impl(ctx, sys, pulses, n_pulses, grid, opts, out, true);
}

void hhg_plan_destroy(hhg_plan *pl) {
    if (!pl) return;
    cudaSetDevice(pl->ctx->device);
    if (pl->ktab_owner) pl->ktab_owner.reset();  // the context may still hold the table
    else cudaFree(pl->d_ktab);
    cudaFree(pl->d_pulses);
    cudaFree(pl->d_coef);
    cudaFree(pl->d_part);
    cudaFree(pl->d_j);
    cudaFree(pl->d_tgrid);
    cudaFree(pl->d_ioff);
    cudaFree(pl->d_counters);
    cudaFree(pl->d_status);
    cudaFree(pl->d_spec);
    cudaFree(pl->d_x);
    cudaFree(pl->d_F);
    cudaFree(pl->d_mlp);
    cudaFree(pl->d_hist);
    cudaFree(pl->d_hist_count);
    cudaFree(pl->d_kout);
    if (pl->gexec) cudaGraphExecDestroy(pl->gexec);
    delete pl;
}

int64_t hhg_plan_j_length(const hhg_plan *pl) { return pl ? pl->j_len : 0; }

const double *hhg_plan_device_j(const hhg_plan *pl) { return pl ? pl->d_j : nullptr; }

}  // extern "C"

namespace {
// Integration + reduction of one execution on stream s; with `events` the
// context's timing events bracket the launches (not inside a graph capture).
hhg_status enqueue_integration(hhg_plan *pl, cudaStream_t s, bool events) {
    hhg_ctx *ctx = pl->ctx;
    HHG_CUDA(ctx, cudaMemsetAsync(pl->d_counters, 0, 8 * sizeof(unsigned long long), s));
    HHG_CUDA(ctx, cudaMemsetAsync(pl->d_status, 0, sizeof(int), s));
    hhg::LaunchReq lr{};
    lr.kp.ktab = pl->d_ktab;
    lr.kp.pulses = pl->d_pulses;
    lr.kp.coef = pl->d_coef;
    lr.kp.part = pl->d_part;
    lr.kp.counters = pl->d_counters;
    lr.kp.status = pl->d_status;
    lr.kp.n_items = pl->n_items;
    lr.kp.n_k = (int)pl->n_k;
    lr.kp.tiles_per_item = pl->tiles_per_item;
    lr.kp.items_per_pulse = pl->items_per_pulse;
    lr.kp.max_failed = pl->opts.max_failed_steps;
    lr.kp.max_attempts = pl->opts.max_attempts_per_interval;
    lr.kp.magnus_substeps = pl->opts.magnus_substeps;
    lr.kp.abs_tol = pl->opts.abs_tol;
    lr.kp.rel_tol = pl->opts.rel_tol;
    lr.kp.err_floor = pow(5.0, -8.0);
    lr.kp.grow_max = 9.0 / 10.0 * pow(pow(5.0, -8.0), -1.0 / 8);
    lr.kp.mlp = pl->d_mlp;
    lr.kp.mlp_every = std::max(pl->opts.mlp_every, 1);
    lr.kp.coarsen = 1.0 / (pl->opts.coarsen_div > 0 ? pl->opts.coarsen_div
                           : pl->opts.precision == HHG_PREC_MIXED ? hhg::kCoarsenDivMixed
                                                                  : hhg::kCoarsenDivFp64);
    lr.kp.hist_every = pl->hist_every;
    lr.kp.hist = pl->d_hist;
    lr.kp.hist_count = pl->d_hist_count;
    lr.kp.hist_cap = pl->hist_cap;
    lr.kp.energy_cut = pl->energy_cut;
    lr.kp.chan_stride = pl->part_len;
    lr.kp.kout = pl->d_kout;
    lr.out_mode = pl->out_mode;
    lr.degree = pl->degree;
    lr.precision = pl->opts.precision;
    lr.stepper = pl->opts.stepper;
    lr.proposer = pl->record ? 4 : kernel_proposer(pl->opts.proposer);
    lr.grid = pl->grid;
    lr.stream = s;
    lr.occupancy_out = nullptr;
    if (events) HHG_CUDA(ctx, cudaEventRecord(ctx->ev[0], s));
    hhg_status st = launch_variant(pl, lr);
    if (st != HHG_OK) return st;
    if (events) HHG_CUDA(ctx, cudaEventRecord(ctx->ev[1], s));
    // one reduction per output channel; k-resolved samples need none
    const int channels = pl->out_mode == 0 ? 1 : (pl->out_mode == 1 ? 2 : 0);
    for (int c = 0; c < channels; ++c) {
        hhg::reduce_partials_kernel<<<(unsigned)hhg::reduce_blocks(pl->j_len), hhg::kReduceThreads, 0, s>>>(
            pl->d_pulses, pl->n_pulses, pl->d_part + c * pl->part_len, pl->d_j + c * pl->j_len, pl->j_len);
        HHG_CUDA(ctx, cudaGetLastError());
    }
    if (events) {
        HHG_CUDA(ctx, cudaEventRecord(ctx->ev[2], s));
        pl->timed = true;
    }
    return HHG_OK;
}
}  // namespace

extern "C" {

hhg_status hhg_plan_execute_async(hhg_plan *pl, void *stream) {
    if (!pl) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    return enqueue_integration(pl, s, true);
}


hhg_status hhg_plan_fetch(hhg_plan *pl, double *j_out, hhg_stats *stats) {
    if (!pl) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    HHG_CUDA(ctx, cudaDeviceSynchronize());
    unsigned long long cnt[8];
    int status = 0;
    HHG_CUDA(ctx, cudaMemcpy(cnt, pl->d_counters, sizeof cnt, cudaMemcpyDeviceToHost));
    HHG_CUDA(ctx, cudaMemcpy(&status, pl->d_status, sizeof status, cudaMemcpyDeviceToHost));
    if (j_out) HHG_CUDA(ctx, cudaMemcpy(j_out, pl->d_j, pl->j_len * sizeof(double), cudaMemcpyDeviceToHost));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->k_points = pl->n_k;
        stats->trajectories = pl->n_k * pl->n_pulses;
        stats->attempted_steps = (int64_t)cnt[1];
        stats->rejected_steps = (int64_t)cnt[2];
        stats->failed_trajectories = (int64_t)(cnt[3] + cnt[4]);
        stats->poly_degree = pl->degree;
        stats->items = (int32_t)pl->n_items;
        if (pl->timed) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
            cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[2]);
            stats->kernel_ms = a;
            stats->total_ms = b;
        }
    }
    if (status == 2)
        return set_err(ctx, HHG_STEP_LIMIT,
                       "Max number of iterations exceeded (" + std::to_string(pl->opts.max_failed_steps) +
                           "). A new step size was not found.");
    if (status == 3) return set_err(ctx, HHG_NONFINITE, "non-finite Bloch vector");
    return HHG_OK;
}

hhg_status hhg_gpu_current_density(hhg_ctx *ctx, const hhg_system_desc *sys,
                                   const hhg_pulse_desc *pulses, int n_pulses,
                                   const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                                   double *j_out, hhg_stats *stats) {
    if (!ctx || !j_out) return set_err(ctx, HHG_BAD_CONFIG, "null context or output");
    if (!sys || !pulses || !grid || n_pulses < 1 || n_pulses > (1 << 20))
        return set_err(ctx, HHG_BAD_CONFIG, "null descriptor or bad pulse count");
    // repeated calls with the same descriptors reuse the plan (k table, pulse
    // staging, device buffers); the integration itself runs every call
    const std::string key = plan_key(sys, pulses, n_pulses, grid, opts);
    hhg_plan *pl = nullptr;
    auto &cache = ctx->plan_cache;
    for (size_t i = 0; i < cache.size(); ++i)
        if (cache[i].first == key) {
            pl = cache[i].second;
            std::rotate(cache.begin(), cache.begin() + i, cache.begin() + i + 1);
            break;
        }
    if (!pl) {
        hhg_status st = hhg_plan_create(ctx, sys, pulses, n_pulses, grid, opts, &pl);
        if (st != HHG_OK) return st;
        cache.insert(cache.begin(), {key, pl});
        while (cache.size() > kPlanCacheSize) {
            hhg_plan_destroy(cache.back().second);
            cache.pop_back();
        }
    }
    hhg_status st = hhg_plan_execute_async(pl, nullptr);
    if (st == HHG_OK) st = hhg_plan_fetch(pl, j_out, stats);
    return st;
}

}  // extern "C"

namespace {
// TrapezoidalFFT::compute of the n host samples j, zero-padded to n_in >= n
// values, through the context's buffers and cuFFT plans.
hhg_status trapezoidal_fft(hhg_ctx *ctx, const double *j, int n, int n_in, double delta_t,
                           double t_begin, double t_end, double *re_out, double *im_out,
                           double *freq_out) {
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n_fft = n_in / 2 + 1;
    cudaStream_t s = ctx->stream;
    if (ctx->x_cap < (size_t)n_in) {
        cudaFree(ctx->d_x);
        ctx->d_x = nullptr;
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_x, sizeof(double) * n_in));
        ctx->x_cap = n_in;
    }
    if (ctx->f_cap < (size_t)n_fft) {
        cudaFree(ctx->d_F);
        cudaFree(ctx->d_out);
        ctx->d_F = nullptr;
        ctx->d_out = nullptr;
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_F, sizeof(double2) * n_fft));
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_out, sizeof(double) * 3 * n_fft));
        ctx->f_cap = n_fft;
    }
    cufftHandle plan;
    auto it = ctx->fft_plans.find(n_in);
    if (it == ctx->fft_plans.end()) {
        if (cufftPlan1d(&plan, n_in, CUFFT_D2Z, 1) != CUFFT_SUCCESS)
            return set_err(ctx, HHG_CUDA_ERROR, "cufftPlan1d failed");
        ctx->fft_plans[n_in] = plan;
    } else {
        plan = it->second;
    }
    if (cufftSetStream(plan, s) != CUFFT_SUCCESS) return set_err(ctx, HHG_CUDA_ERROR, "cufftSetStream failed");
    // the host j goes into the tail of the padded buffer's scratch, then pad
    double *d_j = ctx->d_out;  // 3 n_fft >= n doubles of scratch
    HHG_CUDA(ctx, cudaMemcpyAsync(d_j, j, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    hhg::pad_kernel<<<(n_in + 255) / 256, 256, 0, s>>>(d_j, n, ctx->d_x, n_in);
    HHG_CUDA(ctx, cudaGetLastError());
    if (cufftExecD2Z(plan, ctx->d_x, (cufftDoubleComplex *)ctx->d_F) != CUFFT_SUCCESS)
        return set_err(ctx, HHG_CUDA_ERROR, "cufftExecD2Z failed");
    hhg::trapezoid_correct_kernel<<<(n_fft + 255) / 256, 256, 0, s>>>(
        ctx->d_F, n_fft, n_in, delta_t, t_begin, t_end, ctx->d_x, ctx->d_out,
        ctx->d_out + n_fft, ctx->d_out + 2 * n_fft);
    HHG_CUDA(ctx, cudaGetLastError());
    HHG_CUDA(ctx, cudaMemcpyAsync(re_out, ctx->d_out, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaMemcpyAsync(im_out, ctx->d_out + n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaMemcpyAsync(freq_out, ctx->d_out + 2 * n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaStreamSynchronize(s));
    return HHG_OK;
}
}  // namespace

extern "C" {

hhg_status hhg_gpu_spectrum(hhg_ctx *ctx, const double *j, int n_measurements, double t_begin,
                            double t_end, double *re_out, double *im_out, double *freq_out) {
    if (!ctx || !j || !re_out || !im_out || !freq_out || n_measurements < 1)
        return set_err(ctx, HHG_BAD_CONFIG, "bad spectrum arguments");
    if (!(t_end > t_begin)) return set_err(ctx, HHG_BAD_CONFIG, "empty time window");
    const int n = n_measurements + 1;
    const long long n_in_ll = 8LL * n;  // zero_padding (hhg.cpp:36)
    if (n_in_ll > (1LL << 30)) return set_err(ctx, HHG_BAD_CONFIG, "spectrum too long");
    return trapezoidal_fft(ctx, j, n, (int)n_in_ll, (t_end - t_begin) / n_measurements, t_begin,
                           t_end, re_out, im_out, freq_out);
}

hhg_status hhg_gpu_trapezoidal_fft(hhg_ctx *ctx, const double *input, int64_t n_input,
                                   double delta_t, double t_begin, double t_end, double *re_out,
                                   double *im_out, double *freq_out) {
    if (!ctx || !input || !re_out || !im_out || !freq_out || n_input < 2)
        return set_err(ctx, HHG_BAD_CONFIG, "bad spectrum arguments");
    if (n_input > (1LL << 30)) return set_err(ctx, HHG_BAD_CONFIG, "spectrum too long");
    if (!(delta_t > 0.0) || !std::isfinite(delta_t) || !std::isfinite(t_begin) || !std::isfinite(t_end))
        return set_err(ctx, HHG_BAD_CONFIG, "bad time step or window");
    return trapezoidal_fft(ctx, input, (int)n_input, (int)n_input, delta_t, t_begin, t_end, re_out,
                           im_out, freq_out);
}

namespace {
hhg_status get_fft_plan(hhg_ctx *ctx, int n_in, cufftHandle *out) {
    auto it = ctx->fft_plans.find(n_in);
    if (it != ctx->fft_plans.end()) {
        *out = it->second;
        return HHG_OK;
    }
    cufftHandle plan;
    if (cufftPlan1d(&plan, n_in, CUFFT_D2Z, 1) != CUFFT_SUCCESS)
        return set_err(ctx, HHG_CUDA_ERROR, "cufftPlan1d failed");
    ctx->fft_plans[n_in] = plan;
    *out = plan;
    return HHG_OK;
}

// Spectrum buffers and FFT plans (allocating: never inside a capture).
hhg_status prepare_spectrum(hhg_plan *pl) {
    hhg_ctx *ctx = pl->ctx;
    if (!pl->d_spec) {
        long long max_in = 0, off = 0;
        pl->spec_off.assign(pl->n_pulses + 1, 0);
        for (int p = 0; p < pl->n_pulses; ++p) {
            const long long n_in = 8LL * (pl->pulses[p].n_meas + 1);
            max_in = std::max(max_in, n_in);
            pl->spec_off[p] = off;
            off += n_in / 2 + 1;
        }
        pl->spec_off[pl->n_pulses] = off;
        pl->spec_len = off;
        HHG_CUDA(ctx, cudaMalloc(&pl->d_spec, sizeof(double) * 3 * off));
        HHG_CUDA(ctx, cudaMalloc(&pl->d_x, sizeof(double) * max_in));
        HHG_CUDA(ctx, cudaMalloc(&pl->d_F, sizeof(double2) * (max_in / 2 + 1)));
    }
    for (int p = 0; p < pl->n_pulses; ++p) {
        cufftHandle fp;
        const hhg_status st = get_fft_plan(ctx, 8 * (pl->pulses[p].n_meas + 1), &fp);
        if (st != HHG_OK) return st;
    }
    return HHG_OK;
}

// Zero-padding, FFT and trapezoid correction of every pulse's j on stream s.
hhg_status enqueue_spectrum(hhg_plan *pl, cudaStream_t s) {
    hhg_ctx *ctx = pl->ctx;
    for (int p = 0; p < pl->n_pulses; ++p) {
        const PulseDev &d = pl->pulses[p];
        const int n = d.n_meas + 1;
        const int n_in = 8 * n, n_fft = n_in / 2 + 1;
        cufftHandle fp;
        hhg_status st = get_fft_plan(ctx, n_in, &fp);
        if (st != HHG_OK) return st;
        if (cufftSetStream(fp, s) != CUFFT_SUCCESS) return set_err(ctx, HHG_CUDA_ERROR, "cufftSetStream failed");
        hhg::pad_kernel<<<(n_in + 255) / 256, 256, 0, s>>>(pl->d_j + d.j_off, n, pl->d_x, n_in);
        HHG_CUDA(ctx, cudaGetLastError());
        if (cufftExecD2Z(fp, pl->d_x, (cufftDoubleComplex *)pl->d_F) != CUFFT_SUCCESS)
            return set_err(ctx, HHG_CUDA_ERROR, "cufftExecD2Z failed");
        double *base = pl->d_spec + 3 * pl->spec_off[p];
        hhg::trapezoid_correct_kernel<<<(n_fft + 255) / 256, 256, 0, s>>>(
            pl->d_F, n_fft, n_in, d.measure_every, d.window_begin, pl->window_end[p], pl->d_x,
            base, base + n_fft, base + 2 * n_fft);
        HHG_CUDA(ctx, cudaGetLastError());
    }
    return HHG_OK;
}
}  // namespace

hhg_status hhg_plan_spectrum_async(hhg_plan *pl, void *stream) {
    if (!pl) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    const hhg_status st = prepare_spectrum(pl);
    if (st != HHG_OK) return st;
    return enqueue_spectrum(pl, s);
}


hhg_status hhg_plan_fetch_spectrum(hhg_plan *pl, int pulse, double *re_out, double *im_out,
                                   double *freq_out) {
    if (!pl || pulse < 0 || pulse >= pl->n_pulses || !pl->d_spec) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    HHG_CUDA(ctx, cudaDeviceSynchronize());
    const long long n_fft = pl->spec_off[pulse + 1] - pl->spec_off[pulse];
    const double *base = pl->d_spec + 3 * pl->spec_off[pulse];
    if (re_out) HHG_CUDA(ctx, cudaMemcpy(re_out, base, sizeof(double) * n_fft, cudaMemcpyDeviceToHost));
    if (im_out) HHG_CUDA(ctx, cudaMemcpy(im_out, base + n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost));
    if (freq_out) HHG_CUDA(ctx, cudaMemcpy(freq_out, base + 2 * n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost));
    return HHG_OK;
}

extern "C++" {
namespace {
// Best of 5 timed launches of an FMA-chain probe (after 2 warm-up launches).
template <typename T, typename K>
hhg_status measure_fma_peak(hhg_ctx *ctx, K kern, T a, T b, double *tflops) {
    if (!ctx || !tflops) return HHG_BAD_CONFIG;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    T *d_out = nullptr;
    HHG_CUDA(ctx, cudaMalloc(&d_out, sizeof(T)));
    const int threads = 256, blocks = ctx->sm_count * 8, iters = 4096;
    cudaStream_t s = ctx->stream;
    for (int w = 0; w < 2; ++w) kern<<<blocks, threads, 0, s>>>(d_out, iters, a, b);
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(ctx->ev[0], s);
        kern<<<blocks, threads, 0, s>>>(d_out, iters, a, b);
        cudaEventRecord(ctx->ev[1], s);
        cudaEventSynchronize(ctx->ev[1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        best = std::min(best, ms);
    }
    cudaError_t e = cudaGetLastError();
    cudaFree(d_out);
    if (e != cudaSuccess) return set_err(ctx, HHG_CUDA_ERROR, cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return HHG_OK;
}
}  // namespace
}  // extern "C++"

hhg_status hhg_measure_fp64_peak(hhg_ctx *ctx, double *tflops) {
    return measure_fma_peak<double>(ctx, hhg::fp64_fma_probe_kernel, 0.999999, 1e-7, tflops);
}

hhg_status hhg_measure_fp32_peak(hhg_ctx *ctx, double *tflops) {
    return measure_fma_peak<float>(ctx, hhg::fp32_fma_probe_kernel, 0.999999f, 1e-7f, tflops);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Per-pulse preparation for the allocation-free entry point (hhg_noalloc.cu).
// Same arithmetic as hhg_plan_create for one pulse; kept separate so the plan
// path is untouched.
// ---------------------------------------------------------------------------

namespace hhg_prep {

hhg_status prepare_pulse(const hhg_system_desc *sys, const hhg_pulse_desc *pulse, PulsePrep &out) {
    hhg_status st = check_system(nullptr, sys);
    if (st != HHG_OK) return st;
    if (!pulse) return HHG_BAD_CONFIG;
    if ((st = check_pulse(nullptr, *pulse)) != HHG_OK) return st;
    out.model = kernel_model(*sys);
    out.nf = model_nf(out.model);
    const double nny = 0.5 * kSqrt3;
    double proj[3] = {0, 0, 0};
    switch (hhg::base_model(out.model)) {
    case hhg::PIFLUX2D: proj[0] = sys->pol_x; proj[1] = sys->pol_y; break;
    case hhg::PIFLUX2D_SYM: proj[0] = sys->pol_x; break;
    case hhg::HONEYCOMB:
        proj[0] = 1.0 * sys->pol_x + 0.0 * sys->pol_y;
        proj[1] = -0.5 * sys->pol_x + nny * sys->pol_y;
        proj[2] = -0.5 * sys->pol_x - nny * sys->pol_y;
        break;
    case hhg::HONEYCOMB_X: proj[0] = sys->pol_x; proj[1] = -0.5 * sys->pol_x; break;
    case hhg::PIFLUX3D: proj[0] = 1.0; break;
    }
    const int d = choose_degree(*pulse, proj, out.nf);
    out.degree = d < 0 ? -1 : std::max(5, d);
    const hhg_pulse_desc &q = *pulse;
    if (q.kind == HHG_PULSE_SPLINE) return HHG_UNSUPPORTED;  // its coefficients would need device memory
    PulseDev &p = out.pulse;
    std::memset(&p, 0, sizeof p);
    const HostPulse hp(q);
    fill_pulse_dev(q, hp, p);
    const double es = q.energy_scale;
    switch (sys->kind) {
    case HHG_SYS_DIRAC2D: p.mp[0] = 2.0 * sys->velocity * es; p.mp[1] = 2.0 * sys->mass * es; break;
    case HHG_SYS_PIFLUX3D: p.mp[0] = 4.0 * sys->hopping * es; break;
    case HHG_SYS_PIFLUX2D: p.mp[0] = -4.0 * sys->hopping * es; break;
    case HHG_SYS_HONEYCOMB: p.mp[0] = 2.0 * sys->hopping * es; p.mp[1] = 2.0 * sys->mass * es; break;
    default: break;
    }
    p.mp[2] = sys->pol_x;
    p.mp[3] = sys->pol_y;
    set_relax_params(*sys, es, p.mp);
    for (int n = 0; n < 3; ++n) p.s[n] = proj[n];
    const double A0 = hp.value(0 * p.measure_every + p.window_begin);
    p.s0rec[0] = A0;
    if (out.nf == 1) p.s0rec[1] = A0;
    else if (hhg::base_model(out.model) == hhg::PIFLUX3D) {
        p.s0rec[1] = cos(A0);
        p.s0rec[2] = sin(A0);
    } else
        for (int n = 0; n < out.nf / 2; ++n) {
            p.s0rec[1 + 2 * n] = cos(proj[n] * A0);
            p.s0rec[2 + 2 * n] = sin(proj[n] * A0);
        }
    p.n_meas = q.n_measurements;
    out.tgrid.assign((size_t)q.n_measurements + 1, 0.0);
    double t_begin = p.window_begin, t_end = t_begin + p.measure_every;
    out.tgrid[0] = t_begin;
    for (int i = 1; i <= q.n_measurements; ++i) {
        out.tgrid[i] = t_end;
        t_begin = t_end;
        t_end += p.measure_every;
    }
    return HHG_OK;
}

}  // namespace hhg_prep

// ---------------------------------------------------------------------------
// Learned step-size proposer: collection and the training entry points
// ---------------------------------------------------------------------------
extern "C" {

hhg_status hhg_learned_collect(hhg_ctx *ctx, const hhg_system_desc *sys,
                               const hhg_pulse_desc *pulses, int n_pulses,
                               const hhg_grid_desc *grid, const hhg_solver_opts *opts,
                               int hist_every, float *records, int64_t cap, int64_t *n_records,
                               hhg_stats *stats) {
    if (!ctx) return HHG_BAD_CONFIG;
    if (hist_every < 1 || cap < 0 || (cap > 0 && !records) || cap > ((int64_t)1 << 31))
        return set_err(ctx, HHG_BAD_CONFIG, "hist_every >= 1, 0 <= cap <= 2^31, records for cap > 0");
    hhg_solver_opts o;
    hhg_default_solver_opts(&o);
    if (opts) o = *opts;
    o.stepper = HHG_STEPPER_RKF78;
    o.precision = HHG_PREC_FP64;
    o.proposer = HHG_PROPOSER_CARRY;
    o.mlp = nullptr;
    hhg_plan *pl = nullptr;
    hhg_status st = hhg_plan_create(ctx, sys, pulses, n_pulses, grid, &o, &pl);
    if (st != HHG_OK) return st;
    if (pl->degree == 0) {
        hhg_plan_destroy(pl);
        return set_err(ctx, HHG_UNSUPPORTED,
                       "spline pulse too steep for the staged interpolants: its exact evaluation "
                       "runs the Brillouin-zone current only, without history recording");
    }
    pl->record = true;
    pl->hist_every = hist_every;
    pl->hist_cap = cap;
    cudaError_t e;
    if ((e = cudaMalloc(&pl->d_hist, sizeof(float) * HHG_HIST_FIELDS * std::max<int64_t>(cap, 1))) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_hist_count, sizeof(unsigned long long))) != cudaSuccess) {
        hhg_plan_destroy(pl);
        return set_err(ctx, HHG_CUDA_ERROR, std::string("alloc history: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(pl->d_hist_count, 0, sizeof(unsigned long long), ctx->stream);
    st = hhg_plan_execute_async(pl, nullptr);
    if (st == HHG_OK) st = hhg_plan_fetch(pl, nullptr, stats);
    if (st == HHG_OK) {
        unsigned long long cnt = 0;
        if ((e = cudaMemcpy(&cnt, pl->d_hist_count, sizeof cnt, cudaMemcpyDeviceToHost)) != cudaSuccess) {
            hhg_plan_destroy(pl);
            return set_err(ctx, HHG_CUDA_ERROR, std::string("read history count: ") + cudaGetErrorString(e));
        }
        const int64_t n = std::min<int64_t>((int64_t)cnt, cap);
        if (n > 0 &&
            (e = cudaMemcpy(records, pl->d_hist, sizeof(float) * HHG_HIST_FIELDS * n, cudaMemcpyDeviceToHost)) !=
                cudaSuccess) {
            hhg_plan_destroy(pl);
            return set_err(ctx, HHG_CUDA_ERROR, std::string("read history: ") + cudaGetErrorString(e));
        }
        if (n_records) *n_records = n;
    }
    hhg_plan_destroy(pl);
    return st;
}

hhg_status hhg_mlp_train(hhg_ctx *ctx, const float *records, int64_t n_records,
                         const hhg_train_opts *opts, hhg_mlp *net, float *epoch_loss,
                         double *train_ms) {
    if (!ctx) return HHG_BAD_CONFIG;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    hhg_train_opts o;
    hhg_default_train_opts(&o);
    if (opts) o = *opts;
    std::string msg;
    const hhg_status st =
        hhg::mlp_train_impl(ctx->stream, records, n_records, o, net, epoch_loss, train_ms, &msg);
    return st == HHG_OK ? st : set_err(ctx, st, msg);
}

hhg_status hhg_mlp_gradients(hhg_ctx *ctx, const float *records, int64_t n_records,
                             const hhg_mlp *net, float *grad_out, float *loss_out) {
    if (!ctx) return HHG_BAD_CONFIG;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    std::string msg;
    const hhg_status st = hhg::mlp_gradients_impl(ctx->stream, records, n_records, net, grad_out, loss_out, &msg);
    return st == HHG_OK ? st : set_err(ctx, st, msg);
}

hhg_status hhg_mlp_predict(hhg_ctx *ctx, const float *records, int64_t n_records,
                           const hhg_mlp *net, int path, float *level_out) {
    if (!ctx) return HHG_BAD_CONFIG;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    std::string msg;
    const hhg_status st = hhg::mlp_predict_impl(ctx->stream, records, n_records, net, path, level_out, &msg);
    return st == HHG_OK ? st : set_err(ctx, st, msg);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// CUDA graph execution and the work-decomposition autotuner
// ---------------------------------------------------------------------------
namespace {
void drop_graph(hhg_plan *pl) {
    if (pl->gexec) cudaGraphExecDestroy(pl->gexec);
    pl->gexec = nullptr;
    pl->graph_spec = -1;
}

// k tiles of 32 per work item (tpi) and the persistent grid (ctas, 0 = all
// resident CTAs): re-derive the item list, the partial-row offsets and the
// device pulse table.
hhg_status retile(hhg_plan *pl, int tpi, long long ctas) {
    hhg_ctx *ctx = pl->ctx;
    const long long tiles = (pl->n_k + 31) / 32;
    tpi = (int)std::max(1LL, std::min<long long>(tpi, tiles));
    const int ipp = (int)((tiles + tpi - 1) / tpi);
    long long part_len = 0;
    for (int p = 0; p < pl->n_pulses; ++p) {
        PulseDev &d = pl->pulses[p];
        d.items = ipp;
        d.part_off = part_len;
        part_len += (long long)ipp * (d.n_meas + 1);
    }
    if (part_len > pl->part_cap) {
        cudaFree(pl->d_part);
        pl->d_part = nullptr;
        pl->part_cap = 0;
        HHG_CUDA(ctx, cudaMalloc(&pl->d_part, sizeof(double) * part_len));
        pl->part_cap = part_len;
    }
    pl->part_len = part_len;
    pl->tiles_per_item = tpi;
    pl->items_per_pulse = ipp;
    pl->n_items = (long long)ipp * pl->n_pulses;
    HHG_CUDA(ctx, cudaMemcpy(pl->d_pulses, pl->pulses.data(), sizeof(PulseDev) * pl->n_pulses,
                             cudaMemcpyHostToDevice));
    const long long max_ctas = (long long)pl->occupancy * ctx->sm_count;
    const long long need = (pl->n_items + hhg::kWarpsPerBlock - 1) / hhg::kWarpsPerBlock;
    const long long want = ctas > 0 ? std::min(ctas, max_ctas) : max_ctas;
    pl->grid = (int)std::max(1LL, std::min(want, need));
    drop_graph(pl);
    return HHG_OK;
}
}  // namespace

extern "C" {

hhg_status hhg_plan_execute_graph(hhg_plan *pl, void *stream, int with_spectrum) {
    if (!pl) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    with_spectrum = with_spectrum ? 1 : 0;
    if (!pl->gexec || pl->graph_spec != with_spectrum) {
        drop_graph(pl);
        if (with_spectrum) {
            const hhg_status st = prepare_spectrum(pl);
            if (st != HHG_OK) return st;
        }
        // capture on the context's own (non-blocking) stream; the graph is
        // launched on the caller's stream
        HHG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        HHG_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        hhg_status st = enqueue_integration(pl, ctx->stream, false);
        if (st == HHG_OK && with_spectrum) st = enqueue_spectrum(pl, ctx->stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (st != HHG_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess)
            return set_err(ctx, HHG_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
        const cudaError_t e2 = cudaGraphInstantiate(&pl->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) {
            pl->gexec = nullptr;
            return set_err(ctx, HHG_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(e2));
        }
        pl->graph_spec = with_spectrum;
    }
    // events recorded inside a captured graph do not time; bracket the launch
    HHG_CUDA(ctx, cudaEventRecord(ctx->ev[0], s));
    HHG_CUDA(ctx, cudaGraphLaunch(pl->gexec, s));
    HHG_CUDA(ctx, cudaEventRecord(ctx->ev[1], s));
    HHG_CUDA(ctx, cudaEventRecord(ctx->ev[2], s));
    pl->timed = true;
    return HHG_OK;
}

hhg_status hhg_plan_autotune(hhg_plan *pl, int reps, hhg_tune_report *report) {
    if (!pl) return HHG_BAD_CONFIG;
    hhg_ctx *ctx = pl->ctx;
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    reps = std::max(1, std::min(reps, 16));
    const long long tiles = (pl->n_k + 31) / 32;
    const long long resident = (long long)pl->occupancy * ctx->sm_count;
    std::vector<std::pair<int, long long>> cand;
    for (int tpi : {1, 2, 4, 8, 16}) {
        if (tpi > 1 && tpi > tiles) break;
        // the partial rows stay below 8 GB
        const double part_bytes = 8.0 * (double)((tiles + tpi - 1) / tpi) * (double)pl->j_len;
        if (part_bytes > 8e9) continue;
        for (long long ctas : {resident, resident / 2})
            if ((int)cand.size() < HHG_TUNE_MAX) cand.emplace_back(tpi, std::max(1LL, ctas));
    }
    if (cand.empty()) return set_err(ctx, HHG_UNSUPPORTED, "no tiling fits the partial-row budget");
    std::vector<double> ms(cand.size(), 1e300);
    std::vector<int> grids(cand.size(), 0);
    for (size_t c = 0; c < cand.size(); ++c) {
        hhg_status st = retile(pl, cand[c].first, cand[c].second);
        if (st != HHG_OK) return st;
        grids[c] = pl->grid;
        for (int r = 0; r <= reps; ++r) {  // first run untimed (warm-up)
            st = enqueue_integration(pl, ctx->stream, true);
            if (st != HHG_OK) return st;
            HHG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            float a = 0.f;
            HHG_CUDA(ctx, cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
            if (r > 0) ms[c] = std::min(ms[c], (double)a);
        }
    }
    size_t best = 0;
    for (size_t c = 1; c < cand.size(); ++c)
        if (ms[c] < ms[best]) best = c;
    hhg_status st = retile(pl, cand[best].first, cand[best].second);
    if (st != HHG_OK) return st;
    if (report) {
        std::memset(report, 0, sizeof *report);
        report->n_candidates = (int32_t)cand.size();
        report->best = (int32_t)best;
        for (size_t c = 0; c < cand.size(); ++c) {
            report->tile_k[c] = cand[c].first;
            report->grid[c] = grids[c];
            report->kernel_ms[c] = ms[c];
        }
    }
    return HHG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// k-resolved samples and the energy-split current (the reference's occupation
// tracking and split-current run modes)
// ---------------------------------------------------------------------------
namespace {
// A plan of one pulse switched to output mode `mode` (bz_integrate_kernel's
// OUT): buffers for the mode and the persistent grid of that kernel variant.
hhg_status output_plan(hhg_ctx *ctx, const hhg_system_desc *sys, const hhg_pulse_desc *pulse,
                       const hhg_grid_desc *grid, const hhg_solver_opts *opts, int mode,
                       hhg_plan **out) {
    *out = nullptr;
    if (!sys || !pulse || !grid) return set_err(ctx, HHG_BAD_CONFIG, "null descriptor");
    hhg_solver_opts o;
    hhg_default_solver_opts(&o);
    if (opts) o = *opts;
    if (mode == 4) {
        // per-trajectory weighted currents: the Dirac-3D kernels of its quadrature
        if (sys->kind != HHG_SYS_DIRAC3D)
            return set_err(ctx, HHG_UNSUPPORTED, "per-trajectory currents are Dirac-3D's");
        const bool relax = sys->inv_diag_relax > 0.0;
        if (o.precision != HHG_PREC_FP64 || o.proposer != HHG_PROPOSER_NONE ||
            !(o.stepper == HHG_STEPPER_RKF78 || (!relax && o.stepper == HHG_STEPPER_DIRAC_MAGNUS)))
            return set_err(ctx, HHG_UNSUPPORTED,
                           "per-trajectory currents run FP64 with the NONE proposer: the closed-form "
                           "Magnus step (coherent) or RKF78");
    } else {
        if (sys->kind != HHG_SYS_PIFLUX3D)
            return set_err(ctx, HHG_UNSUPPORTED, "k-resolved and split-current outputs are PiFlux-3D's");
        if (o.stepper != HHG_STEPPER_RKF78 || o.precision != HHG_PREC_FP64 ||
            (o.proposer != HHG_PROPOSER_NONE && o.proposer != HHG_PROPOSER_CARRY))
            return set_err(ctx, HHG_UNSUPPORTED,
                           "k-resolved and split-current outputs run FP64 RKF78 with the NONE or CARRY proposer");
    }
    hhg_plan *pl = nullptr;
    hhg_status st = plan_create_impl(ctx, sys, pulse, 1, grid, &o, &pl, false);  // k order kept
    if (st != HHG_OK) return st;
    if (pl->degree == 0) {
        hhg_plan_destroy(pl);
        return set_err(ctx, HHG_UNSUPPORTED,
                       "spline pulse too steep for the staged interpolants: its exact evaluation "
                       "runs the Brillouin-zone current only");
    }
    auto fail = [&](const char *what, cudaError_t e) {
        hhg_plan_destroy(pl);
        return set_err(ctx, HHG_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    pl->out_mode = mode;
    if (mode == 1) {  // a second channel of partial rows and of j
        cudaFree(pl->d_part);
        cudaFree(pl->d_j);
        pl->d_part = nullptr;
        pl->d_j = nullptr;
        if ((e = cudaMalloc(&pl->d_part, 2 * pl->part_len * sizeof(double))) != cudaSuccess) return fail("alloc partials", e);
        if ((e = cudaMalloc(&pl->d_j, 2 * pl->j_len * sizeof(double))) != cudaSuccess) return fail("alloc j", e);
    } else {
        const int width = mode == 2 ? 3 : (mode == 3 ? 2 : 1);
        pl->kout_len = (long long)(pulse->n_measurements + 1) * pl->n_k * width;
        if ((e = cudaMalloc(&pl->d_kout, pl->kout_len * sizeof(double))) != cudaSuccess)
            return fail("alloc k-resolved output", e);
    }
    int occ = 0;
    hhg::LaunchReq lr{};
    lr.degree = pl->degree;
    lr.precision = o.precision;
    lr.stepper = o.stepper;
    lr.proposer = kernel_proposer(o.proposer);
    lr.out_mode = mode;
    lr.grid = 0;
    lr.occupancy_out = &occ;
    if ((st = launch_variant(pl, lr)) != HHG_OK) {
        hhg_plan_destroy(pl);
        return st;
    }
    const long long need = (pl->n_items + hhg::kWarpsPerBlock - 1) / hhg::kWarpsPerBlock;
    pl->grid = (int)std::max(1LL, std::min((long long)std::max(occ, 1) * ctx->sm_count, need));
    *out = pl;
    return HHG_OK;
}
}  // namespace

extern "C" {

hhg_status hhg_gpu_k_resolved(hhg_ctx *ctx, const hhg_system_desc *sys, const hhg_pulse_desc *pulse,
                              const hhg_grid_desc *grid, const hhg_solver_opts *opts, int kind,
                              double *out, hhg_stats *stats) {
    if (!ctx || !out) return set_err(ctx, HHG_BAD_CONFIG, "null context or output");
    if (kind != HHG_KOUT_BLOCH && kind != HHG_KOUT_OCCUPATIONS && kind != HHG_KOUT_CURRENT)
        return set_err(ctx, HHG_BAD_CONFIG, "unknown k-resolved observable");
    hhg_plan *pl = nullptr;
    const int mode = kind == HHG_KOUT_BLOCH ? 2 : (kind == HHG_KOUT_OCCUPATIONS ? 3 : 4);
    hhg_status st = output_plan(ctx, sys, pulse, grid, opts, mode, &pl);
    if (st != HHG_OK) return st;
    st = hhg_plan_execute_async(pl, nullptr);
    if (st == HHG_OK) st = hhg_plan_fetch(pl, nullptr, stats);
    if (st == HHG_OK || st == HHG_STEP_LIMIT || st == HHG_NONFINITE) {
        const cudaError_t e = cudaMemcpy(out, pl->d_kout, pl->kout_len * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = set_err(ctx, HHG_CUDA_ERROR, std::string("fetch k-resolved output: ") + cudaGetErrorString(e));
    }
    hhg_plan_destroy(pl);
    return st;
}

hhg_status hhg_gpu_split_current(hhg_ctx *ctx, const hhg_system_desc *sys,
                                 const hhg_pulse_desc *pulse, const hhg_grid_desc *grid,
                                 const hhg_solver_opts *opts, double energy_cut, double *j_low,
                                 double *j_high, hhg_stats *stats) {
    if (!ctx || !j_low || !j_high) return set_err(ctx, HHG_BAD_CONFIG, "null context or output");
    if (!std::isfinite(energy_cut)) return set_err(ctx, HHG_BAD_CONFIG, "non-finite energy cut");
    hhg_plan *pl = nullptr;
    hhg_status st = output_plan(ctx, sys, pulse, grid, opts, 1, &pl);
    if (st != HHG_OK) return st;
    pl->energy_cut = energy_cut;
    st = hhg_plan_execute_async(pl, nullptr);
    if (st == HHG_OK) st = hhg_plan_fetch(pl, j_low, stats);
    if (st == HHG_OK || st == HHG_STEP_LIMIT || st == HHG_NONFINITE) {
        const cudaError_t e =
            cudaMemcpy(j_high, pl->d_j + pl->j_len, pl->j_len * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = set_err(ctx, HHG_CUDA_ERROR, std::string("fetch j: ") + cudaGetErrorString(e));
    }
    hhg_plan_destroy(pl);
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The Dirac-3D momentum quadrature: k_z slices x the adaptive kappa rule
// (DiracSystem::compute_current_density, DiracSystem.cpp:271-331)
// ---------------------------------------------------------------------------
namespace {

constexpr int kDefaultHalvings = 12;
constexpr int kKappaLookahead = 8;  // levels integrated ahead of the convergence test
// per-trajectory samples of one launch: up to 16 GiB, at most half the free
// device memory (plus what the context holds already), at least 1 GiB
constexpr double kKappaChunkBytes = 16.0 * (1 << 30);
constexpr double kKappaChunkMinBytes = 1.0 * (1 << 30);

struct KappaSplit {
    int slice;     // index of the k_z slice
    double a, H;   // start and length of the split
    int level;     // halvings of the estimate held on the device
    bool done;
};


hhg_status dirac_quadrature(hhg_ctx *ctx, const hhg_system_desc *sys, const hhg_pulse_desc *pulse,
                            const hhg_kappa_quad *q, const hhg_solver_opts *opts, double *j_out,
                            hhg_kappa_stats *qs, hhg_stats *stats) {
    if (!sys || !pulse || !q) return set_err(ctx, HHG_BAD_CONFIG, "null descriptor");
    if (sys->kind != HHG_SYS_DIRAC3D)
        return set_err(ctx, HHG_UNSUPPORTED, "the kappa quadrature is the Dirac-3D system's");
    if (q->n_z < 3 || q->n_z > (1 << 16))
        return set_err(ctx, HHG_BAD_CONFIG, "n_z out of range (3 .. 65536)");
    if (q->n_kappa < 1 || q->n_kappa > (1 << 20) || q->n_splits < 1 || q->n_splits > (1 << 20))
        return set_err(ctx, HHG_BAD_CONFIG, "n_kappa and n_splits must be in 1 .. 2^20");
    const int max_h = q->max_halvings > 0 ? q->max_halvings : kDefaultHalvings;
    if (q->max_halvings < 0 || max_h > 30 || ((long long)q->n_kappa << max_h) > (1LL << 26))
        return set_err(ctx, HHG_BAD_CONFIG, "max_halvings out of range (n_kappa 2^max_halvings <= 2^26)");
    if (!(q->threshold > 0.0) || !std::isfinite(q->threshold) || !(q->max_k > 0.0) ||
        !std::isfinite(q->max_k))
        return set_err(ctx, HHG_BAD_CONFIG, "threshold and max_k must be finite and > 0");
    hhg_solver_opts o;
    hhg_default_solver_opts(&o);
    if (opts) o = *opts;
    if ((o.stepper != HHG_STEPPER_DIRAC_MAGNUS && o.stepper != HHG_STEPPER_RKF78) ||
        o.precision != HHG_PREC_FP64 || o.proposer != HHG_PROPOSER_NONE)
        return set_err(ctx, HHG_UNSUPPORTED,
                       "the Dirac quadrature runs the closed-form Magnus step or FP64 RKF78 with "
                       "the reference schedule (proposer NONE)");
    if (pulse->n_measurements < 1 || pulse->n_measurements > (1 << 24))
        return set_err(ctx, HHG_BAD_CONFIG, "n_measurements out of range");
    const int n_samples = pulse->n_measurements + 1;

    // k_z slices (DiracSystem.cpp:283, 296-299) and their splits
    const int n_z = q->n_z;
    const double dz = 2 * q->max_k / n_z;
    std::vector<double> kz;
    // one rank's block of the z loop (DiracSystem.cpp:288-295), or all of it
    if (q->z_count < 0 || (q->z_count > 0 && (q->z_first < 1 || q->z_first > n_z - 1 ||
                                              q->z_count > n_z - q->z_first)))
        return set_err(ctx, HHG_BAD_CONFIG, "slice range outside z = 1 .. n_z - 1");
    const int z_lo = q->z_count > 0 ? q->z_first : 1;
    const int z_hi = q->z_count > 0 ? q->z_first + q->z_count : n_z;
    for (int z = z_lo; z < z_hi; ++z)
        if (z != n_z / 2) kz.push_back((z - n_z / 2) * dz);
    const int n_slices = (int)kz.size();
    if (n_slices == 0) {
        // a block holding only the weight-0 slice z = n_z / 2
        std::fill(j_out, j_out + pulse->n_measurements + 1, 0.0);
        if (qs) *qs = hhg_kappa_stats{};
        if (stats) *stats = hhg_stats{};
        return HHG_OK;
    }
    const long long n_total = (long long)n_slices * q->n_splits;
    if (n_total > (1LL << 28)) return set_err(ctx, HHG_BAD_CONFIG, "too many splits");
    std::vector<KappaSplit> sp((size_t)n_total);
    for (int z = 0; z < n_slices; ++z) {
        // kappa_integration_upper_limit (DiracSystem.cpp:257-261)
        const double kmax = sqrt(q->max_k * q->max_k - kz[z] * kz[z]);
        const double H = kmax / q->n_splits;
        for (int s = 0; s < q->n_splits; ++s) sp[(size_t)z * q->n_splits + s] = {z, s * H, H, 0, false};
    }

    // rows per launch: a whole round when its per-trajectory samples fit in
    // the budget, else chunks of whole splits (a split's nodes always fit)
    // (the first round holds a split's n_kappa + 1 trapezoid nodes and its
    // n_kappa first midpoints)
    const long long biggest = std::max<long long>(2LL * q->n_kappa + 1, (long long)q->n_kappa << (max_h - 1));
    size_t free_b = 0, total_b = 0;
    HHG_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b));
    const double held = 8.0 * (double)ctx->kappa_cap * n_samples;
    const double chunk = std::min(kKappaChunkBytes, std::max(kKappaChunkMinBytes, 0.5 * ((double)free_b + held)));
    const long long budget = (long long)(chunk / (8.0 * n_samples));
    const long long limit = std::max(biggest, std::max(budget, 32LL));

    // the plan: pulse staging and launch state, built on one placeholder row
    // (the k table and the per-trajectory buffer are replaced by
    // capacity-sized ones); kept in the context for the next call with the
    // same system, pulse and options
    static const double kPlaceholderRow[8] = {1.0, 1.0, 1.4142135623730951, 0.0, 0.0, 0.0, -1.0, 0.0};
    hhg_grid_desc g{};
    g.kind = HHG_GRID_EXPLICIT;
    g.rows = kPlaceholderRow;
    g.n_rows = 1;
    hhg_status st = HHG_OK;
    const std::string key = plan_key(sys, pulse, 1, &g, &o);
    if (!ctx->kappa_plan || ctx->kappa_key != key) {
        if (ctx->kappa_plan) hhg_plan_destroy(ctx->kappa_plan);
        ctx->kappa_plan = nullptr;
        ctx->kappa_key.clear();
        ctx->kappa_cap = 0;
        hhg_plan *np = nullptr;
        if ((st = hhg_plan_create(ctx, sys, pulse, 1, &g, &o, &np)) != HHG_OK) return st;
        if (np->degree == 0) {
            hhg_plan_destroy(np);
            return set_err(ctx, HHG_UNSUPPORTED,
                           "spline pulse too steep for the staged interpolants: its exact "
                           "evaluation runs the Brillouin-zone current only");
        }
        np->out_mode = 4;
        int occ = 0;
        hhg::LaunchReq lr{};
        lr.degree = np->degree;
        lr.precision = o.precision;
        lr.stepper = o.stepper;
        lr.proposer = 0;
        lr.out_mode = 4;
        lr.grid = 0;
        lr.occupancy_out = &occ;
        if ((st = launch_variant(np, lr)) != HHG_OK) {
            hhg_plan_destroy(np);
            return st;
        }
        ctx->kappa_plan = np;
        ctx->kappa_key = key;
        ctx->kappa_occ = std::max(occ, 1);
    }
    hhg_plan *pl = ctx->kappa_plan;
    const int occ = ctx->kappa_occ;
    long long &cap = ctx->kappa_cap;  // rows the k table and the sample buffer hold
    cudaStream_t s = ctx->stream;
    auto grow = [&](hhg_ctx::Grow &b, size_t bytes) -> cudaError_t {
        if (bytes <= b.bytes) return cudaSuccess;
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        const cudaError_t e = cudaMalloc(&b.p, bytes);
        if (e == cudaSuccess) b.bytes = bytes;
        return e;
    };
    // items per launch <= rows per launch (<= the row capacity, which an
    // earlier call may have grown beyond this call's limit), and <= splits x
    // levels per launch
    const size_t meta =
        (size_t)std::min<long long>((kKappaLookahead + 2) * n_total, std::max(limit, cap));
    HHG_CUDA(ctx, grow(ctx->kappa_T, (size_t)n_total * n_samples * sizeof(double)));
    HHG_CUDA(ctx, grow(ctx->kappa_items, meta * sizeof(hhg::KappaItem)));
    HHG_CUDA(ctx, grow(ctx->kappa_change, meta * sizeof(double)));
    HHG_CUDA(ctx, grow(ctx->kappa_j, (size_t)n_samples * sizeof(double)));
    HHG_CUDA(ctx, grow(ctx->kappa_slice, (size_t)n_slices * n_samples * sizeof(double)));
    double *dT = static_cast<double *>(ctx->kappa_T.p);
    hhg::KappaItem *ditems = static_cast<hhg::KappaItem *>(ctx->kappa_items.p);
    double *dchange = static_cast<double *>(ctx->kappa_change.p);
    double *dj = static_cast<double *>(ctx->kappa_j.p);
    double *dslice = static_cast<double *>(ctx->kappa_slice.p);
    HHG_CUDA(ctx, cudaMemsetAsync(dT, 0, (size_t)n_total * n_samples * sizeof(double), s));

    hhg_kappa_stats qsum{};
    qsum.splits = (int32_t)n_total;
    hhg_stats ssum{};
    hhg_status worst = HHG_OK;
    std::vector<long long> active((size_t)n_total);
    for (long long i = 0; i < n_total; ++i) active[(size_t)i] = i;
    std::vector<hhg::KappaItem> items;
    std::vector<double> change;
    // the item of split `id` at `level`: its nodes' rows start at row0
    auto make_item = [&](long long id, int level, long long row0) {
        const KappaSplit &x = sp[(size_t)id];
        hhg::KappaItem it{};
        it.k_z = kz[x.slice];
        it.a = x.a;
        it.panels = (long long)q->n_kappa << level;
        it.h = x.H / (double)it.panels;
        it.level = level;
        it.split = (int)id;
        it.row0 = row0;
        if (level == 0) {
            // kappa = 0 (the first node of a slice) is left out
            it.first = ref_is_zero(x.a) ? 1 : 0;
            it.stride = 1;
            it.n = q->n_kappa + 1 - it.first;
        } else {
            it.first = 1;
            it.stride = 2;
            it.n = (int)((long long)q->n_kappa << (level - 1));
        }
        return it;
    };
    // lookahead: a launch of a quarter of the resident lanes or fewer is
    // latency-bound (each trajectory is a serial chain over all intervals;
    // measured: such a launch takes as long as one trajectory alone), so
    // further levels of the same splits ride along while the launch stays that
    // small; the estimates still take the levels one by one with the
    // convergence test in between, and rows of levels a split never reaches
    // are discarded
    const long long resident = (long long)occ * ctx->sm_count * hhg::kBlockThreads / 4;
    std::vector<std::vector<hhg::KappaItem>> by_level;
    std::vector<hhg::KappaItem> todo;
    while (!active.empty()) {
        const int L = sp[(size_t)active[0]].level;  // every active split is at L
        auto level_nodes = [&](int l) {
            return l == 0 ? (long long)q->n_kappa + 1 : (long long)q->n_kappa << (l - 1);
        };
        // the first trapezoid and the first halving always go together
        int last = (L == 0) ? 1 : L;
        long long per_split = 0;
        for (int l = L; l <= last; ++l) per_split += level_nodes(l);
        while (last < max_h && last - L < kKappaLookahead && per_split + level_nodes(last + 1) <= limit &&
               (long long)active.size() * (per_split + level_nodes(last + 1)) <= resident) {
            ++last;
            per_split += level_nodes(last);
        }
        const int n_lv = last - L + 1;
        const long long round_rows = (long long)active.size() * per_split;
        const long long want = std::min(limit, round_rows);
        if (want > cap) {
            // grow the k table and the per-trajectory sample buffer
            cap = std::min(limit, std::max(want, 2 * cap));
            if (pl->ktab_owner) pl->ktab_owner.reset();
            else HHG_CUDA(ctx, cudaFree(pl->d_ktab));
            HHG_CUDA(ctx, cudaFree(pl->d_kout));
            pl->d_ktab = nullptr;
            pl->d_kout = nullptr;
            HHG_CUDA(ctx, cudaMalloc(&pl->d_ktab, (size_t)cap * 8 * sizeof(double)));
            HHG_CUDA(ctx, cudaMalloc(&pl->d_kout, (size_t)cap * n_samples * sizeof(double)));
            pl->kout_len = cap * n_samples;
        }
        size_t next = 0;
        while (next < active.size()) {
            // one launch: as many active splits as fit in `cap` rows, each with
            // its levels L..last; items level-major, rows in item order, built
            // on the device
            by_level.assign((size_t)n_lv, {});
            long long n_rows = 0;
            const size_t first = next;
            while (next < active.size()) {
                const long long id = active[next];
                if (next > first && n_rows + per_split > cap) break;
                for (int l = L; l <= last; ++l) by_level[(size_t)(l - L)].push_back(make_item(id, l, 0));
                n_rows += per_split;
                ++next;
            }
            items.clear();
            for (auto &v : by_level) items.insert(items.end(), v.begin(), v.end());
            n_rows = 0;
            for (hhg::KappaItem &it : items) {
                it.row0 = n_rows;
                n_rows += it.n;
            }
            {
                size_t k = 0;  // the row offsets back into the per-level lists
                for (auto &v : by_level)
                    for (hhg::KappaItem &it : v) it.row0 = items[k++].row0;
            }
            const int nb = (int)items.size();
            HHG_CUDA(ctx, cudaMemcpyAsync(ditems, items.data(), nb * sizeof(hhg::KappaItem),
                                          cudaMemcpyHostToDevice, s));
            if (n_rows > 0) {
                const long long blocks = std::min<long long>((n_rows + 255) / 256, 65536);
                hhg::kappa_rows_kernel<<<(unsigned)blocks, 256, 0, s>>>(
                    ditems, nb, n_rows, sys->beta, sys->fermi_energy, pl->d_ktab);
                HHG_CUDA(ctx, cudaGetLastError());
                pl->n_k = n_rows;
                pl->tiles_per_item = 1;
                pl->items_per_pulse = (int)((n_rows + 31) / 32);
                pl->n_items = pl->items_per_pulse;
                const long long need = (pl->n_items + hhg::kWarpsPerBlock - 1) / hhg::kWarpsPerBlock;
                pl->grid = (int)std::max(1LL, std::min((long long)std::max(occ, 1) * ctx->sm_count, need));
                if ((st = enqueue_integration(pl, s, true)) != HHG_OK) return st;
                hhg_stats sc{};
                st = hhg_plan_fetch(pl, nullptr, &sc);
                if (st == HHG_CUDA_ERROR || st == HHG_BAD_CONFIG) return st;
                if (st != HHG_OK && worst == HHG_OK) worst = st;
                ssum.k_points += sc.k_points;
                ssum.trajectories += sc.trajectories;
                ssum.attempted_steps += sc.attempted_steps;
                ssum.rejected_steps += sc.rejected_steps;
                ssum.failed_trajectories += sc.failed_trajectories;
                ssum.poly_degree = sc.poly_degree;
                ssum.items += sc.items;
                ssum.kernel_ms += sc.kernel_ms;
                ssum.total_ms += sc.total_ms;
                ++qsum.launches;
            }
            long long used = 0;
            for (int lv = 0; lv < n_lv; ++lv) {
                // the level's items of the splits still refining
                todo.clear();
                for (const hhg::KappaItem &it : by_level[(size_t)lv])
                    if (!sp[(size_t)it.split].done) todo.push_back(it);
                if (todo.empty()) break;
                const int nt = (int)todo.size();
                HHG_CUDA(ctx, cudaMemcpyAsync(ditems, todo.data(), nt * sizeof(hhg::KappaItem),
                                              cudaMemcpyHostToDevice, s));
                hhg::kappa_round_kernel<<<nt, hhg::kKappaThreads, 0, s>>>(
                    pl->d_kout, std::max(n_rows, 1LL), n_samples, ditems, dT, dchange);
                HHG_CUDA(ctx, cudaGetLastError());
                // the context stream does not synchronise with the legacy
                // stream: copies are ordered on it
                change.resize(nt);
                HHG_CUDA(ctx, cudaMemcpyAsync(change.data(), dchange, nt * sizeof(double),
                                              cudaMemcpyDeviceToHost, s));
                HHG_CUDA(ctx, cudaStreamSynchronize(s));
                // convergence: the change of a halving below the threshold
                for (int b = 0; b < nt; ++b) {
                    KappaSplit &x = sp[(size_t)todo[b].split];
                    used += todo[b].n;
                    x.level = todo[b].level;
                    qsum.max_level = std::max(qsum.max_level, x.level);
                    if (x.level > 0 && change[b] < q->threshold) {
                        x.done = true;
                    } else if (x.level >= max_h || std::isnan(change[b])) {
                        x.done = true;
                        ++qsum.unconverged;
                    } else {
                        ++x.level;
                    }
                }
            }
            qsum.trajectories += used;
            qsum.speculative += n_rows - used;
        }
        std::vector<long long> still;
        for (long long i : active)
            if (!sp[(size_t)i].done) still.push_back(i);
        active.swap(still);
    }
    const int threads = 256;
    const unsigned sblocks = (unsigned)((n_samples + threads - 1) / threads);
    hhg::kappa_slice_kernel<<<dim3(sblocks, (unsigned)n_slices), threads, 0, s>>>(
        dT, q->n_splits, n_samples, dslice);
    HHG_CUDA(ctx, cudaGetLastError());
    hhg::kappa_sum_kernel<<<sblocks, threads, 0, s>>>(dslice, n_slices, n_samples, dz, dj);
    HHG_CUDA(ctx, cudaGetLastError());
    HHG_CUDA(ctx, cudaMemcpyAsync(j_out, dj, (size_t)n_samples * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaStreamSynchronize(s));
    qsum.rounds = qsum.max_level + 1;  // levels evaluated, the first trapezoids included
    if (qs) *qs = qsum;
    if (stats) *stats = ssum;
    return worst;
}
}  // namespace

extern "C" {

hhg_status hhg_gpu_dirac_current_density(hhg_ctx *ctx, const hhg_system_desc *sys,
                                         const hhg_pulse_desc *pulse, const hhg_kappa_quad *quad,
                                         const hhg_solver_opts *opts, double *j_out,
                                         hhg_kappa_stats *qstats, hhg_stats *stats) {
    if (!ctx || !j_out) return set_err(ctx, HHG_BAD_CONFIG, "null context or output");
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    return dirac_quadrature(ctx, sys, pulse, quad, opts, j_out, qstats, stats);
}

}  // extern "C"

extern "C" {

hhg_status hhg_gpu_spectrum_welch(hhg_ctx *ctx, const double *j, int n_measurements, double t_begin,
                                  double t_end, double *re_out, double *im_out, double *freq_out) {
    if (!ctx || !j || !re_out || !im_out || !freq_out || n_measurements < 2)
        return set_err(ctx, HHG_BAD_CONFIG, "bad spectrum arguments");
    if (!(t_end > t_begin)) return set_err(ctx, HHG_BAD_CONFIG, "empty time window");
    if (n_measurements > (1 << 28)) return set_err(ctx, HHG_BAD_CONFIG, "spectrum too long");
    HHG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = n_measurements, n_fft = n / 2 + 1;
    cudaStream_t s = ctx->stream;
    if (ctx->x_cap < (size_t)(2 * n)) {
        cudaFree(ctx->d_x);
        ctx->d_x = nullptr;
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_x, sizeof(double) * 2 * n));
        ctx->x_cap = 2 * n;
    }
    if (ctx->f_cap < (size_t)n_fft) {
        cudaFree(ctx->d_F);
        cudaFree(ctx->d_out);
        ctx->d_F = nullptr;
        ctx->d_out = nullptr;
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_F, sizeof(double2) * n_fft));
        HHG_CUDA(ctx, cudaMalloc(&ctx->d_out, sizeof(double) * 3 * n_fft));
        ctx->f_cap = n_fft;
    }
    cufftHandle plan;
    hhg_status st = get_fft_plan(ctx, n, &plan);
    if (st != HHG_OK) return st;
    if (cufftSetStream(plan, s) != CUFFT_SUCCESS) return set_err(ctx, HHG_CUDA_ERROR, "cufftSetStream failed");
    // the first n samples (the reference's N-point FFT reads N of its N + 1)
    double *d_j = ctx->d_x + n;
    HHG_CUDA(ctx, cudaMemcpyAsync(d_j, j, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    hhg::welch_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_j, n, ctx->d_x);
    HHG_CUDA(ctx, cudaGetLastError());
    if (cufftExecD2Z(plan, ctx->d_x, (cufftDoubleComplex *)ctx->d_F) != CUFFT_SUCCESS)
        return set_err(ctx, HHG_CUDA_ERROR, "cufftExecD2Z failed");
    hhg::split_spectrum_kernel<<<(n_fft + 255) / 256, 256, 0, s>>>(
        ctx->d_F, n_fft, (t_end - t_begin) / n_measurements, ctx->d_out, ctx->d_out + n_fft,
        ctx->d_out + 2 * n_fft);
    HHG_CUDA(ctx, cudaGetLastError());
    HHG_CUDA(ctx, cudaMemcpyAsync(re_out, ctx->d_out, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaMemcpyAsync(im_out, ctx->d_out + n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaMemcpyAsync(freq_out, ctx->d_out + 2 * n_fft, sizeof(double) * n_fft, cudaMemcpyDeviceToHost, s));
    HHG_CUDA(ctx, cudaStreamSynchronize(s));
    return HHG_OK;
}

hhg_status hhg_pulse_values(const hhg_pulse_desc *pulse, const double *t, int64_t n, double *A) {
    if (!pulse || (n > 0 && (!t || !A)) || n < 0) return HHG_BAD_CONFIG;
    const hhg_status st = check_pulse(nullptr, *pulse);
    if (st != HHG_OK) return st;
    const HostPulse hp(*pulse);
    for (int64_t i = 0; i < n; ++i) A[i] = hp.value(t[i]);
    return HHG_OK;
}

}  // extern "C"
