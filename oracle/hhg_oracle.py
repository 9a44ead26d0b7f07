"""CPU oracle bindings and the reference's Fourier tail, restated.

TEST INFRASTRUCTURE ONLY.  The pytest suite, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this module as the checker; the
product package never does.

* ``libhhg_oracle.so`` (built from ``hhg_oracle.c`` by ``oracle/Makefile``)
  holds the FP64 restatement of the per-k Bloch integration and BZ sums.
* ``trapezoidal_fft`` restates ``TrapezoidalFFT::compute``
  (sources/HHG/Fourier/TrapezoidalFFT.cpp:11-49) with the x8 zero padding of
  sources/hhg.cpp:36,280-282, using numpy's r2c FFT in place of FFTW.

Parity status: unpinned at the Boost.Odeint boundary (see hhg_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

DIRAC2D, PIFLUX2D, PIFLUX3D, HONEYCOMB, DIRAC3D = 0, 1, 2, 3, 4
KROW = 8


class OrcModel(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("hopping", ctypes.c_double),
                ("velocity", ctypes.c_double), ("mass", ctypes.c_double),
                ("pol_x", ctypes.c_double), ("pol_y", ctypes.c_double),
                ("beta", ctypes.c_double), ("fermi_energy", ctypes.c_double),
                ("inv_diag_relax", ctypes.c_double), ("inv_offdiag_relax", ctypes.c_double)]


class OrcPulse(ctypes.Structure):
    _fields_ = [("amplitude", ctypes.c_double), ("t_begin", ctypes.c_double),
                ("t_end", ctypes.c_double), ("inv_n_cycles", ctypes.c_double),
                ("phase", ctypes.c_double), ("kind", ctypes.c_int),
                ("gauss_center", ctypes.c_double), ("gauss_sigma", ctypes.c_double),
                ("spline_y", ctypes.POINTER(ctypes.c_double)),
                ("spline_m", ctypes.POINTER(ctypes.c_double)), ("spline_n", ctypes.c_int),
                ("spline_h", ctypes.c_double)]


class OrcTimeConfig(ctypes.Structure):
    _fields_ = [("t_begin", ctypes.c_double), ("t_end", ctypes.c_double),
                ("n_measurements", ctypes.c_int), ("n_subdivisions", ctypes.c_int)]


class OrcSolver(ctypes.Structure):
    _fields_ = [("abs_tol", ctypes.c_double), ("rel_tol", ctypes.c_double),
                ("max_failed", ctypes.c_int), ("stepper", ctypes.c_int),
                ("magnus_substeps", ctypes.c_int)]


class OrcStats(ctypes.Structure):
    _fields_ = [("attempted", ctypes.c_uint64), ("accepted", ctypes.c_uint64),
                ("rejected", ctypes.c_uint64), ("failed_k", ctypes.c_uint64)]


_LIBS: dict[str, ctypes.CDLL] = {}
_D = ctypes.POINTER(ctypes.c_double)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast: bool = False) -> ctypes.CDLL:
    name = "libhhg_oracle_fast.so" if fast else "libhhg_oracle.so"
    if name not in _LIBS:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_laser.restype = ctypes.c_double
        L.orc_raw_laser.restype = ctypes.c_double
        L.orc_vertex.restype = ctypes.c_double
        for fn in ("orc_grid_tensor", "orc_grid_rhombic", "orc_grid_piflux3d_ref",
                   "orc_grid_honeycomb_hex_ref", "orc_evolve_k", "orc_current_density",
                   "orc_step_history", "orc_dirac3d_sigma_k"):
            getattr(L, fn).restype = ctypes.c_int
        L.orc_grid_tensor.argtypes = [ctypes.POINTER(OrcModel), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _D]
        _LIBS[name] = L
    return _LIBS[name]


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


@dataclass
class Pulse:
    """CosineLaser (sources/HHG/Laser/CosineLaser.cpp) plus a carrier phase."""
    amplitude: float
    n_cycles: float
    t_begin: float = 0.0
    phase: float = 0.0

    @property
    def t_end(self) -> float:
        return self.t_begin + 2 * np.pi * self.n_cycles

    def c(self) -> OrcPulse:
        return OrcPulse(self.amplitude, self.t_begin, self.t_end, 1.0 / self.n_cycles, self.phase)


PULSE_CONTINUOUS, PULSE_GAUSS, PULSE_SPLINE = 1, 2, 3


@dataclass
class ContinuousPulse:
    """ContinuousLaser (ContinuousLaser.cpp): envelope 1."""
    amplitude: float
    phase: float = 0.0
    t_begin: float = 0.0

    def c(self) -> OrcPulse:
        p = OrcPulse(self.amplitude, -np.inf, np.inf, 0.0, self.phase)
        p.kind = PULSE_CONTINUOUS
        return p


@dataclass
class GaussPulse:
    """GaussLaser (GaussLaser.cpp): centre t_begin + 3 pi n_cycles, sigma =
    pi n_cycles / sqrt(2 ln 20)."""
    amplitude: float
    n_cycles: float
    t_begin: float = 0.0
    phase: float = 0.0

    def c(self) -> OrcPulse:
        p = OrcPulse(self.amplitude, self.t_begin, self.t_begin + 6 * np.pi * self.n_cycles, 0.0,
                     self.phase)
        p.kind = PULSE_GAUSS
        p.gauss_center = self.t_begin + 0.5 * (2.0 * np.pi * 3.0 * self.n_cycles)
        p.gauss_sigma = np.pi * self.n_cycles / np.sqrt(2.0 * np.log(1.0 / 0.05))
        return p


class SplinePulse:
    """A = amplitude * s(t) for t <= cut, 0 after: the clamped cubic spline
    through samples at t_begin + k dt (orc_spline_moments)."""

    def __init__(self, samples, t_begin, dt, cut=None, deriv=(np.nan, np.nan), amplitude=1.0):
        self.y = np.ascontiguousarray(samples, dtype=np.float64)
        self.m = np.zeros_like(self.y)
        lib().orc_spline_moments(_p(self.y), ctypes.c_int(self.y.size), ctypes.c_double(dt),
                                 ctypes.c_double(deriv[0]), ctypes.c_double(deriv[1]), _p(self.m))
        self.t_begin, self.dt, self.amplitude = t_begin, dt, amplitude
        self.cut = t_begin + (self.y.size - 1) * dt if cut is None else cut

    def c(self) -> OrcPulse:
        p = OrcPulse(self.amplitude, self.t_begin, self.cut, 0.0, 0.0)
        p.kind = PULSE_SPLINE
        p.spline_y, p.spline_m = _p(self.y), _p(self.m)
        p.spline_n, p.spline_h = self.y.size, self.dt
        return p


def model(kind: int, hopping=0.0, velocity=0.0, mass=0.0, pol=(1.0, 0.0), *, beta=0.0,
          fermi_energy=0.0, inv_diag_relax=0.0, inv_offdiag_relax=0.0) -> OrcModel:
    return OrcModel(kind, hopping, velocity, mass, pol[0], pol[1], beta, fermi_energy,
                    inv_diag_relax, inv_offdiag_relax)


def solver(abs_tol=1e-12, rel_tol=1e-8, stepper=0, magnus_substeps=1) -> OrcSolver:
    return OrcSolver(abs_tol, rel_tol, 500, stepper, magnus_substeps)


def time_config(t_begin, t_end, n, n_sub=50) -> OrcTimeConfig:
    return OrcTimeConfig(t_begin, t_end, n, n_sub)


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(ctypes.c_int(n), _p(x), _p(w))
    return x, w


def laser(p: Pulse, t) -> np.ndarray:
    pc = p.c()
    return np.array([lib().orc_laser(ctypes.byref(pc), ctypes.c_double(float(v)))
                     for v in np.atleast_1d(t)])


def experimental_laser(e_a, e_b, dt_ps: float, pe_laser: float, e0: float, lattice: float,
                       shift_ps: float = 0.0, active: str = "both", hbar: float = 6.582119569509065698e-13,
                       n_extra: int = 16, begin_zero: int = 8, zero_buff: int = 8):
    """ExperimentalLaser (sources/HHG/Laser/ExperimentalLaser.cpp:8-108)
    restated for a caller's measured field: returns (SplinePulse of A(t),
    t_end).

    vector_potential (:30-62): begin_zero zeros, then A_i = A_(i-1) - E_i dt
    (dt in ps), then A continued over n_extra - 1 steps by the quartic
    p(t) = A + P t + Q t^2 + c t^3 + d t^4 with P = -E_last, Q = (E_(n-2) -
    E_last) / (2 dt) and c, d from p(T) = p'(T) = 0 (T = (n_extra - 1) dt),
    the last zero_buff + 1 entries zero.  compute_spline (:64-104): each
    record's A splined (zero end slopes) on the unitless spacing h = pe dt /
    (1e12 hbar), read where its (shifted) time lies in [0, laser_end], their
    sum times 0.1 E0 lattice / hbar sampled at spacing h on [0, t_end] (t_end
    = 1.5 laser_end) and splined again with zero end slopes; A(t) = 0 after
    t_end (Laser.hpp:32-37)."""
    def potential(e):
        e = np.asarray(e, dtype=np.float64)
        n = e.size
        a = np.zeros(begin_zero + n + n_extra + zero_buff)
        for i in range(n):
            a[begin_zero + i] = a[begin_zero + i - 1] - e[i] * dt_ps
        A = a[begin_zero + n - 1]
        P = -e[n - 1]
        Q = 0.5 * (e[n - 2] - e[n - 1]) / dt_ps
        T = (n_extra - 1) * dt_ps
        c = -4 * (Q / (2 * T) + (3 * P) / (4 * T * T) + A / (T * T * T))
        d = -0.25 * (3 * c / T + 2 * Q / (T * T) + P / (T * T * T))
        for i in range(1, n_extra):
            t = i * dt_ps
            a[begin_zero + n - 1 + i] = A + P * t + Q * t * t + c * t * t * t + d * t * t * t * t
        a[a.size - begin_zero - 1:] = 0.0
        return a

    per_ps = pe_laser / (1e12 * hbar)
    h = pe_laser * (dt_ps / (1e12 * hbar))
    n_rec = np.asarray(e_a).size
    laser_end_ps = (n_rec - 1) * dt_ps + (n_extra + begin_zero + zero_buff) * dt_ps
    t_end = (1.5 * laser_end_ps) * per_ps
    end = pe_laser * (laser_end_ps / (1e12 * hbar))
    shift = shift_ps * per_ps
    sa = SplinePulse(potential(e_a), 0.0, h, cut=1e300, deriv=(0.0, 0.0))
    sb = SplinePulse(potential(e_b), 0.0, h, cut=1e300, deriv=(0.0, 0.0))
    m = int(t_end / h + 1)
    vals = np.zeros(m + 1)
    for i in range(m + 1):
        t = h * i
        if shift >= 0:
            va = laser(sa, t)[0] if t <= end else 0.0
            vb = laser(sb, t - shift)[0] if 0 <= t - shift <= end else 0.0
        else:
            va = laser(sa, t + shift)[0] if 0 <= t + shift <= end else 0.0
            vb = laser(sb, t)[0] if t <= end else 0.0
        v = va + vb if active == "both" else (va if active == "A" else vb)
        vals[i] = (0.1 / hbar) * e0 * lattice * v
    return SplinePulse(vals, 0.0, h, cut=t_end, deriv=(0.0, 0.0)), t_end


def initial_state(m: OrcModel, kx: float, ky: float, kz: float) -> np.ndarray:
    """orc_initial_state: the model's initial Bloch vector at (kx, ky, kz)."""
    L = lib()
    out = np.zeros(3)
    L.orc_initial_state(ctypes.byref(m), ctypes.c_double(kx), ctypes.c_double(ky),
                        ctypes.c_double(kz), _p(out))
    return out


def grid_tensor(m: OrcModel, nx, ny, x_lo, x_hi, y_lo, y_hi) -> np.ndarray:
    out = np.zeros((nx * ny, KROW))
    lib().orc_grid_tensor(ctypes.byref(m), nx, ny, x_lo, x_hi, y_lo, y_hi, _p(out))
    return out


def grid_rhombic(m: OrcModel, n1, n2) -> np.ndarray:
    out = np.zeros((n1 * n2, KROW))
    lib().orc_grid_rhombic(ctypes.byref(m), ctypes.c_int(n1), ctypes.c_int(n2), _p(out))
    return out


def grid_piflux3d_ref(m: OrcModel, z_range=32, n_coarse=4) -> np.ndarray:
    n = lib().orc_grid_piflux3d_ref(ctypes.byref(m), z_range, n_coarse, None)
    out = np.zeros((n, KROW))
    lib().orc_grid_piflux3d_ref(ctypes.byref(m), z_range, n_coarse, _p(out))
    return out


def grid_piflux3d_debug(m: OrcModel) -> np.ndarray:
    """The 25 momenta of PiFlux::compute_current_density_debug
    (PiFlux.cpp:320-371): momentum_type(pi/2, picked[i], 0.49 pi) with
    picked[i] = 0.5 pi - i 0.02 pi, weight 1, the model's initial state."""
    pi = 3.141592653589793
    out = np.zeros((25, KROW))
    for i in range(25):
        kx, ky, kz = 0.5 * pi, 0.5 * pi - (i * 0.02 * pi), 0.49 * pi
        out[i, :4] = (kx, ky, kz, 1.0)
        out[i, 4:7] = initial_state(m, kx, ky, kz)
    return out


def grid_dirac3d_debug(m: OrcModel, n_z: int, max_k: float) -> np.ndarray:
    """The 25 rows of DiracSystem::compute_current_density_debug
    (DiracSystem.cpp:333-363): k_z = (picked_z - n_z/2) delta_z with picked_z =
    n_z/2 + n_z/10 and delta_z = 2 max_k / n_z, kappa_i = (i + 1) kappa_max / 26
    (kappa_max = sqrt(max_k^2 - k_z^2), DiracSystem.cpp:257-261), weight
    integration_weight = k_z kappa / |k|, the model's initial state."""
    import math
    delta_z = 2 * max_k / n_z
    k_z = (n_z // 2 + n_z // 10 - n_z // 2) * delta_z
    kappa_max = math.sqrt(max_k * max_k - k_z * k_z)
    out = np.zeros((25, KROW))
    for i in range(25):
        kappa = (i + 1) * kappa_max / 26
        mk = math.sqrt(k_z * k_z + kappa * kappa)
        out[i, :4] = (k_z, kappa, mk, k_z * kappa / mk)
        out[i, 4:7] = initial_state(m, k_z, kappa, mk)
    return out


def trapezoidal_fft_unpadded(x: np.ndarray, delta_t: float, t_begin: float, t_end: float):
    """TrapezoidalFFT::compute (TrapezoidalFFT.cpp:11-49) of x as given, as
    hhg.cpp:287-290 applies it to each debug trace: (frequencies, real, imag)."""
    x = np.asarray(x, dtype=np.float64)
    n_in = x.size
    F = np.fft.rfft(x)
    n_fft = n_in // 2 + 1
    freq = 2 * np.arange(n_fft) * np.pi / (n_in * delta_t)
    theta = freq * delta_t
    W = np.empty(n_fft)
    a0 = np.empty(n_fft, dtype=np.complex128)
    for i, th in enumerate(theta):
        if _is_zero(th):
            W[i] = 1.0
            a0[i] = -0.5
        else:
            W[i] = 2.0 * (1.0 - np.cos(th)) / (th * th)
            a0[i] = (-(1.0 - np.cos(th)) + 1j * (th - np.sin(th))) / (th * th)
    corr = a0 * x[0] + np.conj(a0) * np.exp(1j * freq * (t_end - t_begin)) * x[n_in - 1]
    out = (delta_t * W) * np.exp(1j * freq * t_begin) * F + corr
    return freq, delta_t * out.real, delta_t * out.imag


def grid_honeycomb_hex_ref(m: OrcModel, n_k=64) -> np.ndarray:
    n = lib().orc_grid_honeycomb_hex_ref(ctypes.byref(m), n_k, None)
    out = np.zeros((n, KROW))
    lib().orc_grid_honeycomb_hex_ref(ctypes.byref(m), n_k, _p(out))
    return out


def evolve_k(m, p: Pulse, tc, s, krow) -> tuple[np.ndarray, OrcStats]:
    st = OrcStats()
    out = np.zeros((tc.n_measurements + 1, 3))
    krow = np.ascontiguousarray(krow, dtype=np.float64)
    pc = p.c()
    rc = lib().orc_evolve_k(ctypes.byref(m), ctypes.byref(pc), ctypes.byref(tc),
                            ctypes.byref(s), _p(krow), _p(out), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"orc_evolve_k failed with status {rc}")
    return out, st


def step_history(m, p: Pulse, tc, s, krow, cap=1 << 20) -> np.ndarray:
    hist = np.zeros((cap, 4))
    krow = np.ascontiguousarray(krow, dtype=np.float64)
    pc = p.c()
    n = lib().orc_step_history(ctypes.byref(m), ctypes.byref(pc), ctypes.byref(tc),
                               ctypes.byref(s), _p(krow), ctypes.c_int(cap), _p(hist))
    if n < 0:
        raise RuntimeError(f"orc_step_history failed with status {-n}")
    return hist[:n]


def current_density(m, p: Pulse, tc, s, ktab: np.ndarray, threads=0, fast=False):
    ktab = np.ascontiguousarray(ktab, dtype=np.float64)
    j = np.zeros(tc.n_measurements + 1)
    st = OrcStats()
    pc = p.c()
    rc = lib(fast).orc_current_density(ctypes.byref(m), ctypes.byref(pc), ctypes.byref(tc),
                                       ctypes.byref(s), ctypes.c_int(ktab.shape[0]), _p(ktab),
                                       _p(j), ctypes.byref(st), ctypes.c_int(threads))
    return j, st, rc


def k_resolved(m, p, tc, s, ktab: np.ndarray, kind: int, threads=0, fast=False):
    """orc_k_resolved: (n_measurements + 1, n_k, 3 | 2) samples and status
    (fast: the -O3 -ffast-math build, for CPU timing)."""
    ktab = np.ascontiguousarray(ktab, dtype=np.float64)
    w = 3 if kind == 0 else 2
    out = np.zeros((tc.n_measurements + 1, ktab.shape[0], w))
    pc = p.c()
    rc = lib(fast).orc_k_resolved(ctypes.byref(m), ctypes.byref(pc), ctypes.byref(tc), ctypes.byref(s),
                              ctypes.c_int(ktab.shape[0]), _p(ktab), ctypes.c_int(kind), _p(out),
                              ctypes.c_int(threads))
    return out, rc


def split_current(m, p, tc, s, ktab: np.ndarray, cut: float, threads=0):
    """orc_split_current: (j_low, j_high, status)."""
    ktab = np.ascontiguousarray(ktab, dtype=np.float64)
    lo = np.zeros(tc.n_measurements + 1)
    hi = np.zeros(tc.n_measurements + 1)
    pc = p.c()
    rc = lib().orc_split_current(ctypes.byref(m), ctypes.byref(pc), ctypes.byref(tc), ctypes.byref(s),
                                 ctypes.c_int(ktab.shape[0]), _p(ktab), ctypes.c_double(cut), _p(lo),
                                 _p(hi), ctypes.c_int(threads))
    return lo, hi, rc


def kappa_rows(m: OrcModel, k_z: float, a: float, H: float, level: int, n_kappa: int) -> np.ndarray:
    """The Dirac-3D rows one split [a, a + H] integrates at `level`: level 0
    the n_kappa + 1 trapezoid nodes a + i H/n_kappa (ends weighted 1/2),
    level L > 0 the midpoints a + i H/(n_kappa 2^L), i odd; kappa = 0 is left
    out (the reference's integrand is zero there, DiracSystem.cpp:301-303).
    Row: k_z, kappa, |k|, weight x k_z kappa/|k| (DiracSystem.cpp:281), S0, 0."""
    panels = n_kappa << level
    h = H / panels
    idx = range(0, panels + 1) if level == 0 else range(1, panels, 2)
    rows = []
    for i in idx:
        kappa = a + i * h
        if _is_zero(kappa):
            continue
        mk = float(np.sqrt(k_z * k_z + kappa * kappa))
        end = 0.5 if level == 0 and i in (0, panels) else 1.0
        rows.append([k_z, kappa, mk, end * (k_z * kappa / mk), *initial_state(m, k_z, kappa, 0.0), 0.0])
    return np.array(rows, dtype=np.float64).reshape(-1, KROW)


def adaptive_kappa(contrib, slices_kz, kappa_max, n_kappa: int, threshold: float, n_splits: int,
                   max_halvings: int, dz: float, n_samples: int, rows_fn, only=None):
    """The adaptive trapezoidal rule of the Dirac-3D kappa integral, restated
    from the reference's call split_integrate<100>(f, 0, kappa_max, n_kappa,
    threshold, elementwise error) (DiracSystem.cpp:307-310; the integrator's
    library is not available): each of n_splits equal splits starts as the
    n_kappa-panel trapezoid and is halved, T <- T/2 + h sum f(midpoints),
    until max_t |T_new - T_old| < threshold or max_halvings halvings; the
    slice's integral is the sum of its splits in order, and j = dz times the
    sum of the slices in order (DiracSystem.cpp:313-321).  `rows_fn(z, a, H,
    level)` gives a split's rows, `contrib(rows)` the weighted samples
    (n_samples, n_rows).  Every round evaluates all active splits' rows in one
    batch.  `only` restricts the work to a list of (slice, split) pairs (the
    splits are independent; j then sums those only).  Returns j and {rounds,
    unconverged, max_level, trajectories}."""
    n_slices = len(slices_kz)
    T = np.zeros((n_slices, n_splits, n_samples))
    level = np.zeros((n_slices, n_splits), dtype=int)
    active = (list(only) if only is not None else
              [(z, sp) for z in range(n_slices) for sp in range(n_splits)])
    info = {"rounds": 0, "unconverged": 0, "max_level": 0, "trajectories": 0}
    while active:
        info["rounds"] += 1
        H = [kappa_max[z] / n_splits for z in range(n_slices)]
        parts = [rows_fn(z, sp * H[z], H[z], level[z, sp]) for z, sp in active]
        batch = np.concatenate(parts) if parts else np.zeros((0, KROW))
        info["trajectories"] += batch.shape[0]
        c = contrib(batch) if batch.shape[0] else np.zeros((n_samples, 0))
        off = 0
        still = []
        for (z, sp), rows in zip(active, parts):
            L = level[z, sp]
            h = H[z] / (n_kappa << L)
            acc = c[:, off:off + rows.shape[0]].sum(axis=1)
            off += rows.shape[0]
            old = T[z, sp].copy()
            T[z, sp] = (0.0 if L == 0 else 0.5) * old + h * acc
            change = float(np.max(np.abs(T[z, sp] - old)))
            info["max_level"] = max(info["max_level"], int(L))
            if L > 0 and change < threshold:
                continue
            if L >= max_halvings or np.isnan(change):
                info["unconverged"] += 1
                continue
            level[z, sp] = L + 1
            still.append((z, sp))
        active = still
    j = np.zeros(n_samples)
    for z in range(n_slices):
        sl = np.zeros(n_samples)
        for sp in range(n_splits):
            sl = sl + T[z, sp]
        j = j + sl
    return j * dz, info


def dirac_kappa_current(m: OrcModel, p, tc, s, max_k: float, n_z: int, n_kappa: int = 10,
                        threshold: float = 1e-3, n_splits: int = 100, max_halvings: int = 12):
    """DiracSystem::compute_current_density (DiracSystem.cpp:271-331; with
    relaxation compute_current_density_diagonal_relaxation, :365-425) on the
    oracle: k_z = (z - n_z/2) 2 max_k / n_z for z = 1 .. n_z - 1 without
    n_z/2, kappa in [0, sqrt(max_k^2 - k_z^2)] by ``adaptive_kappa``, the
    integrand S_z k_z kappa / |k| from orc_evolve_k with the model's stepper
    (s.stepper 2: the closed-form Magnus step).  Returns (j, info, status)."""
    dz = 2 * max_k / n_z
    kz = [(z - n_z // 2) * dz for z in range(1, n_z) if z != n_z // 2]
    kmax = [float(np.sqrt(max_k * max_k - k * k)) for k in kz]
    status = [0]

    def contrib(rows):
        out, rc = k_resolved(m, p, tc, s, rows, 0)
        if rc != 0:
            status[0] = rc
        return out[:, :, 2] * rows[:, 3][None, :]

    j, info = adaptive_kappa(contrib, kz, kmax, n_kappa, threshold, n_splits, max_halvings, dz,
                             tc.n_measurements + 1,
                             lambda z, a, H, L: kappa_rows(m, kz[z], a, H, L, n_kappa))
    return j, info, status[0]


def magnus_coefficients(p: Pulse, delta_t, t0) -> np.ndarray:
    out = np.zeros(4)
    pc = p.c()
    lib().orc_magnus_coefficients(ctypes.byref(pc), ctypes.c_double(delta_t),
                                  ctypes.c_double(t0), _p(out))
    return out


def dirac_magnus_U(k, kappa, k_z, delta_t, coeffs) -> np.ndarray:
    U = np.zeros(9)
    cf = np.ascontiguousarray(coeffs, dtype=np.float64)
    lib().orc_dirac_magnus_U(ctypes.c_double(k), ctypes.c_double(kappa), ctypes.c_double(k_z),
                             ctypes.c_double(delta_t), _p(cf), _p(U))
    return U.reshape(3, 3)


def dirac3d_magnus_k(p: Pulse, tc, k_z, kappa) -> np.ndarray:
    out = np.zeros(tc.n_measurements + 1)
    pc = p.c()
    lib().orc_dirac3d_magnus_k(ctypes.byref(pc), ctypes.byref(tc), ctypes.c_double(k_z),
                               ctypes.c_double(kappa), _p(out))
    return out


def dirac3d_sigma_k(p: Pulse, tc, s, k_z, kappa) -> np.ndarray:
    out = np.zeros(tc.n_measurements + 1)
    st = OrcStats()
    pc = p.c()
    rc = lib().orc_dirac3d_sigma_k(ctypes.byref(pc), ctypes.byref(tc), ctypes.byref(s),
                                   ctypes.c_double(k_z), ctypes.c_double(kappa), _p(out),
                                   ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"orc_dirac3d_sigma_k failed with status {rc}")
    return out


def rkf78_tableau():
    c = np.zeros(13)
    a = np.zeros(169)
    b = np.zeros(13)
    db = np.zeros(13)
    lib().orc_rkf78_tableau(_p(c), _p(a), _p(b), _p(db))
    return c, a.reshape(13, 13), b, db


# --------------------------------------------------------------------------
# Fourier tail
# --------------------------------------------------------------------------
ZERO_PADDING = 8  # sources/hhg.cpp:36


def _is_zero(x: float) -> bool:
    """GlobalDefinitions.hpp:61-71: |x| < 2^-44 by the biased exponent."""
    bits = np.array([x], dtype=np.float64).view(np.uint64)[0]
    return int((int(bits) >> 52) & 0x7FF) < 0x3D3


def trapezoidal_fft(j: np.ndarray, t_begin: float, t_end: float, n_measurements: int):
    """TrapezoidalFFT::compute on the x8 zero-padded j(t) (hhg.cpp:277-285).

    Returns (frequencies, real, imag), each of length n_in/2 + 1 with
    n_in = 8 (N + 1).  The end-point correction reads input[n_in - 1], which
    the zero padding makes 0, exactly as the reference does.
    """
    delta_t = (t_end - t_begin) / n_measurements
    n_in = ZERO_PADDING * (n_measurements + 1)
    x = np.zeros(n_in)
    x[: len(j)] = j
    F = np.fft.rfft(x)
    n_fft = n_in // 2 + 1
    freq = 2 * np.arange(n_fft) * np.pi / (n_in * delta_t)
    theta = freq * delta_t
    W = np.empty(n_fft)
    a0 = np.empty(n_fft, dtype=np.complex128)
    for i, th in enumerate(theta):
        if _is_zero(th):
            W[i] = 1.0
            a0[i] = -0.5
        else:
            W[i] = 2.0 * (1.0 - np.cos(th)) / (th * th)
            a0[i] = (-(1.0 - np.cos(th)) + 1j * (th - np.sin(th))) / (th * th)
    corr = a0 * x[0] + np.conj(a0) * np.exp(1j * freq * (t_end - t_begin)) * x[n_in - 1]
    out = (delta_t * W) * np.exp(1j * freq * t_begin) * F + corr
    return freq, delta_t * out.real, delta_t * out.imag


def harmonic_intensities(freq, re, im, max_order: int):
    """I(n) = |j_hat(n omega_L)|^2 at integer harmonics n = 1..max_order.

    Frequencies are in units of omega_L (time in 1/omega_L), so harmonic n
    sits at freq = n; the nearest bin is used.
    """
    p = re * re + im * im
    out = np.zeros(max_order)
    for n in range(1, max_order + 1):
        out[n - 1] = p[int(np.argmin(np.abs(freq - n)))]
    return out
