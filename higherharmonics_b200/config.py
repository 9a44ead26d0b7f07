"""The reference's parameter files as engine descriptors.

A parameter file (params/*.config in the reference) holds `key value` lines;
`#` starts a comment; this reader ignores words after the value (wang.config
lists units there).  `from_config` maps
one onto (system, pulse, grid, solver) descriptors with the unit conversions
of the reference's dispatchers and system constructors:

  beta          = photon_energy / (k_B T), T = 0 -> 0       (PiFlux.cpp:63)
  E_F           -> E_F / photon_energy                      (PiFlux.cpp:64)
  hopping       = band_width / sqrt(12) (PiFlux, PiFlux.cpp:65),
                  band_width / 6 (Honeycomb, Honeycomb.cpp:91)
  lattice const = sqrt(3) hbar v_F / (photon_energy band_width) (PiFlux.cpp:66),
                  4 hbar v_F / (photon_energy band_width) (Honeycomb.cpp:92)
  1/tau         = 1e15 hbar / (tau photon_energy)           (PiFlux.cpp:67-68)
  A0            = lattice const * 1e11 E0 / photon_energy   (Laser.cpp:24-25)
  off-diagonal tau <= 0 -> the diagonal one (PiFluxDispatcher.cpp:22-35)
  N             = n_laser_cycles * 1024 intervals           (hhg.cpp:86-87)
  window        = [pi t0_offset, laser end + 2 pi] for the cosine laser
                  (PiFluxDispatcher.cpp:50-53, HoneycombDispatcher.cpp:32-35)
  grids         = the reference's compiled-in quadratures: PiFlux z_range 32,
                  N_coarse 4 (PiFlux.hpp:11-22); Honeycomb N_k 64
                  (Honeycomb.hpp:12-21)

Lasers (the dispatchers' laser_type branches, PiFluxDispatcher.cpp:44-106,
HoneycombDispatcher.cpp:28-56): cosine, continuous and gauss run as analytic
pulses; powerlaw<e>, quench and the double lasers dcos/dcosA/dcosB and
dgauss/dgaussA/dgaussB are splines in the reference and are handed to the
device as the same spline samples (PowerLawField.cpp:19-31,
QuenchedField.cpp:15-29, DoubleLaser.hpp:42-68).  The photon energy of the
system is multiplied by the experimental one for the exp and double lasers
(Dispatcher.cpp:10-19).  The experimental lasers exp/expA/expB build A(t)
from a measured field (ExperimentalLaser.cpp:30-108, `experimental_pulse`):
this package does not carry the reference's measured data, so the caller
names a file with it (`experimental_field <path>`: two columns E_A E_B in
MV/cm at the spacing `experimental_dt`, default 0.03335555 ps; the data's
photon energy `experimental_photon_energy`, default 6.091420442472572 meV,
ExperimentParams.hpp:5,12); without that key they raise UnsupportedConfig.

system_type Dirac follows DiracDispatcher (DiracDispatcher.cpp:16-63) and the
DiracSystem constructor (DiracSystem.cpp:52-63): the same beta, E_F and 1/tau,
max_k = band_width, A0 = (hbar v_F / photon_energy) 1e11 E0 / photon_energy
(laser_model_ratio, DiracSystem.hpp:30-32), the cosine window [pi t0_offset,
laser end] without the extra 2 pi, the lasers continuous / cosine / quench /
powerlaw<e>, and the momentum quadrature n_z slices x the adaptive kappa rule
with n_kappa = 10 and threshold 1e-3 (DiracDispatcher.cpp:13-14); its
coherent path is the closed-form Magnus step, the relaxation path FP64 RKF78
(DiracDispatcher.cpp:66-79).  The
occupation and split-current run modes are in higherharmonics_b200.runmodes;
requesting either shortens the double / Gaussian / experimental laser windows to
0.75 t_end for every mode, as the dispatcher's reduced_duration does
(PiFluxDispatcher.cpp:45).  debug_data yes / only selects the PiFlux
or Dirac debug traces in higherharmonics_b200.runmodes; for Honeycomb (whose
reference throws) it raises UnsupportedConfig.  data_dir and n_z are read by
the run modes only.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

from . import api

HBAR = 6.582119569509065698e-13  # meV s (GlobalDefinitions.hpp:28)
K_B = 0.08617333262145177434     # meV / K (GlobalDefinitions.hpp:29)
SQRT3 = 1.732050807568877293527446341
SQRT12 = 3.464101615137754587054892683
MEASUREMENTS_PER_CYCLE = 1 << 10
EXP_PHOTON_ENERGY = 6.091420442472572  # meV (ExperimentParams.hpp:12)
EXP_DT_PS = 0.03335555  # ps between the measured field samples (ExperimentParams.hpp:5)
# samples of the quartic tail that brings A to rest, and the zero samples
# before and after the measured record (ExperimentParams.hpp:6-9)
EXP_N_EXTRA, EXP_BEGIN_ZERO, EXP_ZERO_BUFF = 16, 8, 8
EXP_LASERS = {"exp": "both", "expA": "A", "expB": "B"}
DOUBLE_LASERS = {"dcos": ("cosine", "both"), "dcosA": ("cosine", "A"), "dcosB": ("cosine", "B"),
                 "dgauss": ("gauss", "both"), "dgaussA": ("gauss", "A"), "dgaussB": ("gauss", "B")}
PIFLUX_Z_RANGE, PIFLUX_N_COARSE = 32, 4
DIRAC_N_KAPPA, DIRAC_KAPPA_THRESHOLD, DIRAC_SPLITS = 10, 1e-3, 100
HONEYCOMB_N_K = 64


class UnsupportedConfig(ValueError):
    """A valid reference configuration that this engine does not run."""


def read_config(source: str) -> dict[str, str]:
    """Parse a parameter file (a path or the text itself) into {key: value}."""
    text = open(source).read() if os.path.exists(source) else source
    out: dict[str, str] = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        parts = line.split()
        if len(parts) < 2:
            raise ValueError(f"config line without a value: {line!r}")
        out[parts[0]] = parts[1]
    return out


def _is_zero(x: float) -> bool:
    # GlobalDefinitions.hpp:61-71: |x| < 2^-44 by the biased exponent
    return abs(x) < 2.0 ** -44


@dataclass
class Run:
    """Descriptors of one run.  `lattice_constant` is the laser model ratio of
    the system (Dirac: hbar v_F / photon_energy); the Dirac system integrates
    over `quad` instead of a grid."""
    system_type: str
    system: api.SystemDesc
    pulse: api.PulseDesc
    grid: api.GridDesc | None
    opts: api.SolverOpts
    lattice_constant: float
    quad: api.KappaQuad | None = None


def from_config(cfg: dict | str, *, grid: api.GridDesc | None = None,
                n_measurements: int | None = None) -> Run:
    """Descriptors for one reference run.  ``grid`` / ``n_measurements``
    override the reference's compiled-in quadrature and its 1024 samples per
    cycle (for smaller test runs)."""
    if isinstance(cfg, str):
        cfg = read_config(cfg)

    def num(key: str) -> float:
        if key not in cfg:
            raise ValueError(f"missing config key {key!r}")
        return float(cfg[key])

    system_type = cfg.get("system_type", "")
    if system_type not in ("PiFlux", "Honeycomb", "Dirac", "ModifiedPiFlux"):
        raise ValueError(f"System type '{system_type}' not recognized!")
    if system_type == "ModifiedPiFlux":
        raise UnsupportedConfig("system_type ModifiedPiFlux is not built")
    if cfg.get("debug_data", "no") != "no" and system_type == "Honeycomb":
        # Honeycomb.cpp:111-115
        raise UnsupportedConfig("Honeycomb::compute_current_density_debug is not implemented yet!")
    reduced = cfg.get("occupations", "no") != "no" or cfg.get("split_current", "no") != "no"
    laser_type = cfg.get("laser_type", "")
    known = {"cosine", "continuous", "gauss", "quench", "exp", "expA", "expB"} | set(DOUBLE_LASERS)
    if not (laser_type in known or laser_type.startswith("powerlaw")) or \
            (system_type in ("Honeycomb", "Dirac") and (laser_type in DOUBLE_LASERS or laser_type == "gauss")):
        raise ValueError(f"Laser type '{laser_type}' is not recognized!")
    measured = None
    if laser_type in EXP_LASERS:
        if "experimental_field" not in cfg:
            raise UnsupportedConfig(f"laser_type {laser_type}: the reference's measured field is "
                                    "not part of this package; name a file with it "
                                    "(experimental_field <path>: columns E_A E_B in MV/cm)")
        measured = MeasuredField.load(cfg["experimental_field"],
                                      float(cfg.get("experimental_dt", EXP_DT_PS)),
                                      float(cfg.get("experimental_photon_energy",
                                                    EXP_PHOTON_ENERGY)))

    T, E_F, v_F = num("T"), num("E_F"), num("v_F")
    band_width, E0, pe_in = num("band_width"), num("field_amplitude"), num("photon_energy")
    # Dispatcher::get_photon_energy: the exp and double lasers' photon energy
    # is in units of the experimental one
    exp_pe = measured.photon_energy if measured is not None else EXP_PHOTON_ENERGY
    pe = pe_in * exp_pe if (laser_type in DOUBLE_LASERS or laser_type in EXP_LASERS) else pe_in
    tau_d = num("diagonal_relaxation_time")
    tau_o = float(cfg.get("offdiagonal_relaxation_time", "-1"))
    n_cycles = int(num("n_laser_cycles"))
    t0_offset = float(cfg.get("t0_offset", "0"))

    beta = 0.0 if _is_zero(T) else pe / (K_B * T)
    inv_d = (1e15 * HBAR) / (tau_d * pe)
    n = n_measurements or n_cycles * MEASUREMENTS_PER_CYCLE
    if system_type == "Dirac":
        relax = tau_d > 0  # DiracDispatcher::compute (DiracDispatcher.cpp:66-79)
        sys_ = api.system(api.SYS_DIRAC3D, beta=beta, fermi_energy=E_F / pe,
                          inv_diag_relax=inv_d if relax else 0.0)
        ratio = HBAR * v_F / pe  # DiracSystem::laser_model_ratio
        if laser_type == "cosine":
            # CosineLaser(.., n_laser_cycles, pi t0_offset) with time_config =
            # {t_begin, t_end} (DiracDispatcher.cpp:34-37)
            t_begin = math.pi * t0_offset
            pulse = api.cosine_pulse(_amplitude(ratio, E0, pe), n_cycles, n, t_begin=t_begin,
                                     window=(t_begin, t_begin + 2 * math.pi * n_cycles))
        elif measured is not None:
            # the system keeps the config's photon energy; the laser's model
            # ratio takes the experimental one (DiracDispatcher.cpp:38-52)
            pe_l = pe_in * measured.photon_energy
            pulse = experimental_pulse(measured, pe_l, E0, HBAR * v_F / pe_l, t0_offset,
                                       EXP_LASERS[laser_type], n)
        else:
            pulse = make_pulse(laser_type, ratio, E0, pe_in, n_cycles, t0_offset, n)
        quad = api.kappa_quad(band_width, int(num("n_z")), DIRAC_N_KAPPA,
                              DIRAC_KAPPA_THRESHOLD, DIRAC_SPLITS)
        opts = (api.solver(1e-12, 1e-8) if relax else
                api.solver(stepper=api.STEPPER_DIRAC_MAGNUS))
        return Run(system_type, sys_, pulse, None, opts, ratio, quad)
    if system_type == "PiFlux":
        hopping = band_width / SQRT12
        lattice = SQRT3 * HBAR * v_F / (pe * band_width)
        inv_o = (1e15 * HBAR) / ((tau_o if tau_o > 0 else tau_d) * pe)
        kind, pol = api.SYS_PIFLUX3D, (1.0, 0.0)
        g = grid or api.grid_piflux3d_ref(PIFLUX_Z_RANGE, PIFLUX_N_COARSE)
    else:
        hopping = band_width / 6
        lattice = 4 * HBAR * v_F / (pe * band_width)
        inv_o = 0.0
        kind, pol = api.SYS_HONEYCOMB, (1.0, 0.0)  # laser_theta = 0 (Honeycomb.hpp:87)
        g = grid or api.grid_honeycomb_hex_ref(HONEYCOMB_N_K)
    relax = inv_d > 0.0  # __time_evolution__ (PiFlux.cpp:509-516, Honeycomb.cpp:214-223)
    sys_ = api.system(kind, hopping=hopping, pol=pol, beta=beta, fermi_energy=E_F / pe,
                      inv_diag_relax=inv_d if relax else 0.0,
                      inv_offdiag_relax=inv_o if relax else 0.0)
    if measured is not None:
        # PiFlux shortens the window to 0.75 t_end for the occupation and
        # split-current runs, Honeycomb does not (PiFluxDispatcher.cpp:59-70,
        # HoneycombDispatcher.cpp:36-47)
        pulse = experimental_pulse(measured, pe, E0, lattice, t0_offset, EXP_LASERS[laser_type], n,
                                   0.75 if (reduced and system_type == "PiFlux") else 1.0)
    else:
        pulse = make_pulse(laser_type, lattice, E0, pe_in, n_cycles, t0_offset, n, reduced)
    return Run(system_type, sys_, pulse, g, api.solver(1e-12, 1e-8), lattice)


def _amplitude(ratio: float, E0: float, pe: float) -> float:
    return ratio * 1e11 * E0 / pe  # Laser.cpp:24-25


def _cosine(A0: float, n: float, t_begin: float, t: float) -> float:
    # CosineLaser::laser_function (CosineLaser.cpp:22-26, Laser.hpp:32-37)
    if t <= t_begin or t >= t_begin + 2 * math.pi * n:
        return 0.0
    return A0 * (0.5 * (1. - math.cos((1. / n) * (t - t_begin))) * math.sin(t))


def _gauss(A0: float, n: float, t_begin: float, t: float) -> float:
    # GaussLaser (GaussLaser.cpp:9-38)
    centre = t_begin + 0.5 * (2.0 * math.pi * 3.0 * n)
    sigma = math.pi * n / math.sqrt(2.0 * math.log(1.0 / 0.05))
    return A0 * (math.exp(-((t - centre) * (t - centre)) / (2.0 * sigma * sigma)) * math.sin(t))


def make_pulse(laser_type: str, ratio: float, E0: float, pe_in: float, n_cycles: int,
               t0_offset: float, n: int, reduced: bool = False) -> api.PulseDesc:
    """The pulse and TimeIntegrationConfig of one laser_type, as the PiFlux /
    Honeycomb dispatchers build them from the config's photon_energy pe_in
    (reduced: the occupation / split-current runs' 0.75 t_end windows)."""
    cut = 0.75 if reduced else 1.0
    pe = pe_in * EXP_PHOTON_ENERGY if laser_type in DOUBLE_LASERS else pe_in
    if laser_type == "cosine":
        t_begin = math.pi * t0_offset
        t_end = t_begin + 2 * math.pi * n_cycles  # CosineLaser::base_duration
        return api.cosine_pulse(_amplitude(ratio, E0, pe), n_cycles, n, t_begin=t_begin,
                                window=(t_begin, t_end + 2 * math.pi))
    if laser_type == "continuous":
        return api.continuous_pulse(_amplitude(ratio, E0, pe), n,
                                    (-n_cycles * math.pi, n_cycles * math.pi))
    if laser_type == "gauss":
        t_begin = t0_offset  # GaussLaser(.., n_laser_cycles, t0_offset)
        return api.gauss_pulse(_amplitude(ratio, E0, pe), n_cycles, n, t_begin=t_begin,
                               window=(t_begin, cut * (t_begin + 2 * math.pi * 3.0 * n_cycles)))
    if laser_type == "quench" or laser_type.startswith("powerlaw"):
        # a 256-sample spline template over [0, duration], duration = t0_offset
        A0, t_end, N = _amplitude(ratio, E0, pe), t0_offset, 256
        if laser_type == "quench":
            y = [0.0 if (i < N // 4 or i > 3 * N // 4) else
                 (0.5 * A0 if i in (N // 4, 3 * N // 4) else A0) for i in range(N)]
            deriv = (0.0, 0.0)
        else:
            e = float(laser_type[len("powerlaw"):])
            dt = t_end / N
            norm = 1. / t_end ** e if e > 0 else 1. / dt ** e
            y = [0.0] + [A0 * (i * dt) ** e * norm for i in range(1, N)]
            deriv = (math.nan, math.nan)  # boost estimates them; exact for the linear ramp
        return api.spline_pulse(y, 0.0, t_end / (N - 1), n, (0.0, t_end), cut=t_end, deriv=deriv)
    base, active = DOUBLE_LASERS[laser_type]
    # DoubleLaser<Base>(photon_energy, E0, ratio, n_cycles, t0_offset): laser A
    # with 1.6 E0 at t = 0, laser B with 0.7 E0 delayed by t0_offset ps, sampled
    # at 1000 points over 1.5 base durations, spline with zero end slopes
    duration = 2 * math.pi * n_cycles * (3.0 if base == "gauss" else 1.0)
    t_max = 1.5 * duration
    shift = pe_in * (t0_offset * EXP_PHOTON_ENERGY / (1e12 * HBAR))  # ps_to_uniteless
    one = _gauss if base == "gauss" else _cosine
    aA, aB = _amplitude(ratio, 1.6 * E0, pe), _amplitude(ratio, 0.7 * E0, pe)
    N = 1000
    dt = t_max / (N - 1)
    y = []
    for i in range(N):
        t = i * dt
        a, b = one(aA, n_cycles, 0.0, t), one(aB, n_cycles, 0.0, t - shift + 0.0)
        y.append(a + b if active == "both" else (a if active == "A" else b))
    return api.spline_pulse(y, 0.0, dt, n, (0.0, cut * t_max), cut=t_max, deriv=(0.0, 0.0))


@dataclass
class MeasuredField:
    """A measured two-pulse electric field: E_A and E_B in MV/cm at spacing
    dt_ps (ps), and the photon energy (meV) the data define."""
    e_a: "np.ndarray"
    e_b: "np.ndarray"
    dt_ps: float = EXP_DT_PS
    photon_energy: float = EXP_PHOTON_ENERGY

    @staticmethod
    def load(path: str, dt_ps: float = EXP_DT_PS,
             photon_energy: float = EXP_PHOTON_ENERGY) -> "MeasuredField":
        import numpy as np
        data = np.loadtxt(path, ndmin=2)
        if data.shape[1] < 2 or data.shape[0] < 3:
            raise ValueError(f"{path}: need at least 3 rows of two columns (E_A E_B, MV/cm)")
        return MeasuredField(np.ascontiguousarray(data[:, 0]), np.ascontiguousarray(data[:, 1]),
                             dt_ps, photon_energy)


def measured_vector_potential(e, dt: float):
    """A = -int E dt of a measured record (the factor c cancels in the Peierls
    substitution), the way ExperimentalLaser's vector_potential builds it
    (ExperimentalLaser.cpp:30-62): EXP_BEGIN_ZERO zeros, the running sum
    -dt sum_{m <= i} E_m, then a quartic over EXP_N_EXTRA - 1 steps that
    continues A with its last value, slope -E_last and curvature (from the
    last two samples) and reaches zero with zero slope, then zeros (the last
    EXP_ZERO_BUFF + 1 entries)."""
    import numpy as np
    e = np.asarray(e, dtype=np.float64)
    n = e.size
    out = np.zeros(n + EXP_N_EXTRA + EXP_ZERO_BUFF + EXP_BEGIN_ZERO)
    acc = 0.0
    for i in range(n):
        acc = acc - e[i] * dt
        out[EXP_BEGIN_ZERO + i] = acc
    a_last = out[EXP_BEGIN_ZERO + n - 1]
    p1 = -e[n - 1]
    p2 = 0.5 * (e[n - 2] - e[n - 1]) / dt
    T = (EXP_N_EXTRA - 1) * dt
    # p(T) = 0 and p'(T) = 0 fix the cubic and quartic coefficients
    c3 = -4 * (p2 / (2 * T) + (3 * p1) / (4 * T * T) + a_last / (T * T * T))
    c4 = -0.25 * (3 * c3 / T + 2 * p2 / (T * T) + p1 / (T * T * T))
    for i in range(1, EXP_N_EXTRA):
        t = i * dt
        out[EXP_BEGIN_ZERO + n - 1 + i] = (a_last + p1 * t + p2 * t * t + c3 * t * t * t +
                                           c4 * t * t * t * t)
    out[out.size - EXP_BEGIN_ZERO - 1:] = 0.0
    return out


def experimental_pulse(field: MeasuredField, pe_laser: float, E0: float, lattice: float,
                       shift_ps: float, active: str, n: int, window_scale: float = 1.0
                       ) -> api.PulseDesc:
    """ExperimentalLaser (ExperimentalLaser.cpp:8-108) as a spline pulse.

    pe_laser is the laser's photon energy in meV (the config's photon_energy
    times the data's), lattice the system's laser model ratio, shift_ps the
    delay of pulse B after pulse A (t0_offset, ps; negative delays A),
    active "both" / "A" / "B".  The two vector potentials are splined on the
    unitless sample spacing dt = pe_laser dt_ps / (1e12 hbar), each is cut
    after the record's end laser_end = (samples - 1 + 32) dt_ps, and their
    sum scaled by 0.1 E0 lattice / hbar is sampled at spacing dt over [0,
    t_end], t_end = 1.5 laser_end (unified_t_max); that sampling, splined
    with zero end slopes, is A(t) for t <= t_end.  The window is [0,
    window_scale t_end] with n measurement intervals."""
    import numpy as np
    to_unitless = pe_laser / (1e12 * HBAR)  # 1/ps
    dt = pe_laser * (field.dt_ps / (1e12 * HBAR))
    laser_end_ps = (field.e_a.size - 1 + EXP_N_EXTRA + EXP_BEGIN_ZERO + EXP_ZERO_BUFF) * field.dt_ps
    t_end = (1.5 * laser_end_ps) * to_unitless
    end = pe_laser * (laser_end_ps / (1e12 * HBAR))
    shift = shift_ps * to_unitless
    inner = []
    for e in (field.e_a, field.e_b):
        a = measured_vector_potential(e, field.dt_ps)
        inner.append(api.spline_pulse(a, 0.0, dt, 1, (0.0, (a.size - 1) * dt), cut=1e300,
                                      deriv=(0.0, 0.0)))
    n_temp = int(t_end / dt + 1)
    t = 0.0 + dt * np.arange(n_temp + 1)
    if shift >= 0:
        ta, tb = t, t - shift
        in_a = ta <= end
        in_b = (tb >= 0) & (tb <= end)
    else:
        ta, tb = t + shift, t
        in_a = (ta >= 0) & (ta <= end)
        in_b = tb <= end
    A = np.where(in_a, api.pulse_values(inner[0], ta), 0.0)
    B = np.where(in_b, api.pulse_values(inner[1], tb), 0.0)
    tot = A + B if active == "both" else (A if active == "A" else B)
    samples = (0.1 / HBAR) * E0 * lattice * tot
    return api.spline_pulse(samples, 0.0, dt, n, (0.0, window_scale * t_end), cut=t_end,
                            deriv=(0.0, 0.0))
