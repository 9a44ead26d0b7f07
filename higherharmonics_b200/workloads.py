"""The synthetic workloads the engine is measured and checked on: the five
configurations of the hot path plus the reference's production PiFlux run
with relaxation.

Units: the reference's (time in 1/omega_L, energies in hbar omega_L).  A
model given in "reduced units" with a laser frequency omega is integrated
with energy_scale = 1/omega, and A(t) = A0 sin^2(pi t/T) sin(omega t + phi)
becomes A0 sin^2(tau / (2 n_cyc)) sin(tau + phi) in tau = omega t, i.e. the
reference's CosineLaser (CosineLaser.cpp:22-26) plus a carrier phase.
Samples: 1024 per cycle (sources/hhg.cpp:87-88).

Seeded pulse tables use splitmix64 -> 53-bit uniforms, seed 20261203.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import api

SEED = 20261203
MEASUREMENTS_PER_CYCLE = 1 << 10


def splitmix64_uniforms(n: int, seed: int = SEED) -> np.ndarray:
    """n uniforms in [0, 1) from splitmix64 (top 53 bits)."""
    out = np.empty(n)
    s = seed & 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        s = (s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z = z ^ (z >> 31)
        out[i] = (z >> 11) * (1.0 / (1 << 53))
    return out


@dataclass
class Workload:
    name: str
    system: api.SystemDesc
    pulses: list
    grid: api.GridDesc
    opts_kw: dict
    description: str

    def opts(self, **kw) -> api.SolverOpts:
        d = dict(self.opts_kw)
        d.update(kw)
        return api.solver(**d)

    @property
    def n_k(self) -> int:
        g = self.grid
        if g.kind in (api.GRID_TENSOR_GL, api.GRID_RHOMBIC_GL):
            return g.n1 * g.n2
        return int(api.grid_rows(self.system, g).shape[0])


def dirac2d_64(n_grid=64, n_cycles=4, omega=0.1) -> Workload:
    """Gapped 2D Dirac, v = 1, Delta = 0.05, omega = 0.1, 4 cycles, A0 = 1,
    phi = 0, 64x64 GL on [-2,2]^2, S0 = -d_hat, RKF78 abs = rel = 1e-10,
    4096 intervals (4097 samples)."""
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05, pol=(1.0, 0.0))
    n = n_cycles * MEASUREMENTS_PER_CYCLE
    p = api.cosine_pulse(1.0, n_cycles, n, energy_scale=1.0 / omega)
    return Workload("dirac2d_64x64_4cyc", sys, [p], api.grid_tensor(n_grid, n_grid, -2, 2, -2, 2),
                    dict(abs_tol=1e-10, rel_tol=1e-10), dirac2d_64.__doc__)


def piflux2d_256(n_grid=256, n_cycles=8, omega=0.05, amplitude=1.0) -> Workload:
    """Square-lattice pi-flux, d = -2t(cos kx, cos ky, 0), t = 1, full BZ
    [-pi,pi]^2 on a 256x256 GL grid, omega = 0.05, 8 cycles, field along
    (1,1)/sqrt2, A0 = 1; window [0, 2 pi (n_cyc + 1)] as the reference's
    PiFlux dispatcher (PiFluxDispatcher.cpp:53), 8192 intervals, RKF78 with
    the reference tolerances 1e-12 / 1e-8."""
    s = 1.0 / math.sqrt(2.0)
    sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
    n = n_cycles * MEASUREMENTS_PER_CYCLE
    p = api.cosine_pulse(amplitude, n_cycles, n, window=(0.0, 2 * math.pi * (n_cycles + 1)),
                         energy_scale=1.0 / omega)
    return Workload("piflux2d_256x256_8cyc", sys, [p],
                    api.grid_tensor(n_grid, n_grid, -math.pi, math.pi, -math.pi, math.pi),
                    dict(abs_tol=1e-12, rel_tol=1e-8), piflux2d_256.__doc__)


def honeycomb_512(n_grid=512, n_cycles=6, omega=0.08) -> Workload:
    """Honeycomb NN hopping t = 1 with staggered mass 0.1, 512x512 GL over the
    rhombic BZ, 6 cycles, omega = 0.08, A0 ~ U[0.5, 1.5] from the seed, field
    along x, window [0, 2 pi (n_cyc + 1)] (HoneycombDispatcher.cpp:33-36)."""
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1, pol=(1.0, 0.0))
    a0 = 0.5 + splitmix64_uniforms(1)[0]
    n = n_cycles * MEASUREMENTS_PER_CYCLE
    p = api.cosine_pulse(a0, n_cycles, n, window=(0.0, 2 * math.pi * (n_cycles + 1)),
                         energy_scale=1.0 / omega)
    return Workload("honeycomb_rhombic_512x512_6cyc", sys, [p], api.grid_rhombic(n_grid, n_grid),
                    dict(abs_tol=1e-12, rel_tol=1e-8), honeycomb_512.__doc__)


def dirac2d_sweep(n_pulses=256, n_grid=128) -> Workload:
    """256 pulses on the gapped Dirac model, 128x128 grid: A0 log-uniform in
    [0.1, 2], phi ~ U[0, 2 pi), n_cyc ~ U[2, 10] (continuous, 1024 samples per
    cycle, rounded), omega ~ U[0.05, 0.15]."""
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05, pol=(1.0, 0.0))
    u = splitmix64_uniforms(4 * n_pulses).reshape(n_pulses, 4)
    pulses = []
    for i in range(n_pulses):
        a0 = math.exp(math.log(0.1) + u[i, 0] * (math.log(2.0) - math.log(0.1)))
        phi = 2 * math.pi * u[i, 1]
        ncyc = 2.0 + 8.0 * u[i, 2]
        omega = 0.05 + 0.1 * u[i, 3]
        n = int(round(MEASUREMENTS_PER_CYCLE * ncyc))
        pulses.append(api.cosine_pulse(a0, ncyc, n, phase=phi, energy_scale=1.0 / omega))
    return Workload("dirac2d_sweep_256x128x128", sys, pulses,
                    api.grid_tensor(n_grid, n_grid, -2, 2, -2, 2),
                    dict(abs_tol=1e-10, rel_tol=1e-10), dirac2d_sweep.__doc__)


def honeycomb_1024x64(n_pulses=64, n_grid=1024, n_cycles=6, omega=0.08) -> Workload:
    """Honeycomb + mass 0.1, 1024x1024 rhombic GL x 64 pulses: A0 ~ U[0.5, 2],
    phi ~ U[0, 2 pi); omega = 0.08 and 6 cycles as the 512x512 workload."""
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1, pol=(1.0, 0.0))
    u = splitmix64_uniforms(2 * n_pulses, SEED + 5).reshape(n_pulses, 2)
    n = n_cycles * MEASUREMENTS_PER_CYCLE
    pulses = [api.cosine_pulse(0.5 + 1.5 * u[i, 0], n_cycles, n, phase=2 * math.pi * u[i, 1],
                               window=(0.0, 2 * math.pi * (n_cycles + 1)),
                               energy_scale=1.0 / omega) for i in range(n_pulses)]
    return Workload("honeycomb_rhombic_1024x1024x64", sys, pulses,
                    api.grid_rhombic(n_grid, n_grid), dict(abs_tol=1e-12, rel_tol=1e-8),
                    honeycomb_1024x64.__doc__)


# params.config's material with the cosine laser (the reference ships that
# file with laser_type powerlaw1, which has no device form yet)
PIFLUX_PRODUCTION_CONFIG = """\
T 300
E_F 118
v_F 1.5e6
band_width 300
field_amplitude 1.6
photon_energy 5.25
diagonal_relaxation_time 15
offdiagonal_relaxation_time -1
laser_type cosine
n_laser_cycles {n_cycles}
t0_offset 0
system_type PiFlux
"""


def piflux3d_relax(n_cycles=16) -> Workload:
    """The reference's production PiFlux run: T = 300 K, E_F = 118 meV,
    v_F = 1.5e6 m/s, band width 300 meV, photon energy 5.25 meV, field
    1.6 MV/cm, diagonal relaxation time 15 fs (off-diagonal -> diagonal),
    cosine laser, 16 cycles, 1024 intervals per cycle over the pulse plus one
    relaxation cycle, on the reference's continuum-limit grid (z_range 32,
    N_coarse 4: 151 552 k-points); FP64 RKF78 1e-12 / 1e-8 with the reference
    step schedule (the relaxation right-hand side reads the step's start
    state, so the schedule is part of the result)."""
    from . import config
    run = config.from_config(PIFLUX_PRODUCTION_CONFIG.format(n_cycles=n_cycles))
    return Workload(f"piflux3d_relax_ref_{n_cycles}cyc", run.system, [run.pulse], run.grid,
                    dict(abs_tol=1e-12, rel_tol=1e-8), piflux3d_relax.__doc__)


def piflux3d_field(n_cycles=4) -> Workload:
    """The production PiFlux material and field without relaxation (the
    coherent path, thermal start at 300 K): the field drives 2t|d| to ~300
    hbar omega, so an interval takes several RKF78 steps and the step size
    follows the pulse (the workload a step proposer is for); reference
    continuum grid, 1024 intervals per cycle plus one relaxation cycle."""
    from . import config
    cfg = PIFLUX_PRODUCTION_CONFIG.format(n_cycles=n_cycles).replace(
        "diagonal_relaxation_time 15", "diagonal_relaxation_time -1")
    run = config.from_config(cfg)
    return Workload(f"piflux3d_field_ref_{n_cycles}cyc", run.system, [run.pulse], run.grid,
                    dict(abs_tol=1e-12, rel_tol=1e-8), piflux3d_field.__doc__)


# experiment.config's material (v_F 1e5 m/s, band width 200 meV, n_z 60) on
# the Dirac system with the cosine laser of params.config's photon energy at
# 0.1 MV/cm (A0 = 24 in the system's momentum units)
DIRAC_CONFIG = """\
T 300
E_F 118
v_F 1e5
band_width 200
field_amplitude 0.1
photon_energy 5.25
diagonal_relaxation_time -1
laser_type cosine
n_laser_cycles {n_cycles}
t0_offset 0
n_z 60
system_type Dirac
"""


@dataclass
class DiracWorkload:
    name: str
    system: api.SystemDesc
    pulse: api.PulseDesc
    quad: api.KappaQuad
    opts: api.SolverOpts
    description: str


def dirac3d_kappa(n_cycles=8, relax=False) -> DiracWorkload:
    """The reference's Dirac run (DiracDispatcher::compute ->
    DiracSystem::compute_current_density, coherent: the closed-form Magnus
    step per interval): T = 300 K, E_F = 118 meV, v_F = 1e5 m/s, band width
    200 meV (max_k = 200), photon energy 5.25 meV, 0.1 MV/cm, cosine laser,
    8 cycles (8192 intervals); 59 k_z slices x 100 splits of the kappa range,
    first trapezoids of 10 panels, halved until the elementwise change is
    below 1e-3 (DiracDispatcher.cpp:13-14)."""
    from . import config
    cfg = DIRAC_CONFIG.format(n_cycles=n_cycles)
    if relax:
        # the reference's configs set a relaxation time: its production path
        # (compute_current_density_diagonal_relaxation, FP64 RKF78)
        cfg = cfg.replace("diagonal_relaxation_time -1", "diagonal_relaxation_time 15")
    run = config.from_config(cfg)
    name = f"dirac3d_kappa{'_relax' if relax else ''}_nz60_{n_cycles}cyc"
    return DiracWorkload(name, run.system, run.pulse, run.quad, run.opts, dirac3d_kappa.__doc__)


ALL = {
    "dirac2d_64": dirac2d_64,
    "piflux2d_256": piflux2d_256,
    "honeycomb_512": honeycomb_512,
    "dirac2d_sweep": dirac2d_sweep,
    "honeycomb_1024x64": honeycomb_1024x64,
    "piflux3d_relax": piflux3d_relax,
    "dirac3d_kappa": dirac3d_kappa,
    "dirac3d_kappa_relax": lambda n_cycles=8: dirac3d_kappa(n_cycles, relax=True),
    "piflux3d_field": piflux3d_field,
}
