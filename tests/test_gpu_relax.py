"""Relaxation-time right-hand sides and thermal initial states on the GPU
(through the C ABI) against the CPU oracle, same nodes, weights and pulses.

Bar for the FP64 RKF78 path: j(t) relative L2 <= 1e-9 and harmonic
intensities within 1e-6 relative above the noise floor, as for the coherent
path; the step proposers are held to the 1e-4 harmonic bar against the
reference schedule.  Reference forms: PiFlux.cpp:113-220,
Honeycomb.cpp:160-212, DiracSystem.cpp:213-251.
"""
import math

import numpy as np
import pytest

from higherharmonics_b200 import api
from tests.helpers import harmonic_rel_err, harmonics, oracle_j, rel_l2

pytestmark = pytest.mark.gpu

J_TOL = 1e-9
H_TOL = 1e-6


def fermi(e, beta):
    if beta == 0.0:
        return 1.0 if e < 0 else (0.0 if e > 0 else 0.5)
    return 1.0 / (1.0 + math.exp(beta * e))


def _parity(engine, sys, pulse, grid, rows=None, abs_tol=1e-12, rel_tol=1e-8):
    if rows is None:
        rows = api.grid_rows(sys, grid)
    j, st = engine.current_density(sys, pulse, grid, api.solver(abs_tol, rel_tol))
    jr, ost = oracle_j(sys, pulse, rows, abs_tol, rel_tol)
    assert st.failed_trajectories == 0
    return rel_l2(j, jr), harmonic_rel_err(harmonics(j, pulse), harmonics(jr, pulse)), st, ost


def test_piflux3d_relaxation_finite_temperature(engine):
    # PiFlux with its reference grid, T > 0, E_F != 0 and unequal rates
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=2.0, fermi_energy=0.5,
                     inv_diag_relax=0.8, inv_offdiag_relax=1.3)
    pulse = api.cosine_pulse(1.0, 1, 512, window=(0.0, 4 * math.pi))
    err, herr, st, ost = _parity(engine, sys, pulse, api.grid_piflux3d_ref(2, 2))
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr
    assert abs(st.attempted_steps - ost.attempted) <= 1e-3 * ost.attempted


def test_piflux3d_relaxation_zero_temperature(engine):
    # T = 0: the off-diagonal equilibrium term vanishes (2 sqrt(a2 b2) = 0)
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, inv_diag_relax=1.5, inv_offdiag_relax=1.5)
    pulse = api.cosine_pulse(1.2, 1, 512, window=(0.0, 4 * math.pi))
    err, herr, st, ost = _parity(engine, sys, pulse, api.grid_piflux3d_ref(2, 2))
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_piflux3d_coherent_finite_temperature(engine):
    # thermal initial state with the coherent right-hand side
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=1.2, fermi_energy=-0.4)
    pulse = api.cosine_pulse(1.0, 1, 512, window=(0.0, 4 * math.pi))
    err, herr, _, _ = _parity(engine, sys, pulse, api.grid_piflux3d_ref(2, 2))
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_piflux3d_relaxation_rescue_rows(engine):
    # cos kx = cos ky = 0 (is_zero) with cos(kz - A) < 0: the equilibrium
    # momentum takes RESCUE_TRAFO (PiFlux.cpp:135-139); without it the
    # equilibrium state is 0/0.  The other rows start from the thermal state:
    # the equilibrium's off-diagonal direction is the start state's component
    # perpendicular to the band axis, normalised (PiFlux.cpp:145-147), which a
    # state on the axis (the T = 0 state at T > 0) leaves to rounding noise.
    from oracle import hhg_oracle as O
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=1.5, fermi_energy=0.3,
                     inv_diag_relax=0.6, inv_offdiag_relax=0.9)
    m = O.model(O.PIFLUX3D, hopping=1.0, beta=1.5, fermi_energy=0.3)
    h = math.pi / 2
    rows = []
    for kz in (2.6, 3.0, -2.8):
        s0 = np.array([0.3, -0.2, 0.9])
        s0 /= np.linalg.norm(s0)
        rows.append([h, h, kz, 0.7, *s0, 0.0])
    rng = np.random.default_rng(5)
    for _ in range(29):
        kx, ky, kz = rng.uniform(0.1, 3.0, 3)
        rows.append([kx, ky, kz, rng.uniform(0.1, 1.0), *O.initial_state(m, kx, ky, kz), 0.0])
    rows = np.array(rows)
    pulse = api.cosine_pulse(0.8, 1, 512, window=(0.0, 4 * math.pi))
    grid, keep = api.grid_explicit(rows)
    err, herr, _, _ = _parity(engine, sys, pulse, grid, rows=rows)
    assert err <= J_TOL, err


def test_honeycomb_relaxation_finite_temperature(engine):
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, pol=(math.cos(0.3), math.sin(0.3)),
                     beta=3.0, fermi_energy=0.4, inv_diag_relax=0.5)
    pulse = api.cosine_pulse(0.8, 1, 1024, window=(0.0, 4 * math.pi), energy_scale=4.0)
    err, herr, _, _ = _parity(engine, sys, pulse, api.grid_honeycomb_hex_ref(8))
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_dirac3d_relaxation_finite_temperature(engine):
    beta, ef, rate = 1.5, 0.3, 0.7
    rng = np.random.default_rng(3)
    rows = []
    for _ in range(64):
        kz, kap = rng.uniform(-1.5, 1.5), rng.uniform(0.05, 1.5)
        mk = math.hypot(kz, kap)
        a0, b0 = fermi(ef + mk, beta), fermi(ef - mk, beta)
        rows.append([kz, kap, mk, kz * kap / mk, 2 * a0 * b0, 0.0, a0 * a0 - b0 * b0, 0.0])
    rows = np.array(rows)
    sys = api.system(api.SYS_DIRAC3D, beta=beta, fermi_energy=ef, inv_diag_relax=rate)
    pulse = api.cosine_pulse(0.5, 2, 1024)
    grid, keep = api.grid_explicit(rows)
    err, _, _, _ = _parity(engine, sys, pulse, grid, rows=rows)
    assert err <= J_TOL, err


@pytest.mark.parametrize("model", ["honeycomb", "piflux3d_t0", "dirac3d"])
def test_relaxation_step_proposers_meet_harmonic_bar(engine, model):
    from higherharmonics_b200.analysis import (default_max_order, harmonic_intensities,
                                               harmonic_rel_err as herr_fn)
    if model == "honeycomb":
        sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, pol=(math.cos(0.3), math.sin(0.3)),
                         beta=3.0, fermi_energy=0.4, inv_diag_relax=0.5)
        pulse = api.cosine_pulse(0.8, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=4.0)
        grid = api.grid_honeycomb_hex_ref(16)
    elif model == "piflux3d_t0":
        sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, inv_diag_relax=0.8, inv_offdiag_relax=1.1)
        pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi))
        grid = api.grid_piflux3d_ref(4, 2)
    else:
        rows = []
        for kz in np.linspace(-1.4, 1.4, 16):
            for kap in np.linspace(0.1, 1.4, 16):
                mk = math.hypot(kz, kap)
                a0, b0 = fermi(0.3 + mk, 1.5), fermi(0.3 - mk, 1.5)
                rows.append([kz, kap, mk, kz * kap / mk, 2 * a0 * b0, 0.0, a0 * a0 - b0 * b0, 0.0])
        sys = api.system(api.SYS_DIRAC3D, beta=1.5, fermi_energy=0.3, inv_diag_relax=0.7)
        pulse = api.cosine_pulse(0.5, 2, 2048)
        grid, keep = api.grid_explicit(np.array(rows))
    ref = api.solver(1e-12, 1e-8)
    jr, st_ref = engine.current_density(sys, pulse, grid, ref)
    b = engine.spectrum(jr, pulse.n_measurements, pulse.window_begin, pulse.window_end)
    mo = default_max_order(b[0])
    for prop in (api.PROPOSER_CARRY, api.PROPOSER_LOCKSTEP):
        j, st = engine.current_density(sys, pulse, grid, api.solver(1e-12, 1e-8, proposer=prop))
        a = engine.spectrum(j, pulse.n_measurements, pulse.window_begin, pulse.window_end)
        assert herr_fn(harmonic_intensities(*a, mo), harmonic_intensities(*b, mo)) <= 1e-4, prop
        assert rel_l2(j, jr) <= 1e-4, prop
        assert st.attempted_steps < st_ref.attempted_steps, prop


def test_relaxation_rejects_unsupported_solvers(engine):
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0, inv_diag_relax=1.0, inv_offdiag_relax=1.0)
    pulse = api.cosine_pulse(1.0, 1, 64, window=(0.0, 4 * math.pi))
    grid = api.grid_piflux3d_ref(1, 1)
    for opts in (api.solver(precision=api.PREC_MIXED),
                 api.solver(stepper=api.STEPPER_MAGNUS4, magnus_substeps=2)):
        with pytest.raises(api.HHGError) as ei:
            engine.current_density(sys, pulse, grid, opts)
        assert ei.value.status == api.UNSUPPORTED
    # PiFlux at T > 0: the frozen start state ties j(t) to the reference schedule
    warm = api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=1.0, inv_diag_relax=1.0, inv_offdiag_relax=1.0)
    with pytest.raises(api.HHGError) as ei:
        engine.current_density(warm, pulse, grid, api.solver(proposer=api.PROPOSER_CARRY))
    assert ei.value.status == api.UNSUPPORTED
    hsys = api.system(api.SYS_HONEYCOMB, hopping=1.0, inv_diag_relax=1.0)
    late = api.cosine_pulse(1.0, 1, 64, window=(1.0, 4 * math.pi))  # A(window_begin) != 0
    with pytest.raises(api.HHGError) as ei:
        engine.current_density(hsys, late, api.grid_honeycomb_hex_ref(2), api.solver())
    assert ei.value.status == api.UNSUPPORTED
    # the context stays usable
    j, _ = engine.current_density(sys, pulse, grid, api.solver())
    assert np.all(np.isfinite(j))
