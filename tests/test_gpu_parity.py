"""GPU path (through the C ABI) against the CPU oracle on identical Gauss
nodes, weights and pulses.

Bar for the plain FP64 RKF78 path: j(t) relative L2 <= 1e-9 and harmonic
intensities within 1e-6 relative above the noise floor (harmonics within 60 dB
of the strongest).  Sizes are chosen so the oracle finishes in seconds.
"""
import math

import numpy as np
import pytest

from higherharmonics_b200 import api
from oracle import hhg_oracle as O
from tests.helpers import harmonic_rel_err, harmonics, oracle_args, oracle_j, rel_l2

pytestmark = pytest.mark.gpu

J_TOL = 1e-9
H_TOL = 1e-6


def _parity(engine, sys, pulse, grid, abs_tol, rel_tol, **okw):
    rows = api.grid_rows(sys, grid)
    j_gpu, st = engine.current_density(sys, pulse, grid, api.solver(abs_tol, rel_tol, **okw))
    j_ref, ost = oracle_j(sys, pulse, rows, abs_tol, rel_tol)
    err = rel_l2(j_gpu, j_ref)
    herr = harmonic_rel_err(harmonics(j_gpu, pulse), harmonics(j_ref, pulse))
    return j_gpu, j_ref, st, ost, err, herr


def test_dirac2d_parity(engine):
    # the 64x64 workload's physics on a 16x16 grid, full 4-cycle pulse
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 4, 4096, energy_scale=10.0)
    grid = api.grid_tensor(16, 16, -2, 2, -2, 2)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-10, 1e-10)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr
    assert st.attempted_steps == ost.attempted
    assert st.failed_trajectories == 0


def test_piflux2d_parity(engine):
    s = 1 / math.sqrt(2)
    sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
    pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=20.0)
    grid = api.grid_tensor(16, 16, -math.pi, math.pi, -math.pi, math.pi)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-12, 1e-8)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr
    assert abs(st.attempted_steps - ost.attempted) <= 1e-3 * ost.attempted


def test_piflux2d_general_polarisation_parity(engine):
    sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(0.6, 0.8))
    pulse = api.cosine_pulse(0.9, 2, 2048, phase=0.3, window=(0.0, 6 * math.pi), energy_scale=10.0)
    grid = api.grid_tensor(12, 12, -math.pi, math.pi, -math.pi, math.pi)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-12, 1e-8)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_long_standard_schedule_parity(engine):
    # n_subdivisions = 2000 gives 6 steps per interval: the tabulated schedule
    # covers 5, the last one runs on the interpolants
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 1, 512, energy_scale=10.0, n_subdivisions=2000)
    grid = api.grid_tensor(8, 8, -2, 2, -2, 2)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-10, 1e-10)
    assert err <= J_TOL, err
    assert st.attempted_steps == ost.attempted


def test_piflux3d_reference_grid_parity(engine):
    # reference PiFlux with its continuum-limit grid (z_range = 2, N_coarse = 2)
    sys = api.system(api.SYS_PIFLUX3D, hopping=1.0)
    pulse = api.cosine_pulse(1.0, 1, 512, window=(0.0, 4 * math.pi))
    grid = api.grid_piflux3d_ref(2, 2)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-12, 1e-8)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_honeycomb_hex_reference_grid_parity(engine):
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, pol=(math.cos(0.3), math.sin(0.3)))
    pulse = api.cosine_pulse(0.8, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=4.0)
    grid = api.grid_honeycomb_hex_ref(8)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-12, 1e-8)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_honeycomb_rhombic_mass_parity(engine):
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1)
    pulse = api.cosine_pulse(1.2, 2, 2048, phase=0.7, window=(0.0, 6 * math.pi), energy_scale=12.5)
    grid = api.grid_rhombic(16, 16)
    j, jr, st, ost, err, herr = _parity(engine, sys, pulse, grid, 1e-12, 1e-8)
    assert err <= J_TOL, err
    assert herr <= H_TOL, herr


def test_dirac3d_explicit_rows_parity(engine):
    # reference DiracSystem sigma RHS on explicit (k_z, kappa) rows, weight k_z kappa/|k|
    rng = np.random.default_rng(3)
    rows = []
    for _ in range(64):
        kz, kap = rng.uniform(-1.5, 1.5), rng.uniform(0.05, 1.5)
        mk = math.hypot(kz, kap)
        rows.append([kz, kap, mk, kz * kap / mk, 0.0, 0.0, -1.0, 0.0])
    rows = np.array(rows)
    sys = api.system(api.SYS_DIRAC3D)
    pulse = api.cosine_pulse(0.5, 2, 1024)
    grid, keep = api.grid_explicit(rows)
    j, st = engine.current_density(sys, pulse, grid, api.solver(1e-12, 1e-8))
    jr, ost = oracle_j(sys, pulse, rows, 1e-12, 1e-8)
    assert rel_l2(j, jr) <= J_TOL


def test_magnus4_parity(engine):
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 2, 2048, energy_scale=10.0)
    grid = api.grid_tensor(8, 8, -2, 2, -2, 2)
    rows = api.grid_rows(sys, grid)
    opts = api.solver(stepper=api.STEPPER_MAGNUS4, magnus_substeps=4)
    j, st = engine.current_density(sys, pulse, grid, opts)
    jr, _ = oracle_j(sys, pulse, rows, 1e-12, 1e-8, stepper=1, magnus_substeps=4)
    assert rel_l2(j, jr) <= J_TOL


def test_spectrum_matches_oracle_fft(engine):
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 4, 4096, energy_scale=10.0)
    grid = api.grid_tensor(8, 8, -2, 2, -2, 2)
    j, _ = engine.current_density(sys, pulse, grid, api.solver(1e-10, 1e-10))
    fr, re, im = engine.spectrum(j, pulse.n_measurements, pulse.window_begin, pulse.window_end)
    fr0, re0, im0 = O.trapezoidal_fft(j, pulse.window_begin, pulse.window_end, pulse.n_measurements)
    assert np.allclose(fr, fr0, rtol=1e-14, atol=0)
    scale = np.abs(re0 + 1j * im0).max()
    assert np.max(np.abs((re + 1j * im) - (re0 + 1j * im0))) <= 1e-12 * scale


def test_deterministic(engine):
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 1, 1024, energy_scale=10.0)
    grid = api.grid_tensor(32, 32, -2, 2, -2, 2)
    a, _ = engine.current_density(sys, pulse, grid, api.solver(1e-10, 1e-10))
    b, _ = engine.current_density(sys, pulse, grid, api.solver(1e-10, 1e-10))
    assert np.array_equal(a, b)


def test_step_limit_status(engine):
    # an unreachable tolerance makes every attempt fail; the device loop stops
    # after max_failed_steps and reports HHG_STEP_LIMIT instead of spinning
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 1, 64, energy_scale=10.0)
    grid = api.grid_tensor(4, 4, -2, 2, -2, 2)
    opts = api.solver(1e-300, 0.0)
    opts.max_failed_steps = 3
    with pytest.raises(api.HHGError) as ei:
        engine.current_density(sys, pulse, grid, opts)
    assert ei.value.status == api.STEP_LIMIT
    # the context stays usable
    j, _ = engine.current_density(sys, pulse, grid, api.solver(1e-10, 1e-10))
    assert np.all(np.isfinite(j))


def test_batched_pulses_match_single(engine):
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulses = [api.cosine_pulse(0.3 + 0.2 * i, 1.5 + 0.5 * i, 1024 + 512 * i, phase=0.4 * i,
                               energy_scale=1 / (0.06 + 0.02 * i)) for i in range(4)]
    grid = api.grid_tensor(16, 16, -2, 2, -2, 2)
    jb, _ = engine.current_density(sys, pulses, grid, api.solver(1e-10, 1e-10))
    off = 0
    for p in pulses:
        js, _ = engine.current_density(sys, p, grid, api.solver(1e-10, 1e-10))
        seg = jb[off:off + p.n_measurements + 1]
        assert np.array_equal(seg, js)
        off += p.n_measurements + 1


def _spectrum_err(engine, sys, pulse, grid, opts, opts_ref):
    from higherharmonics_b200.analysis import (default_max_order, harmonic_intensities,
                                               harmonic_rel_err)
    j, st = engine.current_density(sys, pulse, grid, opts)
    jr, str_ = engine.current_density(sys, pulse, grid, opts_ref)
    a = engine.spectrum(j, pulse.n_measurements, pulse.window_begin, pulse.window_end)
    b = engine.spectrum(jr, pulse.n_measurements, pulse.window_begin, pulse.window_end)
    mo = default_max_order(b[0])
    return (harmonic_rel_err(harmonic_intensities(*a, mo), harmonic_intensities(*b, mo)),
            rel_l2(j, jr), st, str_)


@pytest.mark.parametrize("model", ["piflux2d", "honeycomb", "dirac2d"])
def test_fast_variants_meet_harmonic_bar(engine, model):
    """Mixed precision, the step proposers and the Magnus-4 stepper stay
    within the 1e-4 harmonic-intensity bar of the plain FP64 path."""
    if model == "piflux2d":
        s = 1 / math.sqrt(2)
        sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
        pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=20.0)
        grid = api.grid_tensor(64, 64, -math.pi, math.pi, -math.pi, math.pi)
        ref = api.solver(1e-12, 1e-8)
    elif model == "honeycomb":
        sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1)
        pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=12.5)
        grid = api.grid_rhombic(64, 64)
        ref = api.solver(1e-12, 1e-8)
    else:
        sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
        pulse = api.cosine_pulse(1.0, 4, 4096, energy_scale=10.0)
        grid = api.grid_tensor(32, 32, -2, 2, -2, 2)
        ref = api.solver(1e-10, 1e-10)
    for opts in (api.solver(ref.abs_tol, ref.rel_tol, proposer=api.PROPOSER_CARRY),
                 api.solver(ref.abs_tol, ref.rel_tol, proposer=api.PROPOSER_LOCKSTEP),
                 api.solver(1e-8, 1e-6, precision=api.PREC_MIXED),
                 api.solver(1e-8, 1e-6, precision=api.PREC_MIXED, proposer=api.PROPOSER_CARRY),
                 api.solver(1e-8, 1e-6, precision=api.PREC_MIXED, proposer=api.PROPOSER_LOCKSTEP),
                 # one two-point Magnus step (exact rotation) per measurement interval
                 api.solver(stepper=api.STEPPER_MAGNUS4, magnus_substeps=1)):
        herr, jerr, st, st_ref = _spectrum_err(engine, sys, pulse, grid, opts, ref)
        assert herr <= 1e-4, (opts.precision, opts.proposer, herr)
        assert jerr <= 1e-4, (opts.precision, opts.proposer, jerr)


@pytest.mark.parametrize("beta,ef", [(0.0, 0.0), (1.5, 0.3)])
def test_dirac3d_reference_magnus_parity(engine, beta, ef):
    # DiracSystem::time_evolution_magnus (DiracSystem.cpp:176-211): one closed-form
    # step per interval from the 30-point Legendre moments of A
    rng = np.random.default_rng(11)
    m = O.model(O.DIRAC3D, beta=beta, fermi_energy=ef)
    rows = []
    for _ in range(96):
        kz, kap = rng.uniform(-1.5, 1.5), rng.uniform(0.05, 1.5)
        mk = math.hypot(kz, kap)
        rows.append([kz, kap, mk, kz * kap / mk, *O.initial_state(m, kz, kap, mk), 0.0])
    rows = np.array(rows)
    sys = api.system(api.SYS_DIRAC3D, beta=beta, fermi_energy=ef)
    pulse = api.cosine_pulse(0.6, 2, 2048)
    grid, keep = api.grid_explicit(rows)
    j, st = engine.current_density(sys, pulse, grid, api.solver(stepper=api.STEPPER_DIRAC_MAGNUS))
    jr, ost = oracle_j(sys, pulse, rows, 1e-12, 1e-8, stepper=2)
    assert rel_l2(j, jr) <= 1e-12, rel_l2(j, jr)
    assert st.attempted_steps == ost.attempted == 96 * 2048


def test_dirac_magnus_refused_elsewhere(engine):
    pulse = api.cosine_pulse(0.6, 1, 64)
    grid = api.grid_tensor(4, 4, -1, 1, -1, 1)
    with pytest.raises(api.HHGError) as ei:
        engine.current_density(api.system(api.SYS_DIRAC2D, velocity=1.0), pulse, grid,
                               api.solver(stepper=api.STEPPER_DIRAC_MAGNUS))
    assert ei.value.status == api.UNSUPPORTED


def test_full_size_symmetries(engine):
    # the benchmark's own size (PiFlux-2D 256^2, 8 cycles, 8192 intervals),
    # beyond the oracle's reach, through properties the physics fixes: the
    # lattice is centrosymmetric (cos even), so (k, A) -> (-k, -A) leaves
    # every trajectory unchanged and flips the current vertex: j[-A] = -j[A]
    # up to the order of the BZ sum (this is what removes even harmonics);
    # without a field the start state is stationary and j = 0
    from higherharmonics_b200 import workloads as W
    wl = W.piflux2d_256()
    p = wl.pulses[0]
    opts = wl.opts()
    jp, sp = engine.current_density(wl.system, p, wl.grid, opts)
    pm = api.cosine_pulse(-p.amplitude, p.n_cycles, p.n_measurements,
                          window=(p.window_begin, p.window_end), energy_scale=p.energy_scale)
    jm, sm = engine.current_density(wl.system, pm, wl.grid, opts)
    assert sp.failed_trajectories == 0 and sm.failed_trajectories == 0
    scale = np.max(np.abs(jp))
    assert scale > 0 and np.max(np.abs(jp + jm)) <= 1e-10 * scale, np.max(np.abs(jp + jm)) / scale
    assert abs(sp.attempted_steps - sm.attempted_steps) <= 1e-6 * sp.attempted_steps
    p0 = api.cosine_pulse(0.0, p.n_cycles, p.n_measurements,
                          window=(p.window_begin, p.window_end), energy_scale=p.energy_scale)
    j0, _ = engine.current_density(wl.system, p0, wl.grid, opts)
    assert np.max(np.abs(j0)) <= 1e-12 * scale
