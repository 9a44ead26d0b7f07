"""The Dirac-3D momentum quadrature on the GPU (hhg_gpu_dirac_current_density,
through the C ABI) against the oracle's restatement.

Reference: DiracSystem::compute_current_density (DiracSystem.cpp:271-331) and
compute_current_density_diagonal_relaxation (:365-425), called by
DiracDispatcher::compute (DiracDispatcher.cpp:65-80): k_z slices times the
adaptive trapezoidal kappa rule (restated from the reference's call, its
library being unavailable; see tests/test_oracle_kappa.py).  Bar: the same
refinement (rounds, levels, nodes) as the oracle, and j(t) relative L2
<= 1e-12 for the closed-form Magnus path (no step control), 1e-9 for RKF78.
The debug traces (DiracSystem.cpp:333-363, 427-457) are held to the same bars
trajectory by trajectory.
"""
import math

import numpy as np
import pytest

from higherharmonics_b200 import api, config, runmodes
from oracle import hhg_oracle as O
from tests.helpers import oracle_args, rel_l2

pytestmark = pytest.mark.gpu


def _system(beta=0.0, fermi=0.0, relax=0.0):
    return api.system(api.SYS_DIRAC3D, beta=beta, fermi_energy=fermi, inv_diag_relax=relax)


def _oracle(sys, pulse, quad, stepper):
    m, p, tc, s = oracle_args(sys, pulse, 1e-12, 1e-8, stepper=stepper)
    return O.dirac_kappa_current(m, p, tc, s, max_k=quad.max_k, n_z=quad.n_z,
                                 n_kappa=quad.n_kappa, threshold=quad.threshold,
                                 n_splits=quad.n_splits, max_halvings=quad.max_halvings or 12)


def _same_refinement(qs, info):
    assert (qs.rounds, qs.unconverged, qs.max_level, qs.trajectories) == \
        (info["rounds"], info["unconverged"], info["max_level"], info["trajectories"])


def test_magnus_parity(engine):
    sys, pulse = _system(), api.cosine_pulse(0.6, 1, 256)
    quad = api.kappa_quad(2.5, 8, n_kappa=4, threshold=1e-5, n_splits=5, max_halvings=8)
    j, qs, st = engine.dirac_current_density(sys, pulse, quad)
    jr, info, rc = _oracle(sys, pulse, quad, api.STEPPER_DIRAC_MAGNUS)
    assert rc == 0 and st.failed_trajectories == 0
    assert qs.splits == 6 * 5  # n_z = 8: z = 1 .. 7 without 4
    _same_refinement(qs, info)
    # splits stop at different levels
    uniform = qs.splits * (5 + 4 * ((1 << qs.max_level) - 1))
    assert qs.max_level >= 3 and qs.trajectories < uniform
    # a small problem: later levels are integrated ahead of the convergence
    # test (fewer launches than levels, discarded rows), same result
    assert qs.launches < qs.rounds and qs.speculative > 0
    assert rel_l2(j, jr) <= 1e-12, rel_l2(j, jr)


def test_thermal_magnus_parity(engine):
    sys, pulse = _system(beta=3.0, fermi=0.4), api.gauss_pulse(0.5, 1, 256)
    quad = api.kappa_quad(2.0, 7, n_kappa=3, threshold=1e-5, n_splits=4, max_halvings=8)
    j, qs, _ = engine.dirac_current_density(sys, pulse, quad)
    jr, info, rc = _oracle(sys, pulse, quad, api.STEPPER_DIRAC_MAGNUS)
    assert rc == 0 and qs.splits == 5 * 4  # odd n_z: z = 1 .. 6 without 3
    _same_refinement(qs, info)
    assert rel_l2(j, jr) <= 1e-12, rel_l2(j, jr)


@pytest.mark.parametrize("relax", [0.0, 0.2])
def test_rkf78_parity(engine, relax):
    # the sigma equation (time_evolution_sigma) and the diagonal relaxation
    # path (time_evolution_diagonal_relaxation), both FP64 RKF78
    sys, pulse = _system(beta=2.0, fermi=0.2, relax=relax), api.cosine_pulse(0.5, 1, 128)
    quad = api.kappa_quad(1.5, 6, n_kappa=3, threshold=1e-4, n_splits=3, max_halvings=6)
    j, qs, st = engine.dirac_current_density(sys, pulse, quad, api.solver(1e-12, 1e-8))
    jr, info, rc = _oracle(sys, pulse, quad, api.STEPPER_RKF78)
    assert rc == 0 and st.failed_trajectories == 0 and st.attempted_steps > 0
    _same_refinement(qs, info)
    assert rel_l2(j, jr) <= 1e-9, rel_l2(j, jr)


def test_odd_in_the_field_at_size(engine):
    # even n_z and a T = 0 start: (k_z, A) -> (-k_z, -A) maps the trajectories
    # onto each other with the weight's sign flipped, so j(-A) = -j(A) with
    # the same refinement; at the reference's n_kappa, threshold and splits
    quad = api.kappa_quad(2.5, 40, n_kappa=10, threshold=1e-6, n_splits=100)
    jp, qp, _ = engine.dirac_current_density(_system(), api.cosine_pulse(0.6, 2, 2048), quad)
    jm, qm, _ = engine.dirac_current_density(_system(), api.cosine_pulse(-0.6, 2, 2048), quad)
    assert qp.as_dict() == qm.as_dict() and qp.unconverged == 0 and qp.rounds >= 2
    assert np.max(np.abs(jp + jm)) <= 1e-12 * np.max(np.abs(jp))
    # no field: the equilibrium is stationary and the k_z-odd weights cancel
    j0, q0, _ = engine.dirac_current_density(_system(), api.cosine_pulse(0.0, 2, 2048), quad)
    assert np.max(np.abs(j0)) <= 1e-12 * np.max(np.abs(jp))


DIRAC_CFG = """
T 0
E_F 0
v_F 1e5
band_width 3
field_amplitude 0.5
photon_energy 5
diagonal_relaxation_time -1
laser_type cosine
n_laser_cycles 1
t0_offset 0
n_z 6
occupations no
split_current no
debug_data no
system_type Dirac
"""


def test_dirac_config_end_to_end(engine):
    doc = runmodes.current_density(engine, config.read_config(DIRAC_CFG), n_measurements=128)
    run = config.from_config(DIRAC_CFG, n_measurements=128)
    jr, info, rc = _oracle(run.system, run.pulse, run.quad, api.STEPPER_DIRAC_MAGNUS)
    assert rc == 0
    j = np.array(doc["current_density_time"])
    assert rel_l2(j, jr) <= 1e-12 and np.max(np.abs(jr)) > 0
    assert len(doc["frequencies"]) == len(doc["current_density_frequency_real"])


@pytest.mark.parametrize("relax", [False, True])
def test_dirac_debug_traces(engine, relax):
    # DiracSystem::compute_current_density_debug and its relaxation twin
    # (DiracSystem.cpp:333-363, 427-457): the weighted current of 25 (k_z, kappa)
    # trajectories at picked_z = n_z/2 + n_z/10, each transformed without padding
    text = DIRAC_CFG.replace("debug_data no", "debug_data yes").replace("n_z 6", "n_z 20")
    if relax:
        text = text.replace("diagonal_relaxation_time -1", "diagonal_relaxation_time 20")
    cfg = config.read_config(text)
    n = 128
    doc = runmodes.debug_traces(engine, cfg, n_measurements=n)
    run = config.from_config(cfg, n_measurements=n)
    rows = api.grid_rows(run.system, api.grid_dirac3d_debug(run.quad.n_z, run.quad.max_k))
    stepper = api.STEPPER_RKF78 if relax else api.STEPPER_DIRAC_MAGNUS
    m, p, tc, s = oracle_args(run.system, run.pulse, 1e-12, 1e-8, stepper=stepper)
    tr = np.array(doc["time_evolutions"])
    assert tr.shape == (api.N_DEBUG_POINTS, n + 1)
    for i in range(api.N_DEBUG_POINTS):
        ref, _, rc = O.current_density(m, p, tc, s, rows[i:i + 1])
        assert rc == 0 and np.ptp(ref) > 0
        assert rel_l2(tr[i], ref) <= (1e-9 if relax else 1e-12), i
    pl = run.pulse
    me = (pl.window_end - pl.window_begin) / n
    _, rre, rim = O.trapezoidal_fft_unpadded(tr[7], me, pl.window_begin, pl.window_end)
    got = np.array(doc["debug_fft_real"][7]) + 1j * np.array(doc["debug_fft_imag"][7])
    assert np.max(np.abs(got - (rre + 1j * rim))) <= 1e-13 * np.abs(rre + 1j * rim).max()


def test_refusals(engine):
    pulse = api.cosine_pulse(0.5, 1, 64)
    quad = api.kappa_quad(2.0, 6, n_kappa=2, n_splits=2)
    cases = [
        (api.system(api.SYS_DIRAC2D, velocity=1.0), quad, None, api.UNSUPPORTED),
        (_system(), quad, api.solver(proposer=api.PROPOSER_CARRY), api.UNSUPPORTED),
        (_system(), quad, api.solver(1e-8, 1e-6, precision=api.PREC_MIXED), api.UNSUPPORTED),
        (_system(relax=0.1), quad, api.solver(stepper=api.STEPPER_DIRAC_MAGNUS), api.UNSUPPORTED),
        (_system(), api.kappa_quad(2.0, 2), None, api.BAD_CONFIG),
        (_system(), api.kappa_quad(2.0, 6, threshold=0.0), None, api.BAD_CONFIG),
        (_system(), api.kappa_quad(2.0, 6, n_kappa=1 << 20, max_halvings=12), None, api.BAD_CONFIG),
    ]
    for sys, q, opts, status in cases:
        with pytest.raises(api.HHGError) as ei:
            engine.dirac_current_density(sys, pulse, q, opts)
        assert ei.value.status == status, (ei.value, status)


def test_repeated_calls_reuse_state_exactly(engine):
    # the context keeps the quadrature's plan and buffers between calls; a
    # different quadrature, a different pulse and a return to the first
    # give the same results as fresh calls
    sys = _system()
    p1, p2 = api.cosine_pulse(0.6, 1, 256), api.cosine_pulse(0.4, 1, 128)
    q1 = api.kappa_quad(2.5, 8, n_kappa=4, threshold=1e-5, n_splits=5, max_halvings=8)
    q2 = api.kappa_quad(2.0, 12, n_kappa=6, threshold=1e-6, n_splits=7)
    a, qa, _ = engine.dirac_current_density(sys, p1, q1)
    b, qb, _ = engine.dirac_current_density(sys, p1, q2)
    c, _, _ = engine.dirac_current_density(sys, p2, q1)
    a2, qa2, _ = engine.dirac_current_density(sys, p1, q1)
    assert np.array_equal(a, a2) and qa.as_dict() == qa2.as_dict()
    fresh = api.Engine(0)
    try:
        for (p, q, want) in ((p1, q2, b), (p2, q1, c)):
            j, _, _ = fresh.dirac_current_density(sys, p, q)
            assert np.array_equal(j, want)
    finally:
        fresh.close()


def test_slice_blocks_add_up(engine):
    # the reference's MPI partition of the z loop (DiracSystem.cpp:288-295):
    # per-rank blocks, each with its factor dz, sum to the whole current
    from higherharmonics_b200.distributed import dirac_z_block
    sys, pulse = _system(beta=1.0, fermi=0.2), api.cosine_pulse(0.6, 1, 128)
    base = dict(max_k=2.5, n_z=9, n_kappa=4, threshold=1e-5, n_splits=3, max_halvings=6)
    full, qf, _ = engine.dirac_current_density(sys, pulse, api.kappa_quad(**base))
    parts, traj = [], 0
    for r in range(3):
        zf, zc = dirac_z_block(9, r, 3)
        j, q, _ = engine.dirac_current_density(sys, pulse,
                                               api.kappa_quad(**base, z_first=zf, z_count=zc))
        parts.append(j)
        traj += q.trajectories
    assert traj == qf.trajectories
    assert np.max(np.abs(sum(parts) - full)) <= 1e-13 * np.max(np.abs(full))
    # a block holding only the weight-0 slice z = n_z / 2
    j0, q0, _ = engine.dirac_current_density(sys, pulse, api.kappa_quad(**base, z_first=4, z_count=1))
    assert not j0.any() and q0.trajectories == 0
    for zf, zc in ((0, 2), (8, 2), (3, -1)):
        with pytest.raises(api.HHGError) as ei:
            engine.dirac_current_density(sys, pulse, api.kappa_quad(**base, z_first=zf, z_count=zc))
        assert ei.value.status == api.BAD_CONFIG
