"""Thermal initial states and relaxation-time right-hand sides: oracle
invariants, the host-built k rows of the C ABI against the oracle, and the
requests the ABI rejects (all on the CPU).

The reference's relaxation forms are PiFlux::time_evolution_diagonal_relaxation
(PiFlux.cpp:113-220), Honeycomb::time_evolution_diagonal_relaxation
(Honeycomb.cpp:160-212) and DiracSystem::time_evolution_diagonal_relaxation
(DiracSystem.cpp:213-251); the thermal initial states are their ic_sigma /
Fermi-occupied states (PiFlux.cpp:519-549, Honeycomb.cpp:347-361,
DiracSystem.cpp:155-158).
"""
import ctypes
import json
import math
import os

import numpy as np
import pytest

from higherharmonics_b200 import api
from oracle import hhg_oracle as O


def fermi(e, beta):
    if beta == 0.0:
        return 1.0 if e < 0 else (0.0 if e > 0 else 0.5)
    return 1.0 / (1.0 + math.exp(beta * e))


def test_zero_temperature_state_is_filled_lower_band():
    m = O.model(O.PIFLUX3D, hopping=1.0)
    rows = O.grid_piflux3d_ref(m, 2, 1)
    for r in rows[::37]:
        d = np.array([math.cos(r[0]), math.cos(r[1]), math.cos(r[2])])
        assert np.allclose(r[4:7], -d / np.linalg.norm(d), atol=1e-6)  # rescued cos_z slices differ by 5e-9
    m = O.model(O.HONEYCOMB, hopping=1.0)
    rows = O.grid_honeycomb_hex_ref(m, 4)
    assert np.allclose(np.linalg.norm(rows[:, 4:7], axis=1), 1.0, atol=1e-14)


@pytest.mark.parametrize("beta,ef", [(0.7, 0.3), (2.0, -1.1), (0.05, 0.0)])
def test_thermal_piflux_state_is_pure(beta, ef):
    # the reference's state alpha|upper> + beta|lower> has |S| = alpha^2 + beta^2
    t = 1.3
    m = O.model(O.PIFLUX3D, hopping=t, beta=beta, fermi_energy=ef)
    rows = O.grid_piflux3d_ref(m, 2, 1)
    for r in rows[::23]:
        cx, cy, cz = math.cos(r[0]), math.cos(r[1]), math.cos(r[2])
        if r[2] > 0 and cz < 0:
            cz *= 1 - 0.5e-8  # +k_z slices keep the rescued cos_z (PiFlux.cpp:826-829)
        disp = math.sqrt(cx * cx + cy * cy + cz * cz)
        a2 = fermi(-ef + 2 * t * disp, beta)
        b2 = fermi(-ef - 2 * t * disp, beta)
        assert abs(np.linalg.norm(r[4:7]) - (a2 + b2)) <= 1e-13


def test_thermal_piflux_state_matches_reference_derivation():
    """The oracle's PiFlux ic_sigma against tests/golden/piflux_ic.json: the
    expectation values of helper/piflux_initial_conditions.py (the state
    alpha|a> + beta|b> through the helper's V and normalisation), evaluated with
    sympy at seeded (t, beta_T, E_F, k), and the helper's closed form
    |<sigma(0)>|^2 = (alpha^2 + beta^2)^2."""
    path = os.path.join(os.path.dirname(__file__), "golden", "piflux_ic.json")
    pts = json.load(open(path))["points"]
    assert len(pts) >= 10
    for p in pts:
        m = O.model(O.PIFLUX3D, hopping=p["hopping"], beta=p["beta"],
                    fermi_energy=p["fermi_energy"])
        s0 = O.initial_state(m, *p["k"])
        assert np.max(np.abs(s0 - np.array(p["sigma"]))) <= 1e-13, p
        assert abs(float(s0 @ s0) - p["norm2"]) <= 1e-13
        assert abs(p["norm2"] - (p["alpha2"] + p["beta2"]) ** 2) <= 1e-13


@pytest.mark.parametrize("beta,ef", [(1.5, 0.4), (0.2, -0.5)])
def test_thermal_honeycomb_state(beta, ef):
    t = 0.9
    m = O.model(O.HONEYCOMB, hopping=t, beta=beta, fermi_energy=ef)
    rows = O.grid_honeycomb_hex_ref(m, 4)
    for r in rows[::7]:
        g = sum(np.exp(1j * (nx * r[0] + ny * r[1]))
                for nx, ny in ((1, 0), (-0.5, math.sqrt(3) / 2), (-0.5, -math.sqrt(3) / 2)))
        a2 = fermi(ef - t * abs(g), beta)
        b2 = fermi(ef + t * abs(g), beta)
        want = [-(a2 - b2) * g.real / abs(g), (a2 - b2) * g.imag / abs(g), -2 * math.sqrt(a2 * b2)]
        assert np.allclose(r[4:7], want, rtol=1e-13, atol=1e-15)


def _evolve(m, pulse, tc, row):
    states, st = O.evolve_k(m, pulse, tc, O.solver(1e-12, 1e-10), row)
    return states


def test_piflux_relaxation_stationary_without_field():
    # T = 0 and equal rates: r_d = -d_hat = S0, r_o = 0, so S0 is a fixed point
    m = O.model(O.PIFLUX3D, hopping=1.0, inv_diag_relax=0.9, inv_offdiag_relax=0.9)
    row = O.grid_piflux3d_ref(m, 2, 1)[11].copy()
    states = _evolve(m, O.Pulse(0.0, 1), O.time_config(0.0, 2 * math.pi, 64), row)
    assert np.max(np.abs(states - row[4:7])) <= 1e-12


def test_relaxation_returns_to_equilibrium_after_the_pulse():
    # one-cycle pulse, then 5 cycles of A = 0: the deviation from the
    # equilibrium decays as exp(-rate t)
    rate = 0.8
    tail = 10 * math.pi
    tc = O.time_config(0.0, 2 * math.pi + tail, 384)
    m = O.model(O.PIFLUX3D, hopping=1.0, inv_diag_relax=rate, inv_offdiag_relax=rate)
    row = O.grid_piflux3d_ref(m, 2, 1)[5].copy()
    s = _evolve(m, O.Pulse(1.0, 1), tc, row)
    mid = np.linalg.norm(s[64] - row[4:7])
    assert mid > 1e-3  # the pulse moved the state
    assert np.linalg.norm(s[-1] - row[4:7]) <= 1e-8 + math.exp(-rate * tail) * 10
    m = O.model(O.HONEYCOMB, hopping=1.0, inv_diag_relax=rate)
    row = O.grid_honeycomb_hex_ref(m, 4)[9].copy()
    s = _evolve(m, O.Pulse(1.0, 1), tc, row)
    assert np.linalg.norm(s[64] - row[4:7]) > 1e-3
    assert np.linalg.norm(s[-1] - row[4:7]) <= 1e-8 + math.exp(-rate * tail) * 10


def test_dirac_relaxation_towards_initial_state():
    kz, kap = 0.4, 0.7
    mk = math.hypot(kz, kap)
    m = O.model(O.DIRAC3D, inv_diag_relax=1.1)
    row = np.array([kz, kap, mk, 1.0, 0.0, 0.0, -1.0, 0.0])
    tail = 8 * math.pi
    s = _evolve(m, O.Pulse(0.6, 1), O.time_config(0.0, 2 * math.pi + tail, 512), row)
    assert np.linalg.norm(s[100] - row[4:7]) > 1e-4
    assert np.linalg.norm(s[-1] - row[4:7]) <= 1e-8 + math.exp(-1.1 * tail) * 10


def test_relaxation_without_rate_is_the_coherent_path():
    m0 = O.model(O.PIFLUX3D, hopping=1.0, beta=1.0, fermi_energy=0.2)
    m1 = O.model(O.PIFLUX3D, hopping=1.0, beta=1.0, fermi_energy=0.2, inv_offdiag_relax=3.0)
    rows = O.grid_piflux3d_ref(m0, 1, 1)[:64]
    tc = O.time_config(0.0, 4 * math.pi, 128)
    p = O.Pulse(1.0, 1)
    j0, _, rc0 = O.current_density(m0, p, tc, O.solver(), rows)
    j1, _, rc1 = O.current_density(m1, p, tc, O.solver(), rows)
    assert rc0 == rc1 == 0
    assert np.array_equal(j0, j1)  # inv_diag_relax = 0 selects time_evolution_sigma


# --------------------------------------------------------------------------
# the C ABI's host side (no GPU needed)
# --------------------------------------------------------------------------
def test_abi_thermal_rows_match_oracle():
    sys = api.system(api.SYS_PIFLUX3D, hopping=0.8, beta=1.7, fermi_energy=0.35,
                     inv_diag_relax=0.5, inv_offdiag_relax=0.5)
    rows = api.grid_rows(sys, api.grid_piflux3d_ref(2, 2))
    m = O.model(O.PIFLUX3D, hopping=0.8, beta=1.7, fermi_energy=0.35)
    ref = O.grid_piflux3d_ref(m, 2, 2)
    assert np.allclose(rows, ref, rtol=1e-14, atol=1e-15)
    sys = api.system(api.SYS_HONEYCOMB, hopping=1.2, beta=0.9, fermi_energy=-0.2)
    rows = api.grid_rows(sys, api.grid_honeycomb_hex_ref(6))
    ref = O.grid_honeycomb_hex_ref(O.model(O.HONEYCOMB, hopping=1.2, beta=0.9, fermi_energy=-0.2), 6)
    assert np.allclose(rows, ref, rtol=1e-14, atol=1e-15)


def test_abi_debug_rows_match_oracle():
    # the debug traces' momenta (PiFlux.cpp:320-371), cold and thermal
    for kw in ({}, {"beta": 1.3, "fermi_energy": 0.2, "inv_diag_relax": 0.4}):
        sys = api.system(api.SYS_PIFLUX3D, hopping=0.9, **kw)
        rows = api.grid_rows(sys, api.grid_piflux3d_debug())
        okw = {k: v for k, v in kw.items() if k != "inv_diag_relax"}
        ref = O.grid_piflux3d_debug(O.model(O.PIFLUX3D, hopping=0.9, **okw))
        assert rows.shape == (api.N_DEBUG_POINTS, 8)
        assert np.array_equal(rows[:, :4], ref[:, :4])
        assert np.allclose(rows, ref, rtol=1e-14, atol=1e-15)


def test_abi_dirac_debug_rows_match_oracle():
    # DiracSystem::compute_current_density_debug's (k_z, kappa) rows
    for n_z, max_k, kw in ((58, 15.0, {}), (20, 3.0, {"beta": 0.8, "fermi_energy": 0.3})):
        rows = api.grid_rows(api.system(api.SYS_DIRAC3D, **kw), api.grid_dirac3d_debug(n_z, max_k))
        ref = O.grid_dirac3d_debug(O.model(O.DIRAC3D, **kw), n_z, max_k)
        assert rows.shape == (api.N_DEBUG_POINTS, 8) and np.array_equal(rows, ref)
        assert rows[0, 0] == (n_z // 10) * (2 * max_k / n_z) > 0
    assert _grid_rows_status(api.system(api.SYS_DIRAC3D), api.grid_dirac3d_debug(0, 1.0)) == api.BAD_CONFIG


def _grid_rows_status(sys, grid):
    lib = api.load_library()
    n = ctypes.c_int64(0)
    return lib.hhg_grid_rows(ctypes.byref(sys), ctypes.byref(grid), None, ctypes.byref(n))


def test_abi_rejects_thermal_variant_models():
    grid = api.grid_tensor(4, 4, -1, 1, -1, 1)
    for kw in ({"beta": 1.0}, {"fermi_energy": 0.1}, {"inv_diag_relax": 1.0}):
        assert _grid_rows_status(api.system(api.SYS_PIFLUX2D, hopping=1.0, **kw), grid) == api.UNSUPPORTED
        assert _grid_rows_status(api.system(api.SYS_DIRAC2D, velocity=1.0, **kw), grid) == api.UNSUPPORTED
        assert _grid_rows_status(api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1, **kw),
                                 grid) == api.UNSUPPORTED
    assert _grid_rows_status(api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=-1.0), grid) == api.BAD_CONFIG
    assert _grid_rows_status(api.system(api.SYS_PIFLUX3D, hopping=1.0, inv_diag_relax=-1.0),
                             grid) == api.BAD_CONFIG
    assert _grid_rows_status(api.system(api.SYS_PIFLUX3D, hopping=1.0, beta=1.0, inv_diag_relax=2.0),
                             grid) == api.OK


def test_host_pulse_values_match_the_oracle():
    # hhg_pulse_values (host) and the oracle's A(t) for every pulse kind
    t = np.linspace(-1.0, 30.0, 211)
    cases = [(api.cosine_pulse(0.7, 2, 64, t_begin=1.0, phase=0.2), O.Pulse(0.7, 2, 1.0, 0.2)),
             (api.continuous_pulse(0.4, 64, (-3, 3), phase=0.1), O.ContinuousPulse(0.4, 0.1)),
             (api.gauss_pulse(0.9, 1, 64, t_begin=0.5, phase=0.3), O.GaussPulse(0.9, 1, 0.5, 0.3))]
    y = np.sin(np.linspace(0, 3, 40)) ** 2
    cases.append((api.spline_pulse(y, 0.5, 0.6, 64, (0.5, 20.0), cut=20.0, deriv=(0.0, math.nan),
                                   amplitude=1.5),
                  O.SplinePulse(y, 0.5, 0.6, cut=20.0, deriv=(0.0, math.nan), amplitude=1.5)))
    for desc, op in cases:
        a = api.pulse_values(desc, t)
        b = O.laser(op, t)
        assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.abs(b).max()), desc.kind
