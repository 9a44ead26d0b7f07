"""Magnus propagators of the oracle.

* The Dirac-3D closed form (MagnusMatrix.cpp) is pinned against the
  reference's own sympy derivation (helper/magnus_dirac.py), evaluated at
  seeded points into tests/golden/magnus_dirac.json: U = exp(Omega).
* The reference Magnus path and the reference RKF78 sigma path of the Dirac
  model describe the same equation; they are compared on a few (k_z, kappa).
* The general Magnus-4 stepper converges to the RKF78 solution.
"""
import json
import math
import os

import numpy as np
import pytest
from scipy.linalg import expm

from oracle import hhg_oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "magnus_dirac.json")))


@pytest.mark.parametrize("idx", range(len(GOLD["points"])))
def test_dirac_magnus_matches_sympy_derivation(idx):
    pt = GOLD["points"][idx]
    x = pt["inputs"]
    omega = np.array(pt["omega"])
    U = O.dirac_magnus_U(x["k"], x["kappa"], x["k_z"], 1.0,
                         [x["alpha"], x["beta"], x["gamma"], x["delta"]])
    assert np.max(np.abs(U - expm(omega))) <= 1e-13
    # the reference's (a, b, c) layout (MagnusMatrix.cpp:59-63) is skew
    assert np.allclose(omega, -omega.T, atol=1e-15)


def test_magnus_coefficients_constant_pulse_limit():
    # for a window that sees A(t) ~ A0 sin(t) env(t) the first moment is the mean
    p = O.Pulse(0.7, 4)
    dt, t0 = 0.05, 3.0
    c = O.magnus_coefficients(p, dt, t0)
    ts = t0 + dt * (np.arange(20000) + 0.5) / 20000
    mean = np.mean(O.laser(p, ts))
    assert abs(c[0] - mean) <= 1e-9
    # shifted-Legendre P1 moment, times 3
    m1 = 3 * np.mean(O.laser(p, ts) * (2 * (ts - t0) / dt - 1))
    assert abs(c[1] - m1) <= 1e-8


def test_reference_dirac_magnus_vs_sigma_rkf78():
    p = O.Pulse(0.6, 2)
    tc = O.time_config(0.0, p.t_end, 2048)
    s = O.solver(1e-12, 1e-10)
    for kz, kap in [(0.5, 0.4), (-0.3, 0.9), (1.2, 0.2)]:
        mag = O.dirac3d_magnus_k(p, tc, kz, kap)
        rk = O.dirac3d_sigma_k(p, tc, s, kz, kap)
        # one Magnus step per interval, no error control (DiracSystem.cpp:200-210)
        assert np.max(np.abs(mag - rk)) <= 5e-4, (kz, kap, np.max(np.abs(mag - rk)))


def test_general_magnus4_converges_to_rkf78():
    m = O.model(O.HONEYCOMB, hopping=12.5, mass=1.25)
    p = O.Pulse(1.0, 2)
    tc = O.time_config(0.0, 3 * 2 * math.pi, 1024)
    krow = np.zeros(8)
    krow[0], krow[1], krow[3] = 0.7, -0.4, 1.0
    O.lib().orc_initial_state(O.ctypes.byref(m), O.ctypes.c_double(0.7),
                              O.ctypes.c_double(-0.4), O.ctypes.c_double(0.0),
                              krow[4:7].ctypes.data_as(O._D))
    ref, _ = O.evolve_k(m, p, tc, O.solver(1e-13, 1e-12), krow)
    errs = []
    for sub in (2, 4, 8):
        S, _ = O.evolve_k(m, p, tc, O.solver(stepper=1, magnus_substeps=sub), krow)
        errs.append(np.max(np.abs(S - ref)))
    # fourth order: halving the step cuts the error ~16x
    assert errs[0] / errs[1] > 10 and errs[1] / errs[2] > 10
    assert errs[2] < 1e-7


def test_generic_dirac_magnus_stepper_is_the_reference_loop():
    # the oracle's per-k loop with stepper 2 reproduces its restatement of
    # DiracSystem::time_evolution_magnus bit for bit
    import math
    p = O.Pulse(0.7, 2)
    tc = O.time_config(0.0, 4 * math.pi, 256)
    for kz, kap in ((0.4, 0.9), (-1.1, 0.2), (0.05, 1.3)):
        mk = math.hypot(kz, kap)
        row = np.array([kz, kap, mk, 1.0, 0.0, 0.0, -1.0, 0.0])
        states, st = O.evolve_k(O.model(O.DIRAC3D), p, tc, O.solver(stepper=2), row)
        assert np.array_equal(states[:, 2], O.dirac3d_magnus_k(p, tc, kz, kap))
        assert st.attempted == 256
