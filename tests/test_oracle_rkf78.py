"""Known-answer tests of the oracle's stepper: the Fehlberg 7(8) tableau
(order conditions, convergence order) and the controlled-stepping semantics
restated from Boost.Odeint (integrate_adaptive + controlled_runge_kutta +
default_error_checker / default_step_adjuster) as called by the reference
(PiFlux.cpp:104-110)."""
import math
from fractions import Fraction

import numpy as np
import pytest

from oracle import hhg_oracle as O

C, A, B, DB = O.rkf78_tableau()
B7 = B - DB  # the embedded 7th-order weights


def test_row_sums_equal_nodes():
    assert np.max(np.abs(A.sum(axis=1) - C)) <= 2e-15


@pytest.mark.parametrize("k", range(1, 9))
def test_quadrature_conditions_order8(k):
    # sum_i b_i c_i^(k-1) = 1/k, k = 1..8
    assert abs(np.dot(B, C ** (k - 1)) - 1.0 / k) <= 1e-15


@pytest.mark.parametrize("k", range(1, 8))
def test_quadrature_conditions_order7(k):
    assert abs(np.dot(B7, C ** (k - 1)) - 1.0 / k) <= 1e-15


def test_tree_conditions_up_to_order5():
    for b in (B, B7):
        assert abs(b @ A @ C - 1 / 6) <= 1e-15
        assert abs(b @ (C * (A @ C)) - 1 / 8) <= 1e-15
        assert abs(b @ A @ (C ** 2) - 1 / 12) <= 1e-15
        assert abs(b @ A @ A @ C - 1 / 24) <= 1e-15
        assert abs(b @ (C ** 2 * (A @ C)) - 1 / 10) <= 1e-15
        assert abs(b @ ((A @ C) ** 2) - 1 / 20) <= 1e-15
        assert abs(b @ A @ A @ A @ C - 1 / 120) <= 1e-15


def test_error_weights_are_fehlberg():
    # b8 - b7 = 41/840 (e12 + e13 - e1 - e11)
    want = np.zeros(13)
    want[[0, 10]] = -41 / 840
    want[[11, 12]] = 41 / 840
    assert np.array_equal(DB, want)
    assert abs(float(sum(Fraction(x).limit_denominator(10 ** 6) for x in B)) - 1) < 1e-15


def _rk_fixed(f, y0, t0, t1, n, b):
    h = (t1 - t0) / n
    y = np.array(y0, dtype=np.float64)
    t = t0
    for _ in range(n):
        K = np.zeros((13, len(y)))
        for s in range(13):
            K[s] = f(t + C[s] * h, y + h * (A[s, :s] @ K[:s]))
        y = y + h * (b @ K)
        t += h
    return y


def test_convergence_orders():
    # y' = y cos t, y(0) = 1 -> y = exp(sin t)
    f = lambda t, y: y * math.cos(t)
    exact = math.exp(math.sin(6.0))
    e8 = [abs(_rk_fixed(f, [1.0], 0.0, 6.0, n, B)[0] - exact) for n in (6, 12)]
    e7 = [abs(_rk_fixed(f, [1.0], 0.0, 6.0, n, B7)[0] - exact) for n in (6, 12)]
    assert math.log2(e8[0] / e8[1]) > 7.5
    assert math.log2(e7[0] / e7[1]) > 6.5


def _dirac_setup(n=64):
    m = O.model(O.DIRAC2D, velocity=10.0, mass=0.5)
    p = O.Pulse(1.0, 4)
    tc = O.time_config(0.0, p.t_end, n * 64)
    return m, p, tc


def test_controller_restart_pattern():
    """Smooth trajectories take exactly 4 steps per interval: dt0 = D/50, two
    growths by 0.9 * (5^-8)^(-1/8) = 4.5, then the clipped remainder."""
    m, p, tc = _dirac_setup()
    krow = np.zeros(8)
    krow[0], krow[1], krow[3] = 0.3, -0.2, 1.0
    O.lib().orc_initial_state(O.ctypes.byref(m), O.ctypes.c_double(0.3),
                              O.ctypes.c_double(-0.2), O.ctypes.c_double(0.0),
                              krow[4:7].ctypes.data_as(O._D))
    s = O.solver(1e-10, 1e-10)
    h = O.step_history(m, p, tc, s, krow)
    D = (tc.t_end - tc.t_begin) / tc.n_measurements
    g = 0.9 * pow(pow(5.0, -8.0), -1.0 / 8)
    assert len(h) == 4 * tc.n_measurements
    assert np.all(h[:, 3] == 1.0)
    first = h[:4]
    assert first[0, 1] == D / 50
    assert first[1, 1] == D / 50 * g
    assert first[2, 1] == D / 50 * g * g
    assert abs(first[:, 1].sum() - D) <= 1e-15 * 50


def test_controller_rejects_and_shrinks():
    """A stiff point (large |d|) with tight tolerances rejects; each
    rejection shrinks dt by max(0.9 err^(-1/6), 0.2)."""
    m = O.model(O.DIRAC2D, velocity=400.0, mass=0.5)
    p = O.Pulse(1.0, 1)
    tc = O.time_config(0.0, p.t_end, 16)
    s = O.solver(1e-12, 1e-12)
    krow = np.array([1.5, 1.0, 0.0, 1.0, 0, 0, 0, 0.0])
    O.lib().orc_initial_state(O.ctypes.byref(m), O.ctypes.c_double(1.5), O.ctypes.c_double(1.0),
                              O.ctypes.c_double(0.0), krow[4:7].ctypes.data_as(O._D))
    h = O.step_history(m, p, tc, s, krow)
    rej = np.where(h[:, 3] == 0.0)[0]
    assert len(rej) > 0
    for r in rej[:20]:
        err = h[r, 2]
        want = h[r, 1] * max(0.9 * err ** (-1.0 / 6.0), 0.2)
        assert h[r + 1, 1] == pytest.approx(want, rel=1e-15)
    # steps always land exactly on the interval ends
    D = (tc.t_end - tc.t_begin) / tc.n_measurements
    acc = h[h[:, 3] == 1.0]
    ends = acc[:, 0] + acc[:, 1]
    t_end = 0.0
    hits = 0
    for i in range(1, tc.n_measurements + 1):
        t_end = t_end + D if i > 1 else D
        hits += np.any(ends == t_end)
    assert hits == tc.n_measurements


def test_norm_conserved_and_static_without_field():
    m, p, tc = _dirac_setup(16)
    s = O.solver(1e-10, 1e-10)
    krow = np.array([0.4, 0.9, 0.0, 1.0, 0, 0, 0, 0.0])
    O.lib().orc_initial_state(O.ctypes.byref(m), O.ctypes.c_double(0.4), O.ctypes.c_double(0.9),
                              O.ctypes.c_double(0.0), krow[4:7].ctypes.data_as(O._D))
    S, st = O.evolve_k(m, p, tc, s, krow)
    assert np.max(np.abs(np.linalg.norm(S, axis=1) - 1.0)) <= 1e-9
    p0 = O.Pulse(0.0, 4)
    S0, _ = O.evolve_k(m, p0, tc, s, krow)
    # S0 = -d_hat is stationary when A = 0
    assert np.max(np.abs(S0 - S0[0])) <= 1e-12


def test_step_limit_reported():
    m, p, tc = _dirac_setup(1)
    s = O.solver(1e-300, 0.0)
    s.max_failed = 5
    krow = np.array([0.4, 0.9, 0.0, 1.0, 0.0, 0.0, -1.0, 0.0])
    with pytest.raises(RuntimeError):
        O.evolve_k(m, p, tc, s, krow)
