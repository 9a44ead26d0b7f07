"""Physics invariants of the oracle and the Fourier tail restatement."""
import math

import numpy as np
import pytest

from oracle import hhg_oracle as O


def _rows(m, n=8):
    return O.grid_tensor(m, n, n, -2, 2, -2, 2)


def test_zero_field_gives_static_current():
    m = O.model(O.DIRAC2D, velocity=10.0, mass=0.5)
    rows = _rows(m)
    p = O.Pulse(0.0, 2)
    tc = O.time_config(0.0, p.t_end, 256)
    j, st, rc = O.current_density(m, p, tc, O.solver(1e-10, 1e-10), rows)
    assert rc == 0
    # S0 = -d_hat is stationary; on the symmetric grid the x-current vanishes
    assert np.max(np.abs(j - j[0])) <= 1e-13
    assert abs(j[0]) <= 1e-13


def test_inversion_symmetry_odd_current():
    # A -> -A (phase + pi) maps j -> -j for the inversion-symmetric models
    for kind, kw in [(O.DIRAC2D, dict(velocity=10.0, mass=0.5)),
                     (O.PIFLUX2D, dict(hopping=20.0, pol=(0.6, 0.8)))]:
        m = O.model(kind, **kw)
        lo, hi = (-2, 2) if kind == O.DIRAC2D else (-math.pi, math.pi)
        rows = O.grid_tensor(m, 8, 8, lo, hi, lo, hi)
        tc = O.time_config(0.0, 4 * math.pi, 512)
        s = O.solver(1e-12, 1e-10)
        ja, _, _ = O.current_density(m, O.Pulse(0.8, 2, phase=0.3), tc, s, rows)
        jb, _, _ = O.current_density(m, O.Pulse(0.8, 2, phase=0.3 + math.pi), tc, s, rows)
        assert np.max(np.abs(ja + jb)) <= 1e-7 * np.max(np.abs(ja))


def test_bloch_norm_conserved_all_models():
    cases = [(O.model(O.DIRAC2D, velocity=10.0, mass=0.5), (0.3, 0.2, 0.0)),
             (O.model(O.PIFLUX2D, hopping=20.0, pol=(0.7, 0.7)), (0.4, -1.1, 0.0)),
             (O.model(O.PIFLUX3D, hopping=1.0), (0.4, 1.0, 2.0)),
             (O.model(O.HONEYCOMB, hopping=10.0, mass=1.0), (0.5, 0.3, 0.0))]
    p = O.Pulse(1.0, 1)
    tc = O.time_config(0.0, p.t_end, 256)
    for m, (kx, ky, kz) in cases:
        krow = np.zeros(8)
        krow[:4] = [kx, ky, kz, 1.0]
        O.lib().orc_initial_state(O.ctypes.byref(m), O.ctypes.c_double(kx),
                                  O.ctypes.c_double(ky), O.ctypes.c_double(kz),
                                  krow[4:7].ctypes.data_as(O._D))
        assert abs(np.linalg.norm(krow[4:7]) - 1) <= 1e-14
        S, _ = O.evolve_k(m, p, tc, O.solver(1e-12, 1e-10), krow)
        assert np.max(np.abs(np.linalg.norm(S, axis=1) - 1)) <= 1e-8


def _direct_trapezoid(j, tb, te, n):
    """TrapezoidalFFT::compute (TrapezoidalFFT.cpp:11-49) evaluated with an
    explicit O(N^2) DFT in place of FFTW, on the x8 zero-padded input."""
    dt = (te - tb) / n
    n_in = 8 * (n + 1)
    x = np.zeros(n_in)
    x[: len(j)] = j
    k = np.arange(n_in)
    out = []
    for m in range(n_in // 2 + 1):
        F = np.sum(x * np.exp(-2j * np.pi * m * k / n_in))
        w = 2 * m * np.pi / (n_in * dt)
        th = w * dt
        if m == 0:
            W, a0 = 1.0, -0.5
        else:
            W = 2 * (1 - math.cos(th)) / th ** 2
            a0 = (-(1 - math.cos(th)) + 1j * (th - math.sin(th))) / th ** 2
        corr = a0 * x[0] + np.conj(a0) * np.exp(1j * w * (te - tb)) * x[n_in - 1]
        out.append(dt * (dt * W * np.exp(1j * w * tb) * F + corr))
    return np.array(out)


def test_trapezoidal_fft_matches_direct_formula():
    rng = np.random.default_rng(5)
    n = 31
    j = rng.normal(size=n + 1)
    tb, te = 0.3, 4.0
    fr, re, im = O.trapezoidal_fft(j, tb, te, n)
    d = _direct_trapezoid(j, tb, te, n)
    assert np.max(np.abs((re + 1j * im) - d)) <= 1e-12 * np.max(np.abs(d))
    assert np.allclose(fr, 2 * np.arange(len(fr)) * np.pi / (8 * (n + 1) * (te - tb) / n))


def test_unpadded_transform_is_the_padded_one_on_padded_input():
    # hhg.cpp transforms j after padding it x8 and each debug trace as given;
    # both are TrapezoidalFFT::compute on the vector it receives
    rng = np.random.default_rng(3)
    n = 200
    j = rng.normal(size=n + 1)
    tb, te = -0.4, 9.6
    f1, r1, i1 = O.trapezoidal_fft(j, tb, te, n)
    x = np.zeros(O.ZERO_PADDING * (n + 1))
    x[: n + 1] = j
    f2, r2, i2 = O.trapezoidal_fft_unpadded(x, (te - tb) / n, tb, te)
    assert np.array_equal(f1, f2) and np.array_equal(r1, r2) and np.array_equal(i1, i2)
    f3, r3, i3 = O.trapezoidal_fft_unpadded(j, (te - tb) / n, tb, te)
    assert f3.size == (n + 1) // 2 + 1
    # the unpadded grid is every 8th frequency of the padded one
    assert np.allclose(f3[1:], f1[8:8 * f3.size:8][: f3.size - 1], rtol=1e-14)


def test_harmonics_of_a_pure_tone():
    # j(t) = sin(3t) env(t): the spectrum peaks at harmonic 3
    n = 4096
    tb, te = 0.0, 8 * math.pi
    t = tb + (te - tb) * np.arange(n + 1) / n
    j = np.sin(3 * t) * np.sin(t / 8) ** 2
    fr, re, im = O.trapezoidal_fft(j, tb, te, n)
    I = O.harmonic_intensities(fr, re, im, 6)
    assert int(np.argmax(I)) == 2
    assert I[2] > 1e3 * max(I[0], I[4])
