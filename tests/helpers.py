"""Shared test helpers: map C-ABI descriptors onto the oracle's structs and
compare currents / spectra the way the parity bar is stated."""
from __future__ import annotations

import math

import numpy as np

from oracle import hhg_oracle as O

SYS_TO_ORC = {0: O.DIRAC2D, 1: O.PIFLUX2D, 2: O.PIFLUX3D, 3: O.HONEYCOMB, 4: O.DIRAC3D}


def oracle_pulse(pulse):
    """The oracle's pulse for a C-ABI pulse descriptor."""
    if pulse.kind == 1:
        return O.ContinuousPulse(pulse.amplitude, pulse.phase)
    if pulse.kind == 2:
        return O.GaussPulse(pulse.amplitude, pulse.n_cycles, pulse.t_begin, pulse.phase)
    if pulse.kind == 3:
        return O.SplinePulse(pulse._samples, pulse.t_begin, pulse.sample_dt, cut=pulse.spline_cut,
                             deriv=(pulse.deriv_begin, pulse.deriv_end), amplitude=pulse.amplitude)
    return O.Pulse(pulse.amplitude, pulse.n_cycles, pulse.t_begin, pulse.phase)


def oracle_args(sys, pulse, abs_tol, rel_tol, stepper=0, magnus_substeps=1):
    es = pulse.energy_scale
    m = O.model(SYS_TO_ORC[sys.kind], hopping=sys.hopping * es, velocity=sys.velocity * es,
                mass=sys.mass * es, pol=(sys.pol_x, sys.pol_y), beta=sys.beta / es,
                fermi_energy=sys.fermi_energy * es, inv_diag_relax=sys.inv_diag_relax * es,
                inv_offdiag_relax=sys.inv_offdiag_relax * es)
    p = oracle_pulse(pulse)
    tc = O.time_config(pulse.window_begin, pulse.window_end, pulse.n_measurements,
                       pulse.n_subdivisions)
    s = O.solver(abs_tol, rel_tol, stepper=stepper, magnus_substeps=magnus_substeps)
    return m, p, tc, s


def oracle_j(sys, pulse, rows, abs_tol, rel_tol, **kw):
    m, p, tc, s = oracle_args(sys, pulse, abs_tol, rel_tol, **kw)
    j, st, rc = O.current_density(m, p, tc, s, rows, threads=0)
    assert rc == 0, f"oracle status {rc}"
    return j, st


def rel_l2(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


NOISE_FLOOR_REL = 1e-6  # harmonics within 60 dB of the strongest one are compared


def harmonics(j, pulse, max_order=None):
    freq, re, im = O.trapezoidal_fft(j, pulse.window_begin, pulse.window_end,
                                     pulse.n_measurements)
    if max_order is None:
        max_order = int(min(freq[-1] - 1, 60))
    return O.harmonic_intensities(freq, re, im, max_order)


def harmonic_rel_err(I, I_ref, floor_rel=NOISE_FLOOR_REL) -> float:
    floor = floor_rel * I_ref.max()
    mask = I_ref > floor
    return float(np.max(np.abs(I[mask] - I_ref[mask]) / I_ref[mask]))
