"""Harmonic analysis of spectra produced by the engine.

The reference writes Re/Im of j_hat and the frequencies
(sources/hhg.cpp:317-329) and leaves intensities to post-processing; here
I(n) = |j_hat(n omega_L)|^2 at integer harmonics n (nearest frequency bin,
frequencies in units of omega_L), and a relative-error measure restricted to
harmonics above a noise floor (a fraction of the strongest harmonic).
"""
from __future__ import annotations

import numpy as np


def harmonic_intensities(freq, re, im, max_order: int) -> np.ndarray:
    p = np.asarray(re) ** 2 + np.asarray(im) ** 2
    freq = np.asarray(freq)
    out = np.zeros(max_order)
    for n in range(1, max_order + 1):
        out[n - 1] = p[int(np.argmin(np.abs(freq - n)))]
    return out


def default_max_order(freq) -> int:
    return int(min(float(np.asarray(freq)[-1]) - 1, 60))


def harmonic_rel_err(I, I_ref, floor_rel: float = 1e-6) -> float:
    """max |I - I_ref| / I_ref over harmonics with I_ref > floor_rel * max(I_ref)."""
    I = np.asarray(I)
    I_ref = np.asarray(I_ref)
    mask = I_ref > floor_rel * I_ref.max()
    return float(np.max(np.abs(I[mask] - I_ref[mask]) / I_ref[mask]))
