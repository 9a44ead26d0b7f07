"""The reference's run modes (sources/hhg.cpp) on the engine.

`run(engine, source)` executes what a parameter file asks for, in the
reference's order: the occupation tracking (occupations != "no",
hhg.cpp:120-168), the energy-split current (split_current != "no",
hhg.cpp:170-219) and, unless either says "only", the current density with its
spectrum (hhg.cpp:236-337), followed by the PiFlux or Dirac debug traces when
debug_data is "yes" or "only" (hhg.cpp:235-238, 287-291, 343-352).  Each mode returns the
JSON document the reference writes (the same keys; the metadata files are not
produced), and `save` writes one gzip-compressed as `*.json.gz`.

Integration, Brillouin-zone sums and spectra run on the GPU through the C
ABI; the host only builds descriptors, relabels the occupation grid and
assembles the documents.
"""
from __future__ import annotations

import gzip
import json
import math
import time

import numpy as np

from . import api, config

OCCUPATION_SAMPLES = 499            # N_time of the occupation run (hhg.cpp:121)
SPLIT_ENERGY_CUT = 0.5 * math.sqrt(3.0)  # energy_cut (PiFlux.cpp:958)


def _header(cfg: dict, run: config.Run, N: int, laser_type: str) -> dict:
    p = run.pulse
    me = (p.window_end - p.window_begin) / p.n_measurements
    extra = int(laser_type != "continuous")
    t = p.window_begin + me * np.arange(p.n_measurements + extra)
    pe = float(cfg["photon_energy"])
    if laser_type in config.DOUBLE_LASERS:
        pe *= config.EXP_PHOTON_ENERGY  # the laser's photon_energy member
    return {
        "time": time.strftime("%Y-%m-%d %H:%M:%S"),
        "laser_function": api.pulse_values(p, t).tolist(),
        "N": N,
        "t_begin": p.window_begin,
        "t_end": p.window_end,
        "n_laser_cycles": int(float(cfg["n_laser_cycles"])),
        "n_measurements": p.n_measurements + extra,
        "T": float(cfg["T"]),
        "E_F": float(cfg["E_F"]),
        "v_F": float(cfg["v_F"]),
        "band_width": float(cfg["band_width"]),
        "field_amplitude": float(cfg["field_amplitude"]),
        "photon_energy": pe,
        "laser_type": laser_type,
        "diagonal_relaxation_time": float(cfg["diagonal_relaxation_time"]),
        "offdiagonal_relaxation_time": float(cfg.get("offdiagonal_relaxation_time", "-1")),
        "system_type": cfg["system_type"],
        "n_z": int(float(cfg.get("n_z", "0"))),
        "t0_offset": float(cfg.get("t0_offset", "0")),
    }


def current_density(eng: api.Engine, cfg: dict, grid: api.GridDesc | None = None,
                    n_measurements: int | None = None) -> dict:
    """The main mode: j(t) on the system's grid (the Dirac system: its k_z
    slices and adaptive kappa rule) and its spectrum (trapezoidal FFT with 8x
    zero padding, or the Welch FFT for the continuous laser).  With
    debug_data "only" the reference skips the integration and transforms its
    zero-initialised j (hhg.cpp:235-236)."""
    run = config.from_config(cfg, grid=grid, n_measurements=n_measurements)
    p = run.pulse
    if cfg.get("debug_data", "no") == "only":
        j = np.zeros(p.n_measurements + 1)
    elif run.quad is not None:  # the Dirac system's k_z x kappa quadrature
        j, _, _ = eng.dirac_current_density(run.system, p, run.quad, run.opts)
    else:
        j, _ = eng.current_density(run.system, p, run.grid, run.opts)
    lt = cfg["laser_type"]
    if lt == "continuous":
        fr, re, im = eng.spectrum_welch(j, p.n_measurements, p.window_begin, p.window_end)
    else:
        fr, re, im = eng.spectrum(j, p.n_measurements, p.window_begin, p.window_end)
    doc = _header(cfg, run, p.n_measurements, lt)
    doc.update({"current_density_time": j.tolist(),
                "current_density_frequency_real": re.tolist(),
                "current_density_frequency_imag": im.tolist(),
                "frequencies": fr.tolist(), "zero_padding": 8})
    return doc


def occupations(eng: api.Engine, cfg: dict, N: int | None = None,
                n_measurements: int = OCCUPATION_SAMPLES) -> dict:
    """PiFlux::compute_occupation_numbers (PiFlux.cpp:909-953) on the N x N
    grid (N = n_z): the band amplitudes of every k at every sample, stored at
    (x, (z - round(A(t_i) / dz)) mod N) (coordinate_shift)."""
    if cfg["system_type"] != "PiFlux":
        raise config.UnsupportedConfig("occupation tracking is PiFlux's (PiFluxDispatcher.cpp:150-162)")
    N = N or int(float(cfg["n_z"]))
    run = config.from_config(cfg, grid=api.grid_piflux3d_occupation(N), n_measurements=n_measurements)
    p = run.pulse
    occ, _ = eng.k_resolved(run.system, p, run.grid, run.opts, kind=api.KOUT_OCCUPATIONS)
    occ = occ.reshape(p.n_measurements + 1, N, N, 2)  # [i][x][z]
    me = (p.window_end - p.window_begin) / p.n_measurements
    # the accumulated t_begin of sample i (PiFlux.cpp:941-946)
    t, tb = [], p.window_begin
    for _ in range(p.n_measurements + 1):
        t.append(tb)
        tb = tb + me
    A = api.pulse_values(p, np.array(t))
    dz = math.pi / N
    lower = np.zeros_like(occ[..., 0])
    upper = np.zeros_like(occ[..., 1])
    z = np.arange(N)
    for i in range(p.n_measurements + 1):
        v = A[i] / dz
        shift = int(math.copysign(math.floor(abs(v) + 0.5), v))  # std::round (half away from zero)
        zs = ((z - shift) % N + N) % N
        lower[i][:, zs] = occ[i, :, :, 0]
        upper[i][:, zs] = occ[i, :, :, 1]
    doc = _header(cfg, run, p.n_measurements, cfg["laser_type"])
    doc.update({"lower_band": lower.tolist(), "upper_band": upper.tolist()})
    return doc


def split_current(eng: api.Engine, cfg: dict, N: int | None = None,
                  n_measurements: int | None = None) -> dict:
    """PiFlux::current_per_energy (PiFlux.cpp:955-1035) on the N^3 grid (N =
    n_z): j(t) of the k with |d(k - A)| below and above sqrt(3)/2."""
    if cfg["system_type"] != "PiFlux":
        raise config.UnsupportedConfig("the split current is PiFlux's (PiFluxDispatcher.cpp:164-180)")
    N = N or int(float(cfg["n_z"]))
    run = config.from_config(cfg, grid=api.grid_piflux3d_cube(N), n_measurements=n_measurements)
    lo, hi, _ = eng.split_current(run.system, run.pulse, run.grid, run.opts, SPLIT_ENERGY_CUT)
    doc = _header(cfg, run, run.pulse.n_measurements, cfg["laser_type"])
    doc.update({"dirac_current": lo.tolist(), "non_dirac_current": hi.tolist()})
    return doc


def debug_traces(eng: api.Engine, cfg: dict, n_measurements: int | None = None,
                 frequencies=None) -> dict:
    """The debug traces: PiFlux::compute_current_density_debug
    (PiFlux.cpp:320-371), S_z(t_i) of the 25 momenta k = (pi/2, pi/2 - 0.02 pi i,
    0.49 pi) with the system's dynamics (coherent or relaxation), or the Dirac
    system's 25 weighted (k_z, kappa) currents, each transformed by
    TrapezoidalFFT without padding (hhg.cpp:287-291).  The document is time_evolution.json
    (hhg.cpp:343-352); its "frequencies" are the main spectrum's
    (`frequencies`, the 8x padded grid, as the reference stores them)."""
    if cfg["system_type"] == "Dirac":
        # DiracSystem::compute_current_density_debug and its relaxation twin
        # (DiracSystem.cpp:333-363, 427-457): the weighted current of 25 (k_z,
        # kappa) trajectories, by the dispatcher's stepper (DiracDispatcher.cpp:82-92)
        run = config.from_config(cfg, n_measurements=n_measurements)
        p = run.pulse
        grid = api.grid_dirac3d_debug(run.quad.n_z, run.quad.max_k)
        cur, _ = eng.k_resolved(run.system, p, grid, run.opts, kind=api.KOUT_CURRENT)
        traces = np.ascontiguousarray(cur.T)
    elif cfg["system_type"] == "PiFlux":
        run = config.from_config(cfg, grid=api.grid_piflux3d_debug(), n_measurements=n_measurements)
        p = run.pulse
        S, _ = eng.k_resolved(run.system, p, run.grid, run.opts, kind=api.KOUT_BLOCH)
        traces = np.ascontiguousarray(S[:, :, 2].T)  # [point][sample]
    else:
        raise config.UnsupportedConfig("Honeycomb::compute_current_density_debug is not implemented yet!")
    me = (p.window_end - p.window_begin) / p.n_measurements
    re, im = [], []
    for tr in traces:
        if cfg["laser_type"] == "continuous":  # no transform on the Welch branch (hhg.cpp:258-275)
            r = i = np.zeros(p.n_measurements + 1)
        else:
            _, r, i = eng.trapezoidal_fft(tr, me, p.window_begin, p.window_end)
        re.append(r.tolist())
        im.append(i.tolist())
    if frequencies is None:
        zero = np.zeros(p.n_measurements + 1)
        spec = eng.spectrum_welch if cfg["laser_type"] == "continuous" else eng.spectrum
        frequencies, _, _ = spec(zero, p.n_measurements, p.window_begin, p.window_end)
    return {"time": time.strftime("%Y-%m-%d %H:%M:%S"),
            "frequencies": list(frequencies),
            "time_evolutions": traces.tolist(),
            "debug_fft_real": re, "debug_fft_imag": im}


def run(eng: api.Engine, source: str) -> dict:
    """All modes a parameter file asks for: {"occupations": doc,
    "split_current": doc, "current_density": doc, "debug": doc} (present
    ones only)."""
    cfg = config.read_config(source)
    out = {}
    if cfg.get("occupations", "no") != "no":
        out["occupations"] = occupations(eng, cfg)
        if cfg["occupations"] == "only":
            return out
    if cfg.get("split_current", "no") != "no":
        out["split_current"] = split_current(eng, cfg)
        if cfg["split_current"] == "only":
            return out
    out["current_density"] = current_density(eng, cfg)
    if cfg.get("debug_data", "no") != "no":
        out["debug"] = debug_traces(eng, cfg, frequencies=out["current_density"]["frequencies"])
    return out


def save(doc: dict, path: str) -> None:
    """Write a document as gzip-compressed JSON (4-space indent, as
    nlohmann::json::dump(4) in hhg.cpp:336)."""
    with gzip.open(path, "wt") as f:
        json.dump(doc, f, indent=4)
