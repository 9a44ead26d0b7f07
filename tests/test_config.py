"""The reference's parameter files -> descriptors (higherharmonics_b200.config):
parsing, the unit mapping of the reference's dispatchers and constructors,
and the configurations the engine refuses.  CPU only."""
import math

import numpy as np
import pytest

from higherharmonics_b200 import api, config

HBAR = 6.582119569509065698e-13
K_B = 0.08617333262145177434

PIFLUX = """\
# material
T 300
E_F 118
v_F 1.5e6
band_width 300   # meV
field_amplitude 1.6
photon_energy 5.25
diagonal_relaxation_time 15
offdiagonal_relaxation_time -1
laser_type cosine
n_laser_cycles 4
t0_offset 2
n_z 51
data_dir test
debug_data no
occupations no
split_current no
system_type PiFlux
"""


def test_read_config_strips_comments_and_units():
    cfg = config.read_config("E_F 118 meV\n# a comment\n\nv_F 1.5e6 m/s # tail\n")
    assert cfg == {"E_F": "118", "v_F": "1.5e6"}
    with pytest.raises(ValueError):
        config.read_config("lonely_key\n")


def test_piflux_mapping():
    run = config.from_config(PIFLUX)
    s, p = run.system, run.pulse
    pe = 5.25
    assert s.kind == api.SYS_PIFLUX3D
    assert s.beta == pytest.approx(pe / (K_B * 300), rel=1e-15)
    assert s.fermi_energy == pytest.approx(118 / pe, rel=1e-15)
    assert s.hopping == pytest.approx(300 / math.sqrt(12), rel=1e-15)
    rate = 1e15 * HBAR / (15 * pe)
    assert s.inv_diag_relax == pytest.approx(rate, rel=1e-15)
    assert s.inv_offdiag_relax == pytest.approx(rate, rel=1e-15)  # tau_offdiag <= 0 -> tau_diag
    lattice = math.sqrt(3) * HBAR * 1.5e6 / (pe * 300)
    assert run.lattice_constant == pytest.approx(lattice, rel=1e-15)
    assert p.amplitude == pytest.approx(lattice * 1e11 * 1.6 / pe, rel=1e-15)
    assert p.n_measurements == 4 * 1024
    assert p.t_begin == pytest.approx(2 * math.pi)
    assert p.window_begin == pytest.approx(2 * math.pi)
    assert p.window_end == pytest.approx(2 * math.pi + 2 * math.pi * 4 + 2 * math.pi)
    assert p.n_subdivisions == 50
    assert run.grid.kind == api.GRID_PIFLUX3D_REF and (run.grid.n1, run.grid.n2) == (32, 4)
    assert (run.opts.abs_tol, run.opts.rel_tol) == (1e-12, 1e-8)


def test_offdiagonal_time_and_coherent_path():
    run = config.from_config(PIFLUX.replace("offdiagonal_relaxation_time -1",
                                            "offdiagonal_relaxation_time 30"))
    assert run.system.inv_offdiag_relax == pytest.approx(1e15 * HBAR / (30 * 5.25))
    run = config.from_config(PIFLUX.replace("diagonal_relaxation_time 15\n",
                                            "diagonal_relaxation_time -1\n"))
    assert run.system.inv_diag_relax == 0.0 and run.system.inv_offdiag_relax == 0.0
    run = config.from_config(PIFLUX.replace("T 300", "T 0"))
    assert run.system.beta == 0.0


def test_honeycomb_mapping():
    run = config.from_config(PIFLUX.replace("system_type PiFlux", "system_type Honeycomb"))
    s = run.system
    assert s.kind == api.SYS_HONEYCOMB and (s.pol_x, s.pol_y) == (1.0, 0.0)
    assert s.hopping == pytest.approx(50.0)
    assert s.inv_offdiag_relax == 0.0
    assert run.lattice_constant == pytest.approx(4 * HBAR * 1.5e6 / (5.25 * 300))
    assert run.grid.kind == api.GRID_HONEYCOMB_HEX_REF and run.grid.n1 == 64


def test_descriptors_pass_the_abi_checks():
    run = config.from_config(PIFLUX, grid=api.grid_piflux3d_ref(1, 1))
    rows = api.grid_rows(run.system, run.grid)
    assert rows.shape[1] == 8 and rows.shape[0] > 0


@pytest.mark.parametrize("edit,exc", [
    (("laser_type cosine", "laser_type expA"), config.UnsupportedConfig),
    (("system_type PiFlux", "system_type ModifiedPiFlux"), config.UnsupportedConfig),
    (("system_type PiFlux", "system_type Dirac\n"), None),
    (("debug_data no", "debug_data yes"), None),
    (("debug_data no\noccupations no\nsplit_current no\nsystem_type PiFlux",
      "debug_data only\noccupations no\nsplit_current no\nsystem_type Honeycomb"),
     config.UnsupportedConfig),
    (("system_type PiFlux", "system_type Graphene"), ValueError),
    (("E_F 118\n", ""), ValueError),
])
def test_refused_configurations(edit, exc):
    if exc is None:
        config.from_config(PIFLUX.replace(*edit))
        return
    with pytest.raises(exc):
        config.from_config(PIFLUX.replace(*edit))


def _laser(lt, t0="8", cycles="2"):
    return config.from_config(PIFLUX.replace("laser_type cosine", f"laser_type {lt}")
                              .replace("t0_offset 2", f"t0_offset {t0}")
                              .replace("n_laser_cycles 4", f"n_laser_cycles {cycles}"))


def test_laser_types_map_to_pulses():
    pe, E0 = 5.25, 1.6
    lattice = math.sqrt(3) * HBAR * 1.5e6 / (pe * 300)
    A0 = lattice * 1e11 * E0 / pe
    r = _laser("continuous")
    assert r.pulse.kind == api.PULSE_CONTINUOUS and r.pulse.amplitude == pytest.approx(A0)
    assert (r.pulse.window_begin, r.pulse.window_end) == pytest.approx((-2 * math.pi, 2 * math.pi))
    r = _laser("gauss")
    assert r.pulse.kind == api.PULSE_GAUSS and r.pulse.t_begin == 8.0
    assert r.pulse.window_end == pytest.approx(8.0 + 12 * math.pi)
    r = _laser("quench")
    p = r.pulse
    assert p.kind == api.PULSE_SPLINE and p.n_samples == 256 and p.spline_cut == 8.0
    y = p._samples
    assert y[63] == 0 and y[64] == pytest.approx(0.5 * A0) and y[100] == pytest.approx(A0) and y[193] == 0
    assert p.sample_dt == pytest.approx(8.0 / 255) and (p.deriv_begin, p.deriv_end) == (0.0, 0.0)
    r = _laser("powerlaw1")
    y = r.pulse._samples
    assert y[0] == 0 and y[128] == pytest.approx(A0 * 0.5) and math.isnan(r.pulse.deriv_begin)


def test_double_lasers_use_the_experimental_photon_energy():
    r = _laser("dcos", t0="0.5")
    pe = 5.25 * config.EXP_PHOTON_ENERGY
    lattice = math.sqrt(3) * HBAR * 1.5e6 / (pe * 300)
    assert r.lattice_constant == pytest.approx(lattice, rel=1e-15)
    assert r.system.fermi_energy == pytest.approx(118 / pe)
    p = r.pulse
    assert p.n_samples == 1000 and p.spline_cut == pytest.approx(1.5 * 4 * math.pi)
    # laser A (1.6 E0) plus laser B (0.7 E0) delayed by 0.5 ps
    shift = 5.25 * (0.5 * config.EXP_PHOTON_ENERGY / (1e12 * HBAR))
    t = 500 * p.sample_dt
    a = lattice * 1e11 * 1.6 * 1.6 / pe
    b = lattice * 1e11 * 0.7 * 1.6 / pe

    def cosl(A, t):
        return 0.0 if (t <= 0 or t >= 4 * math.pi) else A * 0.5 * (1 - math.cos(t / 2)) * math.sin(t)
    assert p._samples[500] == pytest.approx(cosl(a, t) + cosl(b, t - shift), rel=1e-12, abs=1e-12)
    assert _laser("dcosA", t0="0.5").pulse._samples[500] == pytest.approx(cosl(a, t), abs=1e-12)


def synthetic_field(n=201, seed=7):
    """A smooth two-pulse field in MV/cm at the reference's sample spacing
    (seeded; not measured data): Gaussian-enveloped carriers near the data's
    photon energy, pulse B weaker and later."""
    rng = np.random.default_rng(seed)
    t = np.arange(n) * config.EXP_DT_PS
    w = 2 * math.pi * config.EXP_PHOTON_ENERGY / (1e12 * HBAR) * 1e-12  # rad / ps
    a = 0.03 * np.exp(-((t - 2.5) / 0.9) ** 2) * np.cos(w * (t - 2.5) + rng.uniform(0, 1))
    b = 0.012 * np.exp(-((t - 4.0) / 0.8) ** 2) * np.cos(w * (t - 4.0) + rng.uniform(0, 1))
    return a, b


def _exp_config(tmp_path, lt, t0="0", extra=""):
    a, b = synthetic_field()
    path = tmp_path / "field.dat"
    np.savetxt(path, np.c_[a, b])
    return PIFLUX.replace("laser_type cosine", f"laser_type {lt}\nexperimental_field {path}{extra}") \
        .replace("t0_offset 2", f"t0_offset {t0}").replace("photon_energy 5.25", "photon_energy 1")


def test_experimental_and_unknown_lasers():
    # without a measured field the experimental lasers are refused
    with pytest.raises(config.UnsupportedConfig):
        _laser("expB")
    with pytest.raises(ValueError):
        config.from_config(PIFLUX.replace("laser_type cosine", "laser_type dgauss")
                           .replace("system_type PiFlux", "system_type Honeycomb"))


def test_run_modes_shorten_the_double_laser_window():
    # reduced_duration (PiFluxDispatcher.cpp:45): 0.75 t_end for every mode
    full = _laser("dcos", t0="0.5").pulse
    cfg = PIFLUX.replace("laser_type cosine", "laser_type dcos").replace("t0_offset 2", "t0_offset 0.5") \
        .replace("n_laser_cycles 4", "n_laser_cycles 2").replace("occupations no", "occupations yes")
    red = config.from_config(cfg).pulse
    assert red.window_end == pytest.approx(0.75 * full.window_end)
    assert red.spline_cut == full.spline_cut
    # the cosine laser's window is not shortened
    cos_full = config.from_config(PIFLUX).pulse
    cos_red = config.from_config(PIFLUX.replace("split_current no", "split_current yes")).pulse
    assert cos_red.window_end == cos_full.window_end


def test_dirac_mapping():
    # DiracDispatcher (DiracDispatcher.cpp:16-79) and DiracSystem (DiracSystem.cpp:52-63)
    cfg = PIFLUX.replace("system_type PiFlux", "system_type Dirac")
    run = config.from_config(cfg)
    s, p, q = run.system, run.pulse, run.quad
    pe = 5.25
    assert s.kind == api.SYS_DIRAC3D and run.grid is None
    assert s.beta == pytest.approx(pe / (K_B * 300), rel=1e-15)
    assert s.fermi_energy == pytest.approx(118 / pe, rel=1e-15)
    assert s.inv_diag_relax == pytest.approx(1e15 * HBAR / (15 * pe), rel=1e-15)
    assert s.inv_offdiag_relax == 0.0
    ratio = HBAR * 1.5e6 / pe
    assert p.amplitude == pytest.approx(ratio * 1e11 * 1.6 / pe, rel=1e-15)
    # the cosine window ends with the laser (no extra cycle)
    assert (p.window_begin, p.window_end) == pytest.approx((2 * math.pi, 2 * math.pi + 8 * math.pi))
    assert p.n_measurements == 4 * 1024
    assert (q.max_k, q.n_z, q.n_kappa, q.threshold, q.n_splits) == (300.0, 51, 10, 1e-3, 100)
    # relaxation: FP64 RKF78; coherent: the closed-form Magnus step
    assert run.opts.stepper == api.STEPPER_RKF78 and (run.opts.abs_tol, run.opts.rel_tol) == (1e-12, 1e-8)
    coh = config.from_config(cfg.replace("diagonal_relaxation_time 15", "diagonal_relaxation_time -1"))
    assert coh.system.inv_diag_relax == 0.0 and coh.opts.stepper == api.STEPPER_DIRAC_MAGNUS
    # the Dirac dispatcher knows no Gaussian or double lasers
    for lt in ("gauss", "dcos", "dgaussA"):
        with pytest.raises(ValueError):
            config.from_config(cfg.replace("laser_type cosine", f"laser_type {lt}"))
    with pytest.raises(ValueError):
        config.from_config(cfg.replace("n_z 51\n", ""))


def test_measured_vector_potential_construction():
    """ExperimentalLaser's vector_potential: running sum, quartic tail that
    lands on zero with zero slope, zero padding."""
    a, _ = synthetic_field()
    dt = config.EXP_DT_PS
    A = config.measured_vector_potential(a, dt)
    n, bz, ne = a.size, config.EXP_BEGIN_ZERO, config.EXP_N_EXTRA
    assert A.size == n + ne + config.EXP_ZERO_BUFF + bz
    assert np.all(A[:bz] == 0) and np.all(A[A.size - bz - 1:] == 0)
    assert A[bz + n - 1] == pytest.approx(-dt * a.sum(), rel=1e-12)
    # the tail's polynomial reaches 0 with zero slope at T = (n_extra - 1) dt
    tail = A[bz + n - 1: bz + n - 1 + ne]
    assert abs(tail[-1]) <= 1e-12 * np.abs(A).max()
    # it is one quartic: its fit through the 16 points has p'(T) = 0 and
    # continues A with slope -E_last
    tt = np.arange(ne) * dt
    c = np.polynomial.polynomial.polyfit(tt, tail, 4)
    d = np.polynomial.polynomial.polyder(c)
    scale = np.abs(tail).max() / tt[-1]
    assert abs(np.polynomial.polynomial.polyval(tt[-1], d)) <= 1e-8 * scale
    assert np.polynomial.polynomial.polyval(0.0, d) == pytest.approx(-a[-1], rel=1e-6, abs=1e-8 * scale)


@pytest.mark.parametrize("lt,t0", [("exp", "0"), ("expA", "0"), ("expB", "0.4"), ("exp", "-0.3")])
def test_experimental_laser_matches_the_oracle(tmp_path, lt, t0):
    """The config reader's experimental pulse (the engine's spline samples)
    against the oracle's independent restatement of ExperimentalLaser."""
    from oracle import hhg_oracle as O
    run = config.from_config(_exp_config(tmp_path, lt, t0))
    p = run.pulse
    assert p.kind == api.PULSE_SPLINE and (p.deriv_begin, p.deriv_end) == (0.0, 0.0)
    pe_l = 1.0 * config.EXP_PHOTON_ENERGY
    # the system takes the experimental photon energy too (get_photon_energy)
    assert run.system.fermi_energy == pytest.approx(118 / pe_l)
    lattice = math.sqrt(3) * HBAR * 1.5e6 / (pe_l * 300)
    assert run.lattice_constant == pytest.approx(lattice, rel=1e-15)
    a, b = synthetic_field()
    sp, t_end = O.experimental_laser(a, b, config.EXP_DT_PS, pe_l, 1.6, lattice, float(t0),
                                     {"exp": "both", "expA": "A", "expB": "B"}[lt])
    assert p.spline_cut == pytest.approx(t_end, rel=1e-15)
    assert (p.window_begin, p.window_end) == (0.0, pytest.approx(t_end, rel=1e-15))
    assert p.n_samples == sp.y.size and p.sample_dt == pytest.approx(sp.dt, rel=1e-15)
    scale = np.abs(sp.y).max()
    assert scale > 0
    assert np.max(np.abs(p._samples - sp.y)) <= 1e-13 * scale
    # and A(t) between the knots
    t = np.linspace(0.0, 1.1 * t_end, 777)
    assert np.max(np.abs(api.pulse_values(p, t) - O.laser(sp, t))) <= 1e-12 * scale


def test_experimental_laser_windows(tmp_path):
    # PiFlux shortens the window for the run modes, Honeycomb does not
    full = config.from_config(_exp_config(tmp_path, "exp")).pulse
    red = config.from_config(_exp_config(tmp_path, "exp").replace("occupations no",
                                                                  "occupations yes")).pulse
    assert red.window_end == pytest.approx(0.75 * full.window_end)
    hc = config.from_config(_exp_config(tmp_path, "exp").replace("system_type PiFlux",
                                                                 "system_type Honeycomb")
                            .replace("occupations no", "occupations yes")).pulse
    assert hc.window_end == pytest.approx(full.window_end)
    # the data's spacing and photon energy are keys of their own
    alt = config.from_config(_exp_config(tmp_path, "exp",
                                         extra="\nexperimental_photon_energy 5.0")).pulse
    assert alt.sample_dt == pytest.approx(full.sample_dt * 5.0 / config.EXP_PHOTON_ENERGY)
