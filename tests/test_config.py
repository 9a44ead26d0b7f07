"""The reference's parameter files -> descriptors (higherharmonics_b200.config):
parsing, the unit mapping of the reference's dispatchers and constructors,
and the configurations the engine refuses.  CPU only."""
import math

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
    (("laser_type cosine", "laser_type powerlaw1"), config.UnsupportedConfig),
    (("laser_type cosine", "laser_type expA"), config.UnsupportedConfig),
    (("system_type PiFlux", "system_type Dirac"), config.UnsupportedConfig),
    (("occupations no", "occupations only"), config.UnsupportedConfig),
    (("split_current no", "split_current yes"), config.UnsupportedConfig),
    (("system_type PiFlux", "system_type Graphene"), ValueError),
    (("E_F 118\n", ""), ValueError),
])
def test_refused_configurations(edit, exc):
    with pytest.raises(exc):
        config.from_config(PIFLUX.replace(*edit))
