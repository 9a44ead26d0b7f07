"""CPU checks of the C ABI: the library loads and exports every entry point
include/hhg_gpu.h declares, the ctypes layouts equal the C layouts, and the
host-only entry points (Gauss rules, grid rows, descriptor validation) agree
with the oracle.  No kernel is launched here."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from higherharmonics_b200 import api
from oracle import hhg_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hhg_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hhg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(api.EXPORTED)
    assert lib.hhg_abi_version() == api.ABI_VERSION


def _c_layout():
    structs = {"hhg_system_desc": ["kind", "hopping", "velocity", "mass", "pol_x", "pol_y"],
               "hhg_pulse_desc": ["kind", "n_measurements", "n_subdivisions", "amplitude",
                                  "n_cycles", "t_begin", "phase", "window_begin", "window_end",
                                  "energy_scale"],
               "hhg_grid_desc": ["kind", "n1", "n2", "x_lo", "x_hi", "y_lo", "y_hi", "rows",
                                 "n_rows"],
               "hhg_solver_opts": ["stepper", "precision", "proposer", "magnus_substeps",
                                   "abs_tol", "rel_tol", "max_failed_steps",
                                   "max_attempts_per_interval", "tile_k", "block_threads",
                                   "mlp", "mlp_every", "coarsen_div"],
               "hhg_mlp": ["params", "in_mu", "in_isig", "out_mu", "out_sigma", "level_margin",
                           "reserved"],
               "hhg_train_opts": ["epochs", "batch", "lr", "beta1", "beta2", "eps", "lr_final",
                                  "reserved", "seed"],
               "hhg_tune_report": ["n_candidates", "best", "tile_k", "grid", "kernel_ms"],
               "hhg_stats": ["k_points", "trajectories", "attempted_steps", "rejected_steps",
                             "failed_trajectories", "poly_degree", "items", "kernel_ms",
                             "total_ms"],
               "hhg_kappa_quad": ["max_k", "threshold", "n_z", "n_kappa", "n_splits",
                                  "max_halvings", "z_first", "z_count"],
               "hhg_kappa_stats": ["trajectories", "speculative", "rounds", "splits", "unconverged",
                                   "max_level", "launches", "reserved"]}
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(){"]
    for s, fields in structs.items():
        src.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for f in fields:
            src.append(f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "l")
        subprocess.run(["/usr/bin/gcc", "-std=c99", "-o", exe, c], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        a, b, c = line.split()
        res[(a, b)] = int(c)
    return res


def test_ctypes_layout_matches_c():
    lay = _c_layout()
    for cname, py in [("hhg_system_desc", api.SystemDesc), ("hhg_pulse_desc", api.PulseDesc),
                      ("hhg_grid_desc", api.GridDesc), ("hhg_solver_opts", api.SolverOpts),
                      ("hhg_stats", api.Stats), ("hhg_mlp", api.Mlp),
                      ("hhg_train_opts", api.TrainOpts), ("hhg_tune_report", api.TuneReport),
                      ("hhg_kappa_quad", api.KappaQuad), ("hhg_kappa_stats", api.KappaStats)]:
        assert lay[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            if (cname, fname) in lay:
                assert lay[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_gauss_rule_matches_oracle_bitwise():
    for n in (4, 30, 64, 256, 1000):
        x, w = api.gauss_legendre(n)
        xo, wo = O.gauss_legendre(n)
        assert np.array_equal(x, xo) and np.array_equal(w, wo)


@pytest.mark.parametrize("case", ["tensor", "rhombic", "piflux3d", "hex", "dirac2d", "piflux2d"])
def test_grid_rows_match_oracle(case):
    if case == "tensor":
        sys_ = api.system(api.SYS_DIRAC2D, velocity=10.0, mass=0.5)
        rows = api.grid_rows(sys_, api.grid_tensor(12, 7, -2, 2, -1, 3))
        ref = O.grid_tensor(O.model(O.DIRAC2D, velocity=10.0, mass=0.5), 12, 7, -2, 2, -1, 3)
    elif case == "rhombic":
        sys_ = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1)
        rows = api.grid_rhombic(16, 16) and api.grid_rows(sys_, api.grid_rhombic(16, 16))
        ref = O.grid_rhombic(O.model(O.HONEYCOMB, hopping=1.0, mass=0.1), 16, 16)
    elif case == "piflux3d":
        sys_ = api.system(api.SYS_PIFLUX3D, hopping=1.0)
        rows = api.grid_rows(sys_, api.grid_piflux3d_ref(32, 4))
        ref = O.grid_piflux3d_ref(O.model(O.PIFLUX3D, hopping=1.0), 32, 4)
        assert rows.shape[0] == 151552  # 64 z-nodes x 2368 xy-nodes
    elif case == "hex":
        sys_ = api.system(api.SYS_HONEYCOMB, hopping=1.0)
        rows = api.grid_rows(sys_, api.grid_honeycomb_hex_ref(64))
        ref = O.grid_honeycomb_hex_ref(O.model(O.HONEYCOMB, hopping=1.0), 64)
        assert rows.shape[0] == 16384
    elif case == "dirac2d":
        sys_ = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
        rows = api.grid_rows(sys_, api.grid_tensor(64, 64, -2, 2, -2, 2))
        ref = O.grid_tensor(O.model(O.DIRAC2D, velocity=1.0, mass=0.05), 64, 64, -2, 2, -2, 2)
    else:
        sys_ = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(0.6, 0.8))
        rows = api.grid_rows(sys_, api.grid_tensor(16, 16, -3.14, 3.14, -3.14, 3.14))
        ref = O.grid_tensor(O.model(O.PIFLUX2D, hopping=1.0, pol=(0.6, 0.8)), 16, 16, -3.14,
                            3.14, -3.14, 3.14)
    assert rows.shape == ref.shape
    assert np.array_equal(rows, ref)


def test_piflux3d_reference_rescue_quirk():
    """+k_z slices with cos k_z < 0 start from cos k_z (1 - 0.5e-8) (the
    rescue at PiFlux.cpp:812-816 leaves cos_z scaled); -k_z slices do not."""
    sys_ = api.system(api.SYS_PIFLUX3D, hopping=1.0)
    rows = api.grid_rows(sys_, api.grid_piflux3d_ref(4, 2))
    kz = rows[:, 2]
    cx, cy, cz = np.cos(rows[:, 0]), np.cos(rows[:, 1]), np.cos(kz)
    plus = (kz > 0) & (cz < 0)
    czr = cz * (1 - 0.5e-8)
    s_rescued = -czr / np.sqrt(cx ** 2 + cy ** 2 + czr ** 2)
    s_plain = -cz / np.sqrt(cx ** 2 + cy ** 2 + cz ** 2)
    assert np.allclose(rows[plus, 6], s_rescued[plus], rtol=1e-15, atol=1e-16)
    minus = (kz < 0) & (cz < 0)
    assert np.allclose(rows[minus, 6], s_plain[minus], rtol=1e-15, atol=1e-16)
    assert not np.allclose(rows[plus, 6], s_plain[plus], rtol=1e-12, atol=0)


def test_explicit_rows_roundtrip():
    rows = np.random.default_rng(1).normal(size=(10, 8))
    g, keep = api.grid_explicit(rows)
    out = api.grid_rows(api.system(api.SYS_DIRAC2D, velocity=1.0), g)
    assert np.array_equal(out, rows)


def test_host_validation_errors():
    L = api.load_library()
    sys_ = api.system(api.SYS_DIRAC2D, velocity=1.0)
    n = ctypes.c_int64(0)
    bad_grid = api.grid_tensor(0, 4, -1, 1, -1, 1)
    assert L.hhg_grid_rows(ctypes.byref(sys_), ctypes.byref(bad_grid), None, ctypes.byref(n)) == api.BAD_CONFIG
    bad_sys = api.system(17, velocity=1.0)
    good_grid = api.grid_tensor(4, 4, -1, 1, -1, 1)
    assert L.hhg_grid_rows(ctypes.byref(bad_sys), ctypes.byref(good_grid), None, ctypes.byref(n)) == api.BAD_CONFIG
    nan_sys = api.system(api.SYS_DIRAC2D, velocity=float("nan"))
    assert L.hhg_grid_rows(ctypes.byref(nan_sys), ctypes.byref(good_grid), None, ctypes.byref(n)) == api.BAD_CONFIG
    x = np.zeros(4)
    assert L.hhg_gauss_legendre(0, x.ctypes.data_as(api._D), x.ctypes.data_as(api._D)) == api.BAD_CONFIG


def test_create_without_device_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    with pytest.raises(api.HHGError) as ei:
        api.Engine(0)
    assert ei.value.status == api.CUDA_ERROR
