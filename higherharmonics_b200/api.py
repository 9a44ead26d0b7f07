"""ctypes binding of the C ABI (include/hhg_gpu.h) and thin Python helpers.

The compute path is ``libhhg_gpu.so`` (sm_100a kernels); this module only
marshals descriptors.  There is no CPU fallback: if the library is missing or
no CUDA device is visible, every call raises.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhhg_gpu.so")

# enums (hhg_gpu.h)
OK, BAD_CONFIG, STEP_LIMIT, NONFINITE, CUDA_ERROR, UNSUPPORTED = range(6)
STATUS_NAMES = {0: "HHG_OK", 1: "HHG_BAD_CONFIG", 2: "HHG_STEP_LIMIT", 3: "HHG_NONFINITE",
                4: "HHG_CUDA_ERROR", 5: "HHG_UNSUPPORTED"}
SYS_DIRAC2D, SYS_PIFLUX2D, SYS_PIFLUX3D, SYS_HONEYCOMB, SYS_DIRAC3D = range(5)
(GRID_TENSOR_GL, GRID_RHOMBIC_GL, GRID_PIFLUX3D_REF, GRID_HONEYCOMB_HEX_REF, GRID_EXPLICIT,
 GRID_PIFLUX3D_OCCUPATION, GRID_PIFLUX3D_CUBE, GRID_PIFLUX3D_DEBUG, GRID_DIRAC3D_DEBUG) = range(9)
N_DEBUG_POINTS = 25  # n_debug_points (GlobalDefinitions.hpp)
KOUT_BLOCH, KOUT_OCCUPATIONS, KOUT_CURRENT = 0, 1, 2
STEPPER_RKF78, STEPPER_MAGNUS4, STEPPER_DIRAC_MAGNUS = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
PROPOSER_NONE, PROPOSER_CARRY, PROPOSER_LEARNED, PROPOSER_LOCKSTEP = 0, 1, 2, 3
PULSE_COSINE, PULSE_CONTINUOUS, PULSE_GAUSS, PULSE_SPLINE = 0, 1, 2, 3

EXPORTED = [
    "hhg_abi_version", "hhg_gpu_create", "hhg_gpu_destroy", "hhg_last_error",
    "hhg_default_solver_opts", "hhg_gauss_legendre", "hhg_grid_rows",
    "hhg_gpu_current_density", "hhg_gpu_spectrum", "hhg_plan_create", "hhg_plan_destroy",
    "hhg_plan_j_length", "hhg_plan_execute_async", "hhg_plan_device_j", "hhg_plan_fetch",
    "hhg_plan_spectrum_async", "hhg_plan_fetch_spectrum", "hhg_measure_fp64_peak",
    "hhg_gpu_current_density_noalloc", "hhg_noalloc_status",
    "hhg_learned_collect", "hhg_default_train_opts", "hhg_mlp_init", "hhg_mlp_train",
    "hhg_mlp_gradients", "hhg_mlp_predict", "hhg_plan_execute_graph", "hhg_plan_autotune", "hhg_measure_fp32_peak",
    "hhg_gpu_k_resolved", "hhg_gpu_split_current", "hhg_gpu_spectrum_welch", "hhg_pulse_values",
    "hhg_gpu_dirac_current_density", "hhg_gpu_trapezoidal_fft",
]
TUNE_MAX = 16
ABI_VERSION = 4
MLP_INPUTS, MLP_HIDDEN = 8, 64
MLP_N_PARAMS = 64 * 8 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1
HIST_FIELDS = 12
# slices of hhg_mlp.params: w1[64][8], b1, w2[64][64], b2, w3[64][64], b3, w4[64], b4
MLP_LAYOUT = [("w1", (64, 8)), ("b1", (64,)), ("w2", (64, 64)), ("b2", (64,)),
              ("w3", (64, 64)), ("b3", (64,)), ("w4", (64,)), ("b4", (1,))]


class SystemDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("hopping", ctypes.c_double), ("velocity", ctypes.c_double),
                ("mass", ctypes.c_double), ("pol_x", ctypes.c_double), ("pol_y", ctypes.c_double),
                ("beta", ctypes.c_double), ("fermi_energy", ctypes.c_double),
                ("inv_diag_relax", ctypes.c_double), ("inv_offdiag_relax", ctypes.c_double)]


class PulseDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n_measurements", ctypes.c_int32),
                ("n_subdivisions", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("amplitude", ctypes.c_double), ("n_cycles", ctypes.c_double),
                ("t_begin", ctypes.c_double), ("phase", ctypes.c_double),
                ("window_begin", ctypes.c_double), ("window_end", ctypes.c_double),
                ("energy_scale", ctypes.c_double), ("samples", ctypes.POINTER(ctypes.c_double)),
                ("n_samples", ctypes.c_int64), ("sample_dt", ctypes.c_double),
                ("deriv_begin", ctypes.c_double), ("deriv_end", ctypes.c_double),
                ("spline_cut", ctypes.c_double)]


class GridDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n1", ctypes.c_int32), ("n2", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("x_lo", ctypes.c_double),
                ("x_hi", ctypes.c_double), ("y_lo", ctypes.c_double), ("y_hi", ctypes.c_double),
                ("rows", ctypes.POINTER(ctypes.c_double)), ("n_rows", ctypes.c_int64)]


class Mlp(ctypes.Structure):
    """hhg_mlp: the learned step-size proposer's weights and standardisation."""
    _fields_ = [("params", ctypes.c_float * MLP_N_PARAMS),
                ("in_mu", ctypes.c_float * MLP_INPUTS), ("in_isig", ctypes.c_float * MLP_INPUTS),
                ("out_mu", ctypes.c_float), ("out_sigma", ctypes.c_float),
                ("level_margin", ctypes.c_float), ("reserved", ctypes.c_float)]

    def param_array(self) -> np.ndarray:
        """Writable float32 view of params."""
        return np.ctypeslib.as_array(self.params)

    def tensors(self) -> dict:
        """params split into the named layer arrays (copies, float64)."""
        flat = self.param_array().astype(np.float64)
        out, o = {}, 0
        for name, shape in MLP_LAYOUT:
            n = int(np.prod(shape))
            out[name] = flat[o:o + n].reshape(shape)
            o += n
        return out


class SolverOpts(ctypes.Structure):
    _fields_ = [("stepper", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("proposer", ctypes.c_int32), ("magnus_substeps", ctypes.c_int32),
                ("abs_tol", ctypes.c_double), ("rel_tol", ctypes.c_double),
                ("max_failed_steps", ctypes.c_int32), ("max_attempts_per_interval", ctypes.c_int32),
                ("tile_k", ctypes.c_int32), ("block_threads", ctypes.c_int32),
                ("mlp", ctypes.POINTER(Mlp)), ("mlp_every", ctypes.c_int32),
                ("coarsen_div", ctypes.c_int32)]


class TrainOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("lr_final", ctypes.c_float), ("reserved", ctypes.c_int32),
                ("seed", ctypes.c_uint64)]


class TuneReport(ctypes.Structure):
    _fields_ = [("n_candidates", ctypes.c_int32), ("best", ctypes.c_int32),
                ("tile_k", ctypes.c_int32 * TUNE_MAX), ("grid", ctypes.c_int32 * TUNE_MAX),
                ("kernel_ms", ctypes.c_double * TUNE_MAX)]

    def as_list(self) -> list:
        return [{"tile_k": self.tile_k[i], "grid": self.grid[i], "kernel_ms": self.kernel_ms[i]}
                for i in range(self.n_candidates)]


class Stats(ctypes.Structure):
    _fields_ = [("k_points", ctypes.c_int64), ("trajectories", ctypes.c_int64),
                ("attempted_steps", ctypes.c_int64), ("rejected_steps", ctypes.c_int64),
                ("failed_trajectories", ctypes.c_int64), ("poly_degree", ctypes.c_int32),
                ("items", ctypes.c_int32), ("kernel_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class KappaQuad(ctypes.Structure):
    """hhg_kappa_quad: the Dirac-3D momentum quadrature (k_z slices x the
    adaptive kappa rule of DiracSystem::compute_current_density)."""
    _fields_ = [("max_k", ctypes.c_double), ("threshold", ctypes.c_double),
                ("n_z", ctypes.c_int32), ("n_kappa", ctypes.c_int32),
                ("n_splits", ctypes.c_int32), ("max_halvings", ctypes.c_int32),
                ("z_first", ctypes.c_int32), ("z_count", ctypes.c_int32)]


class KappaStats(ctypes.Structure):
    _fields_ = [("trajectories", ctypes.c_int64), ("speculative", ctypes.c_int64),
                ("rounds", ctypes.c_int32), ("splits", ctypes.c_int32),
                ("unconverged", ctypes.c_int32), ("max_level", ctypes.c_int32),
                ("launches", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


def kappa_quad(max_k: float, n_z: int, n_kappa: int = 10, threshold: float = 1e-3,
               n_splits: int = 100, max_halvings: int = 0, z_first: int = 0,
               z_count: int = 0) -> KappaQuad:
    """Defaults: the reference's DiracDispatcher (n_kappa 10, threshold 1e-3,
    DiracDispatcher.cpp:13-14) and split_integrate<100>; z_count > 0 takes the
    slices z_first .. z_first + z_count - 1 only (one rank's block)."""
    return KappaQuad(max_k, threshold, n_z, n_kappa, n_splits, max_halvings, z_first, z_count)


class HHGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None
_D = ctypes.POINTER(ctypes.c_double)


def load_library() -> ctypes.CDLL:
    """Load libhhg_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -c 'import __graft_entry__ as g; g.build()'` or "
                              "`make -C higherharmonics_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        L.hhg_last_error.restype = ctypes.c_char_p
        L.hhg_last_error.argtypes = [ctypes.c_void_p]
        L.hhg_gpu_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        L.hhg_gpu_destroy.argtypes = [ctypes.c_void_p]
        L.hhg_plan_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(SystemDesc),
                                      ctypes.POINTER(PulseDesc), ctypes.c_int,
                                      ctypes.POINTER(GridDesc), ctypes.POINTER(SolverOpts),
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.hhg_plan_destroy.argtypes = [ctypes.c_void_p]
        L.hhg_plan_j_length.argtypes = [ctypes.c_void_p]
        L.hhg_plan_j_length.restype = ctypes.c_int64
        L.hhg_plan_execute_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.hhg_plan_device_j.argtypes = [ctypes.c_void_p]
        L.hhg_plan_device_j.restype = ctypes.c_void_p
        L.hhg_plan_fetch.argtypes = [ctypes.c_void_p, _D, ctypes.POINTER(Stats)]
        L.hhg_gpu_current_density.argtypes = [ctypes.c_void_p, ctypes.POINTER(SystemDesc),
                                              ctypes.POINTER(PulseDesc), ctypes.c_int,
                                              ctypes.POINTER(GridDesc), ctypes.POINTER(SolverOpts),
                                              _D, ctypes.POINTER(Stats)]
        L.hhg_gpu_spectrum.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, _D, _D, _D]
        L.hhg_grid_rows.argtypes = [ctypes.POINTER(SystemDesc), ctypes.POINTER(GridDesc), _D,
                                    ctypes.POINTER(ctypes.c_int64)]
        L.hhg_gauss_legendre.argtypes = [ctypes.c_int, _D, _D]
        L.hhg_plan_spectrum_async.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.hhg_plan_fetch_spectrum.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.hhg_measure_fp64_peak.argtypes = [ctypes.c_void_p, _D]
        L.hhg_measure_fp32_peak.argtypes = [ctypes.c_void_p, _D]
        L.hhg_gpu_current_density_noalloc.argtypes = [
            ctypes.POINTER(SystemDesc), ctypes.POINTER(PulseDesc), ctypes.c_void_p, ctypes.c_int64,
            ctypes.POINTER(SolverOpts), ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Stats),
            ctypes.c_char_p, ctypes.c_size_t]
        L.hhg_noalloc_status.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats), ctypes.c_char_p,
                                         ctypes.c_size_t]
        L.hhg_default_solver_opts.argtypes = [ctypes.POINTER(SolverOpts)]
        L.hhg_gpu_k_resolved.argtypes = [ctypes.c_void_p, ctypes.POINTER(SystemDesc),
                                         ctypes.POINTER(PulseDesc), ctypes.POINTER(GridDesc),
                                         ctypes.POINTER(SolverOpts), ctypes.c_int, _D,
                                         ctypes.POINTER(Stats)]
        L.hhg_gpu_split_current.argtypes = [ctypes.c_void_p, ctypes.POINTER(SystemDesc),
                                            ctypes.POINTER(PulseDesc), ctypes.POINTER(GridDesc),
                                            ctypes.POINTER(SolverOpts), ctypes.c_double, _D, _D,
                                            ctypes.POINTER(Stats)]
        L.hhg_gpu_spectrum_welch.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, _D, _D, _D]
        L.hhg_pulse_values.argtypes = [ctypes.POINTER(PulseDesc), _D, ctypes.c_int64, _D]
        L.hhg_gpu_trapezoidal_fft.argtypes = [ctypes.c_void_p, _D, ctypes.c_int64, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, _D, _D, _D]
        L.hhg_gpu_dirac_current_density.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(SystemDesc), ctypes.POINTER(PulseDesc),
            ctypes.POINTER(KappaQuad), ctypes.POINTER(SolverOpts), _D, ctypes.POINTER(KappaStats),
            ctypes.POINTER(Stats)]
        _F = ctypes.POINTER(ctypes.c_float)
        L.hhg_learned_collect.argtypes = [ctypes.c_void_p, ctypes.POINTER(SystemDesc),
                                          ctypes.POINTER(PulseDesc), ctypes.c_int,
                                          ctypes.POINTER(GridDesc), ctypes.POINTER(SolverOpts),
                                          ctypes.c_int, _F, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(Stats)]
        L.hhg_default_train_opts.argtypes = [ctypes.POINTER(TrainOpts)]
        L.hhg_plan_execute_graph.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.hhg_plan_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(TuneReport)]
        L.hhg_mlp_init.argtypes = [ctypes.c_uint64, _F, ctypes.c_int64, ctypes.POINTER(Mlp)]
        L.hhg_mlp_train.argtypes = [ctypes.c_void_p, _F, ctypes.c_int64, ctypes.POINTER(TrainOpts),
                                    ctypes.POINTER(Mlp), _F, _D]
        L.hhg_mlp_gradients.argtypes = [ctypes.c_void_p, _F, ctypes.c_int64, ctypes.POINTER(Mlp),
                                        _F, _F]
        L.hhg_mlp_predict.argtypes = [ctypes.c_void_p, _F, ctypes.c_int64, ctypes.POINTER(Mlp),
                                      ctypes.c_int, _F]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _records(rec) -> np.ndarray:
    rec = np.ascontiguousarray(rec, dtype=np.float32)
    assert rec.ndim == 2 and rec.shape[1] == HIST_FIELDS, rec.shape
    return rec


# ---------------------------------------------------------------------------
# descriptor helpers
# ---------------------------------------------------------------------------
def system(kind: int, hopping=0.0, velocity=0.0, mass=0.0, pol=(1.0, 0.0), *, beta=0.0,
           fermi_energy=0.0, inv_diag_relax=0.0, inv_offdiag_relax=0.0) -> SystemDesc:
    """System descriptor.  beta = photon_energy / (k_B T) (0: T = 0),
    fermi_energy = E_F / photon_energy, inv_*_relax = 1e15 hbar / (tau
    photon_energy) (PiFlux.cpp:56-71); inv_diag_relax > 0 selects the
    relaxation right-hand side."""
    return SystemDesc(kind, 0, hopping, velocity, mass, pol[0], pol[1], beta, fermi_energy,
                      inv_diag_relax, inv_offdiag_relax)


def cosine_pulse(amplitude: float, n_cycles: float, n_measurements: int, *, t_begin=0.0,
                 phase=0.0, window=None, energy_scale=1.0, n_subdivisions=50) -> PulseDesc:
    """CosineLaser + its TimeIntegrationConfig.  ``window`` defaults to the
    pulse itself, [t_begin, t_begin + 2 pi n_cycles] (DiracDispatcher.cpp:37);
    the PiFlux/Honeycomb dispatchers add one cycle (PiFluxDispatcher.cpp:53)."""
    if window is None:
        window = (t_begin, t_begin + 2 * math.pi * n_cycles)
    return PulseDesc(PULSE_COSINE, n_measurements, n_subdivisions, 0, amplitude, n_cycles,
                     t_begin, phase, window[0], window[1], energy_scale)


def continuous_pulse(amplitude: float, n_measurements: int, window, *, phase=0.0,
                     energy_scale=1.0, n_subdivisions=50) -> PulseDesc:
    """ContinuousLaser: A(t) = A0 sin(t + phase) (ContinuousLaser.cpp); the
    reference samples it on [-n_cycles pi, n_cycles pi] (PiFluxDispatcher.cpp:46-48)."""
    return PulseDesc(PULSE_CONTINUOUS, n_measurements, n_subdivisions, 0, amplitude, 0.0, 0.0,
                     phase, window[0], window[1], energy_scale)


def gauss_pulse(amplitude: float, n_cycles: float, n_measurements: int, *, t_begin=0.0,
                phase=0.0, window=None, energy_scale=1.0, n_subdivisions=50) -> PulseDesc:
    """GaussLaser: A0 exp(-(t - c)^2 / 2 s^2) sin(t + phase), c = t_begin +
    3 pi n_cycles, s = pi n_cycles / sqrt(2 ln 20) (GaussLaser.cpp); the
    default window is the laser's [t_begin, t_begin + 6 pi n_cycles]."""
    if window is None:
        window = (t_begin, t_begin + 6 * math.pi * n_cycles)
    return PulseDesc(PULSE_GAUSS, n_measurements, n_subdivisions, 0, amplitude, n_cycles,
                     t_begin, phase, window[0], window[1], energy_scale)


def spline_pulse(samples, t_begin: float, sample_dt: float, n_measurements: int, window, *,
                 cut=None, deriv=(math.nan, math.nan), amplitude=1.0, energy_scale=1.0,
                 n_subdivisions=50) -> PulseDesc:
    """A(t) = amplitude * s(t) for t <= cut (default: the last sample), 0
    after: s is the clamped cubic spline through the samples at t_begin +
    k sample_dt with end slopes ``deriv`` (NaN: estimated), as the
    reference's spline lasers (Laser.hpp:32-37).  The descriptor keeps a
    reference to the sample array."""
    y = np.ascontiguousarray(samples, dtype=np.float64)
    if cut is None:
        cut = t_begin + (y.size - 1) * sample_dt
    d = PulseDesc(PULSE_SPLINE, n_measurements, n_subdivisions, 0, amplitude, 0.0, t_begin, 0.0,
                  window[0], window[1], energy_scale, y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                  y.size, sample_dt, deriv[0], deriv[1], cut)
    d._samples = y
    return d


def grid_tensor(n1, n2, x_lo, x_hi, y_lo, y_hi) -> GridDesc:
    return GridDesc(GRID_TENSOR_GL, n1, n2, 0, x_lo, x_hi, y_lo, y_hi, None, 0)


def grid_rhombic(n1, n2) -> GridDesc:
    return GridDesc(GRID_RHOMBIC_GL, n1, n2, 0, 0, 0, 0, 0, None, 0)


def grid_piflux3d_ref(z_range=32, n_coarse=4) -> GridDesc:
    return GridDesc(GRID_PIFLUX3D_REF, z_range, n_coarse, 0, 0, 0, 0, 0, None, 0)


def grid_honeycomb_hex_ref(n_k=64) -> GridDesc:
    return GridDesc(GRID_HONEYCOMB_HEX_REF, n_k, 0, 0, 0, 0, 0, 0, None, 0)


def grid_piflux3d_occupation(n: int) -> GridDesc:
    """PiFlux::compute_occupation_numbers' N x N grid (PiFlux.cpp:909-953)."""
    return GridDesc(GRID_PIFLUX3D_OCCUPATION, n, 0, 0, 0, 0, 0, 0, None, 0)


def grid_piflux3d_cube(n: int) -> GridDesc:
    """PiFlux::current_per_energy's N^3 grid and its -z mirror (PiFlux.cpp:955-1035)."""
    return GridDesc(GRID_PIFLUX3D_CUBE, n, 0, 0, 0, 0, 0, 0, None, 0)


def grid_piflux3d_debug() -> GridDesc:
    """The 25 momenta of PiFlux::compute_current_density_debug (PiFlux.cpp:320-371):
    k = (pi/2, pi/2 - 0.02 pi i, 0.49 pi), weight 1."""
    return GridDesc(GRID_PIFLUX3D_DEBUG, 0, 0, 0, 0, 0, 0, 0, None, 0)


def grid_dirac3d_debug(n_z: int, max_k: float) -> GridDesc:
    """The 25 (k_z, kappa) of DiracSystem::compute_current_density_debug
    (DiracSystem.cpp:333-363): k_z = (n_z/10) 2 max_k / n_z, kappa_i =
    (i + 1) kappa_max / 26, weighted by k_z kappa / |k|."""
    return GridDesc(GRID_DIRAC3D_DEBUG, n_z, 0, 0, 0.0, max_k, 0, 0, None, 0)


def pulse_values(pulse: PulseDesc, t) -> np.ndarray:
    """A(t) of a pulse as the engine stages it (host)."""
    t = np.ascontiguousarray(np.atleast_1d(t), dtype=np.float64)
    out = np.zeros_like(t)
    st = load_library().hhg_pulse_values(ctypes.byref(pulse), _ptr(t), t.size, _ptr(out))
    if st != OK:
        raise HHGError(st, "hhg_pulse_values")
    return out


def grid_explicit(rows: np.ndarray) -> tuple[GridDesc, np.ndarray]:
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    assert rows.ndim == 2 and rows.shape[1] == 8
    return GridDesc(GRID_EXPLICIT, 0, 0, 0, 0, 0, 0, 0, _ptr(rows), rows.shape[0]), rows


def solver(abs_tol=1e-12, rel_tol=1e-8, stepper=STEPPER_RKF78, precision=PREC_FP64,
           proposer=PROPOSER_NONE, magnus_substeps=1, tile_k=0, mlp: "Mlp | None" = None,
           mlp_every=16, coarsen_div=0) -> SolverOpts:
    o = SolverOpts()
    load_library().hhg_default_solver_opts(ctypes.byref(o))
    o.abs_tol, o.rel_tol = abs_tol, rel_tol
    o.stepper, o.precision, o.proposer = stepper, precision, proposer
    o.magnus_substeps, o.tile_k = magnus_substeps, tile_k
    if mlp is not None:
        o.mlp = ctypes.pointer(mlp)
        o._mlp_ref = mlp  # keep the network alive as long as the options
    o.mlp_every = mlp_every
    o.coarsen_div = coarsen_div
    return o


def train_opts(**kw) -> TrainOpts:
    o = TrainOpts()
    load_library().hhg_default_train_opts(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def mlp_init(seed: int = 1, records: np.ndarray | None = None) -> Mlp:
    """Initial weights from `seed` and, with records, the fitted standardisation."""
    net = Mlp()
    if records is None:
        st = load_library().hhg_mlp_init(seed, None, 0, ctypes.byref(net))
    else:
        rec = _records(records)
        st = load_library().hhg_mlp_init(seed, _fptr(rec), rec.shape[0], ctypes.byref(net))
    if st != OK:
        raise HHGError(st, "hhg_mlp_init")
    return net


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    st = load_library().hhg_gauss_legendre(n, _ptr(x), _ptr(w))
    if st != OK:
        raise HHGError(st, "hhg_gauss_legendre")
    return x, w


def grid_rows(sys: SystemDesc, grid: GridDesc) -> np.ndarray:
    L = load_library()
    n = ctypes.c_int64(0)
    st = L.hhg_grid_rows(ctypes.byref(sys), ctypes.byref(grid), None, ctypes.byref(n))
    if st != OK:
        raise HHGError(st, "hhg_grid_rows")
    out = np.zeros((n.value, 8))
    st = L.hhg_grid_rows(ctypes.byref(sys), ctypes.byref(grid), _ptr(out), ctypes.byref(n))
    if st != OK:
        raise HHGError(st, "hhg_grid_rows")
    return out


# ---------------------------------------------------------------------------
# context / plans
# ---------------------------------------------------------------------------
class Engine:
    """One hhg_ctx on one device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.ctx = ctypes.c_void_p()
        st = self.lib.hhg_gpu_create(ctypes.byref(self.ctx), device)
        if st != OK:
            raise HHGError(st, f"hhg_gpu_create(device={device}) failed")

    def _check(self, st: int, what: str):
        if st != OK:
            raise HHGError(st, f"{what}: {self.lib.hhg_last_error(self.ctx).decode()}")

    def close(self):
        if self.ctx:
            self.lib.hhg_gpu_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def current_density(self, sys: SystemDesc, pulses, grid: GridDesc,
                        opts: SolverOpts | None = None) -> tuple[np.ndarray, Stats]:
        pulses = list(pulses) if not isinstance(pulses, PulseDesc) else [pulses]
        arr = (PulseDesc * len(pulses))(*pulses)
        n = sum(p.n_measurements + 1 for p in pulses)
        j = np.zeros(n)
        st = Stats()
        o = opts if opts is not None else solver()
        self._check(self.lib.hhg_gpu_current_density(self.ctx, ctypes.byref(sys), arr,
                                                     len(pulses), ctypes.byref(grid),
                                                     ctypes.byref(o), _ptr(j), ctypes.byref(st)),
                    "hhg_gpu_current_density")
        return j, st

    def spectrum(self, j: np.ndarray, n_measurements: int, t_begin: float, t_end: float):
        j = np.ascontiguousarray(j, dtype=np.float64)
        n_fft = 4 * (n_measurements + 1) + 1
        re = np.zeros(n_fft)
        im = np.zeros(n_fft)
        fr = np.zeros(n_fft)
        self._check(self.lib.hhg_gpu_spectrum(self.ctx, _ptr(j), n_measurements, t_begin, t_end,
                                              _ptr(re), _ptr(im), _ptr(fr)), "hhg_gpu_spectrum")
        return fr, re, im

    def k_resolved(self, sys: SystemDesc, pulse: PulseDesc, grid: GridDesc,
                   opts: SolverOpts | None = None, kind: int = KOUT_BLOCH):
        """Every trajectory at every sample: (n_measurements + 1, n_k, 3) Bloch
        vectors, (.., 2) band occupations or (n_measurements + 1, n_k) weighted
        currents (hhg_gpu_k_resolved)."""
        n_k = int(grid_rows(sys, grid).shape[0])
        w = 3 if kind == KOUT_BLOCH else (2 if kind == KOUT_OCCUPATIONS else 1)
        out = np.zeros((pulse.n_measurements + 1, n_k, w))
        st = Stats()
        self._check(self.lib.hhg_gpu_k_resolved(self.ctx, ctypes.byref(sys), ctypes.byref(pulse),
                                                ctypes.byref(grid),
                                                ctypes.byref(opts) if opts else None, kind,
                                                _ptr(out), ctypes.byref(st)), "hhg_gpu_k_resolved")
        return (out[..., 0] if w == 1 else out), st

    def split_current(self, sys: SystemDesc, pulse: PulseDesc, grid: GridDesc,
                      opts: SolverOpts | None = None, energy_cut: float = 0.5 * math.sqrt(3.0)):
        """j(t) split at the instantaneous energy cut (hhg_gpu_split_current)."""
        lo = np.zeros(pulse.n_measurements + 1)
        hi = np.zeros(pulse.n_measurements + 1)
        st = Stats()
        self._check(self.lib.hhg_gpu_split_current(self.ctx, ctypes.byref(sys), ctypes.byref(pulse),
                                                   ctypes.byref(grid),
                                                   ctypes.byref(opts) if opts else None,
                                                   energy_cut, _ptr(lo), _ptr(hi), ctypes.byref(st)),
                    "hhg_gpu_split_current")
        return lo, hi, st

    def dirac_current_density(self, sys: SystemDesc, pulse: PulseDesc, quad: KappaQuad,
                              opts: SolverOpts | None = None):
        """The Dirac-3D current density over k_z slices and the adaptive kappa
        rule (hhg_gpu_dirac_current_density): j, KappaStats, Stats.  The
        default stepper is the reference's closed-form Magnus step; with
        relaxation pass an RKF78 solver."""
        j = np.zeros(pulse.n_measurements + 1)
        qs, st = KappaStats(), Stats()
        o = opts if opts is not None else solver(stepper=STEPPER_DIRAC_MAGNUS)
        self._check(self.lib.hhg_gpu_dirac_current_density(
            self.ctx, ctypes.byref(sys), ctypes.byref(pulse), ctypes.byref(quad), ctypes.byref(o),
            _ptr(j), ctypes.byref(qs), ctypes.byref(st)), "hhg_gpu_dirac_current_density")
        return j, qs, st

    def spectrum_welch(self, j: np.ndarray, n_measurements: int, t_begin: float, t_end: float):
        """Welch-windowed N-point FFT of a continuous-laser current (hhg_gpu_spectrum_welch)."""
        j = np.ascontiguousarray(j, dtype=np.float64)
        n_fft = n_measurements // 2 + 1
        re, im, fr = np.zeros(n_fft), np.zeros(n_fft), np.zeros(n_fft)
        self._check(self.lib.hhg_gpu_spectrum_welch(self.ctx, _ptr(j), n_measurements, t_begin, t_end,
                                                    _ptr(re), _ptr(im), _ptr(fr)),
                    "hhg_gpu_spectrum_welch")
        return fr, re, im

    def trapezoidal_fft(self, x: np.ndarray, delta_t: float, t_begin: float, t_end: float):
        """TrapezoidalFFT::compute of x as given, without padding
        (hhg_gpu_trapezoidal_fft): (frequencies, real, imag), len(x) // 2 + 1 each."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n_fft = x.size // 2 + 1
        re, im, fr = np.zeros(n_fft), np.zeros(n_fft), np.zeros(n_fft)
        self._check(self.lib.hhg_gpu_trapezoidal_fft(self.ctx, _ptr(x), x.size, delta_t, t_begin,
                                                     t_end, _ptr(re), _ptr(im), _ptr(fr)),
                    "hhg_gpu_trapezoidal_fft")
        return fr, re, im

    def plan(self, sys: SystemDesc, pulses, grid: GridDesc, opts: SolverOpts | None = None):
        return Plan(self, sys, pulses, grid, opts)

    def learned_collect(self, sys: SystemDesc, pulses, grid: GridDesc,
                        opts: SolverOpts | None = None, hist_every: int = 4,
                        cap: int = 1 << 20) -> tuple[np.ndarray, Stats]:
        """Step-size history records (n x HIST_FIELDS float32) of a carry run."""
        pulses = list(pulses) if not isinstance(pulses, PulseDesc) else [pulses]
        arr = (PulseDesc * len(pulses))(*pulses)
        rec = np.zeros((cap, HIST_FIELDS), np.float32)
        n = ctypes.c_int64(0)
        st = Stats()
        o = opts if opts is not None else solver()
        self._check(self.lib.hhg_learned_collect(self.ctx, ctypes.byref(sys), arr, len(pulses),
                                                 ctypes.byref(grid), ctypes.byref(o), hist_every,
                                                 _fptr(rec), cap, ctypes.byref(n),
                                                 ctypes.byref(st)), "hhg_learned_collect")
        return rec[:n.value].copy(), st

    def mlp_train(self, records: np.ndarray, net: Mlp, opts: TrainOpts | None = None):
        """Train `net` in place on the GPU; returns (per-epoch loss, device ms)."""
        rec = _records(records)
        o = opts if opts is not None else train_opts()
        loss = np.zeros(o.epochs, np.float32)
        ms = ctypes.c_double(0.0)
        self._check(self.lib.hhg_mlp_train(self.ctx, _fptr(rec), rec.shape[0], ctypes.byref(o),
                                           ctypes.byref(net), _fptr(loss), ctypes.byref(ms)),
                    "hhg_mlp_train")
        return loss, ms.value

    def mlp_gradients(self, records: np.ndarray, net: Mlp) -> tuple[np.ndarray, float]:
        rec = _records(records)
        g = np.zeros(MLP_N_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self.lib.hhg_mlp_gradients(self.ctx, _fptr(rec), rec.shape[0],
                                               ctypes.byref(net), _fptr(g), _fptr(loss)),
                    "hhg_mlp_gradients")
        return g, float(loss[0])

    def mlp_predict(self, records: np.ndarray, net: Mlp, path: int = 0) -> np.ndarray:
        rec = _records(records)
        out = np.zeros(rec.shape[0], np.float32)
        self._check(self.lib.hhg_mlp_predict(self.ctx, _fptr(rec), rec.shape[0],
                                             ctypes.byref(net), path, _fptr(out)),
                    "hhg_mlp_predict")
        return out

    def fp64_peak_tflops(self) -> float:
        v = ctypes.c_double(0.0)
        self._check(self.lib.hhg_measure_fp64_peak(self.ctx, ctypes.byref(v)),
                    "hhg_measure_fp64_peak")
        return v.value

    def fp32_peak_tflops(self) -> float:
        v = ctypes.c_double(0.0)
        self._check(self.lib.hhg_measure_fp32_peak(self.ctx, ctypes.byref(v)),
                    "hhg_measure_fp32_peak")
        return v.value


class Plan:
    def __init__(self, eng: Engine, sys, pulses, grid, opts=None):
        self.eng = eng
        pulses = list(pulses) if not isinstance(pulses, PulseDesc) else [pulses]
        self.pulses = pulses
        arr = (PulseDesc * len(pulses))(*pulses)
        o = opts if opts is not None else solver()
        self.handle = ctypes.c_void_p()
        eng._check(eng.lib.hhg_plan_create(eng.ctx, ctypes.byref(sys), arr, len(pulses),
                                           ctypes.byref(grid), ctypes.byref(o),
                                           ctypes.byref(self.handle)), "hhg_plan_create")
        self.j_len = int(eng.lib.hhg_plan_j_length(self.handle))

    def execute_async(self, stream: int | None = None):
        self.eng._check(self.eng.lib.hhg_plan_execute_async(
            self.handle, ctypes.c_void_p(stream) if stream else None), "hhg_plan_execute_async")

    def execute_graph(self, stream: int | None = None, with_spectrum: bool = True):
        """One CUDA-graph launch of the execution (+ spectra)."""
        self.eng._check(self.eng.lib.hhg_plan_execute_graph(
            self.handle, ctypes.c_void_p(stream) if stream else None, int(with_spectrum)),
            "hhg_plan_execute_graph")

    def autotune(self, reps: int = 2) -> TuneReport:
        rep = TuneReport()
        self.eng._check(self.eng.lib.hhg_plan_autotune(self.handle, reps, ctypes.byref(rep)),
                        "hhg_plan_autotune")
        return rep

    def spectrum_async(self, stream: int | None = None):
        self.eng._check(self.eng.lib.hhg_plan_spectrum_async(
            self.handle, ctypes.c_void_p(stream) if stream else None), "hhg_plan_spectrum_async")

    def fetch_spectrum(self, pulse: int = 0):
        n_fft = 4 * (self.pulses[pulse].n_measurements + 1) + 1
        re, im, fr = np.zeros(n_fft), np.zeros(n_fft), np.zeros(n_fft)
        self.eng._check(self.eng.lib.hhg_plan_fetch_spectrum(self.handle, pulse, _ptr(re),
                                                             _ptr(im), _ptr(fr)),
                        "hhg_plan_fetch_spectrum")
        return fr, re, im

    def device_j_ptr(self) -> int:
        return int(self.eng.lib.hhg_plan_device_j(self.handle))

    def fetch(self, copy_j: bool = True):
        j = np.zeros(self.j_len) if copy_j else None
        st = Stats()
        self.eng._check(self.eng.lib.hhg_plan_fetch(self.handle, _ptr(j) if copy_j else None,
                                                    ctypes.byref(st)), "hhg_plan_fetch")
        return j, st

    def close(self):
        if self.handle:
            self.eng.lib.hhg_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
