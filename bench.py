#!/usr/bin/env python
"""Benchmark: spectra/s of the per-k-point Bloch integration -> Brillouin-zone
current sum -> trapezoidal FFT path, learned-step mixed-precision engine vs
plain FP64 RKF78, on the learned-proposer workload: honeycomb with staggered
mass 0.1 on a 1024 x 1024 rhombic Gauss-Legendre grid x 64 pulse instances
(A0 ~ U[0.5, 2], carrier phase ~ U[0, 2 pi), omega = 0.08, 6 cycles, 6144
intervals), seeded synthetic inputs.

One step = one batch of 8 of the 64 pulse instances: 8.4 M trajectories in
one persistent work-stealing launch, the BZ reduction and 8 trapezoidal FFTs,
replayed as one CUDA graph.  Consecutive steps take consecutive batches, so 8
timed steps cover all 64 spectra once.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--variant NAME]
                  [--workload NAME] [--scaling weak|strong]
  python bench.py --impl reference ...   # the reference's algorithm (the
                                         # oracle port) on the host cores

--gpus N without torchrun re-launches itself under torch.distributed.run with
N ranks (one GPU each).  Weak scaling (default): every rank integrates its own
batches (rank r takes batch k N + r at step k), no data-path collective.
Strong scaling: every rank integrates a contiguous block of each batch's k
rows (the reference's jobs_per_rank blocks, PiFlux.cpp:811-820) and j(t) is
summed over the ranks with one NCCL all_reduce before the FFT (the
reference's MPI_Reduce, sources/hhg.cpp:240-246).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "spectra/sec at harmonic err <=1e-4 vs FP64; learned+FP32 vs plain FP64"
UNIT = "spectra/s"
DEFAULT_WORKLOAD = "honeycomb_1024x64"
SEED = 20261203
MEASUREMENTS_PER_CYCLE = 1 << 10

# Algorithmic FP64 flops per attempted RKF78 step (one k-point): 13 right-hand
# sides plus the tableau arithmetic 2*3*55 (stages) + 2*3*7 (solution) +
# 2*3*4 (error) + ~25 (norm and control) = 421.  Right-hand sides: 2D pi-flux
# 12 flops + two cosines; gapped Dirac 16; honeycomb 30 (three complex bond
# phases, the mass and the cross product) + three sincos.  The PiFlux
# relaxation right-hand side (PiFlux.cpp:113-186 in the kernel's form) costs
# 76 flops + 5 special operations (2 exp, 3 rsqrt).
ALG_FLOPS_PER_KSTEP = {"piflux2d_256": 13 * 12 + 421, "dirac2d_64": 13 * 16 + 421,
                       "honeycomb_512": 13 * 30 + 421, "dirac2d_sweep": 13 * 16 + 421,
                       "honeycomb_1024x64": 13 * 30 + 421,
                       "piflux3d_relax": 13 * 76 + 421, "piflux3d_field": 13 * 12 + 421}
SPECIAL_OPS_PER_KSTEP = {"piflux2d_256": 26, "dirac2d_64": 0, "honeycomb_512": 78,
                         "honeycomb_1024x64": 78, "dirac2d_sweep": 0, "piflux3d_relax": 13 * 5}
# the relaxation workload runs the reference step schedule in FP64 only
DEFAULT_VARIANT = {"piflux3d_relax": "fp64"}
# pulse instances per step (one graph launch); default: all of the workload's
PULSES_PER_STEP = {"honeycomb_1024x64": 8}
# The mixed-precision variant splits that work: solution, error estimate, error
# norm and control stay FP64 (2*3*7 + 2*3*4 + ~25 = 91 flops); the right-hand
# sides and the stage sums (13 F_rhs + 2*3*55) run on the FP32 pipe.
FP64_FLOPS_MIXED = 91

VARIANTS = {
    "fp64": dict(),
    "carry": dict(proposer=1),
    "mixed": dict(precision=1, abs_tol=1e-8, rel_tol=1e-6),
    "mixed_carry": dict(precision=1, proposer=1, abs_tol=1e-8, rel_tol=1e-6),
    "lockstep": dict(proposer=3),
    "mixed_lockstep": dict(precision=1, proposer=3, abs_tol=1e-8, rel_tol=1e-6),
    "learned": dict(proposer=2),
    "mixed_learned": dict(precision=1, proposer=2, abs_tol=1e-8, rel_tol=1e-6),
    # one two-point Gauss Magnus step per measurement interval, the rotation
    # exp([omega]_x) applied exactly (FP64)
    "magnus4": dict(stepper=1, magnus_substeps=1),
}
# Magnus-4 flops per k.interval (PiFlux-2D): two evaluations of the staged
# interpolants (2 functions x degree 7 Horner: 56), two d vectors (~20), the
# generator h (d1 + d2) + c h^2 (d2 x d1) (~20), the rotation (~50); plus one
# sqrt and one sincos
MAGNUS4_FLOPS_PER_KSTEP = 150
LEARNED_RECORDS = 1 << 21
LEARNED_EPOCHS = 20
# the learned-proposer workload's network is trained on the three
# single-pulse configurations (gapped Dirac 64^2, pi-flux 256^2, honeycomb
# 512^2), never on the workload it is evaluated on
TRAIN_SOURCES = {"honeycomb_1024x64": ("dirac2d_64", "piflux2d_256", "honeycomb_512")}
# k rows of the oracle subsample behind harmonic_err_vs_oracle, and pulses
ORACLE_ROWS = 384
ORACLE_PULSES = 2


# ---------------------------------------------------------------------------
# The workloads as the oracle sees them.  The reference arm and the CPU
# baseline build their inputs here, from the oracle alone (no import of the
# engine package, whose library they must not load); tests/test_bench_contract.py
# checks these against the engine's workloads (higherharmonics_b200.workloads).
# ---------------------------------------------------------------------------
def splitmix64_uniforms(n: int, seed: int = SEED) -> np.ndarray:
    """n uniforms in [0, 1) from splitmix64 (top 53 bits)."""
    out = np.empty(n)
    s = seed & 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        s = (s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z = z ^ (z >> 31)
        out[i] = (z >> 11) * (1.0 / (1 << 53))
    return out


class RefWorkload:
    """Oracle inputs of one workload: per pulse instance the model (constants
    already multiplied by the pulse's energy scale), the pulse and the time
    configuration; the solver; a builder of the k rows."""

    def __init__(self, name, jobs, tol, rows_fn):
        self.name = name
        self.jobs = jobs          # [(model, pulse, time_config)]
        self.tol = tol            # (abs, rel)
        self._rows_fn = rows_fn
        self._rows = None

    @property
    def rows(self) -> np.ndarray:
        if self._rows is None:
            self._rows = self._rows_fn()
        return self._rows

    @property
    def n_meas(self) -> int:
        return int(self.jobs[0][2].n_measurements)


def ref_workload(name: str) -> RefWorkload:
    if name in _REF_OVERRIDE:
        return _REF_OVERRIDE[name]
    from oracle import hhg_oracle as O
    two_pi = 2 * math.pi
    if name == "dirac2d_64":
        es = 1.0 / 0.1
        m = O.model(O.DIRAC2D, velocity=1.0 * es, mass=0.05 * es, pol=(1.0, 0.0))
        jobs = [(m, O.Pulse(1.0, 4), O.time_config(0.0, two_pi * 4, 4 * MEASUREMENTS_PER_CYCLE))]
        return RefWorkload("dirac2d_64x64_4cyc", jobs, (1e-10, 1e-10),
                           lambda: O.grid_tensor(m, 64, 64, -2, 2, -2, 2))
    if name == "piflux2d_256":
        es = 1.0 / 0.05
        s = 1.0 / math.sqrt(2.0)
        m = O.model(O.PIFLUX2D, hopping=1.0 * es, pol=(s, s))
        jobs = [(m, O.Pulse(1.0, 8), O.time_config(0.0, two_pi * 9, 8 * MEASUREMENTS_PER_CYCLE))]
        return RefWorkload("piflux2d_256x256_8cyc", jobs, (1e-12, 1e-8),
                           lambda: O.grid_tensor(m, 256, 256, -math.pi, math.pi, -math.pi, math.pi))
    if name == "honeycomb_512":
        es = 1.0 / 0.08
        m = O.model(O.HONEYCOMB, hopping=1.0 * es, mass=0.1 * es, pol=(1.0, 0.0))
        a0 = 0.5 + splitmix64_uniforms(1)[0]
        jobs = [(m, O.Pulse(a0, 6), O.time_config(0.0, two_pi * 7, 6 * MEASUREMENTS_PER_CYCLE))]
        return RefWorkload("honeycomb_rhombic_512x512_6cyc", jobs, (1e-12, 1e-8),
                           lambda: O.grid_rhombic(m, 512, 512))
    if name == "dirac2d_sweep":
        u = splitmix64_uniforms(4 * 256).reshape(256, 4)
        jobs = []
        for i in range(256):
            a0 = math.exp(math.log(0.1) + u[i, 0] * (math.log(2.0) - math.log(0.1)))
            phi = two_pi * u[i, 1]
            ncyc = 2.0 + 8.0 * u[i, 2]
            es = 1.0 / (0.05 + 0.1 * u[i, 3])
            n = int(round(MEASUREMENTS_PER_CYCLE * ncyc))
            mi = O.model(O.DIRAC2D, velocity=1.0 * es, mass=0.05 * es, pol=(1.0, 0.0))
            jobs.append((mi, O.Pulse(a0, ncyc, 0.0, phi), O.time_config(0.0, two_pi * ncyc, n)))
        m0 = jobs[0][0]
        return RefWorkload("dirac2d_sweep_256x128x128", jobs, (1e-10, 1e-10),
                           lambda: O.grid_tensor(m0, 128, 128, -2, 2, -2, 2))
    if name == "honeycomb_1024x64":
        es = 1.0 / 0.08
        m = O.model(O.HONEYCOMB, hopping=1.0 * es, mass=0.1 * es, pol=(1.0, 0.0))
        u = splitmix64_uniforms(2 * 64, SEED + 5).reshape(64, 2)
        jobs = [(m, O.Pulse(0.5 + 1.5 * u[i, 0], 6, 0.0, two_pi * u[i, 1]),
                 O.time_config(0.0, two_pi * 7, 6 * MEASUREMENTS_PER_CYCLE)) for i in range(64)]
        return RefWorkload("honeycomb_rhombic_1024x1024x64", jobs, (1e-12, 1e-8),
                           lambda: O.grid_rhombic(m, 1024, 1024))
    raise KeyError(name)


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


class CpuBaseline:
    """The reference's plain FP64 algorithm (the oracle port with the
    reference's Release flags: -O3 -ffast-math, OpenMP over k-points) on all
    host cores, over a strided k-subsample of one pulse instance per run;
    spectra/s are the sampled fraction of a spectrum per second."""

    def __init__(self, rw: RefWorkload, target_s: float):
        from oracle import hhg_oracle as O
        self.O = O
        self.rw = rw
        self.cores = host_cores()
        self.s = O.solver(*rw.tol)
        rows = rw.rows
        self.n_k = rows.shape[0]
        m, p, tc = rw.jobs[0]
        calib = rows[:: max(1, self.n_k // max(self.cores, 8))][: max(self.cores, 8)]
        t0 = time.perf_counter()
        O.current_density(m, p, tc, self.s, calib, threads=self.cores, fast=True)
        per_k = (time.perf_counter() - t0) / calib.shape[0]
        n_sample = int(min(self.n_k, max(self.cores, target_s / max(per_k, 1e-9))))
        self.stride = max(1, self.n_k // n_sample)
        self.sample = np.ascontiguousarray(rows[:: self.stride])
        self.runs = 0

    def run(self, job: int | None = None):
        """One sample (pulse instance `job`, default: the next one): returns
        (spectra/s, seconds, description, attempted k.steps/s)."""
        if job is None:
            job = self.runs % len(self.rw.jobs)
        self.runs += 1
        m, p, tc = self.rw.jobs[job]
        t0 = time.perf_counter()
        _, st, rc = self.O.current_density(m, p, tc, self.s, self.sample, threads=self.cores,
                                           fast=True)
        el = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"oracle status {rc}")
        frac = self.sample.shape[0] / self.n_k
        desc = (f"every {self.stride}th k-point ({self.sample.shape[0]} of {self.n_k}) of pulse "
                f"instance {job} over its full {tc.n_measurements}-interval pulse: {st.attempted} "
                f"k.steps in {el:.2f} s on {self.cores} threads (oracle port, -O3 -ffast-math, "
                f"OpenMP); spectra/s = {frac:.3e} of a spectrum / time")
        return frac / el, el, desc, st.attempted / el

    @property
    def timed_fraction(self) -> float:
        return self.sample.shape[0] / self.n_k


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_arm(args):
    """The reference's algorithm on the host cores (oracle port; the
    reference itself cannot be built here), on the same workload: each step is
    one bounded sample -- a strided k-subsample of one pulse instance over its
    full pulse -- sized so all K + W steps take about --reference-seconds.
    ms_per_step is the measured wall time of a step; value = the spectra the
    sampled fractions amount to, per second."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    rw = ref_workload(args.workload)
    per_step_s = max(0.5, args.reference_seconds / (args.steps + args.warmup))
    cb = CpuBaseline(rw, target_s=per_step_s)
    secs, fracs = [], []
    desc = ksps = None
    for i in range(args.warmup + args.steps):
        _, el, desc, ksps = cb.run()
        if i >= args.warmup:
            secs.append(el)
            fracs.append(cb.timed_fraction)
    total_s = float(np.sum(secs))
    value = float(np.sum(fracs)) / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": rw.name, "k_points": int(rw.rows.shape[0]),
                   "n_measurements": rw.n_meas, "pulses": len(rw.jobs),
                   "tolerances": f"{rw.tol[0]:g}/{rw.tol[1]:g}",
                   "variant": "oracle port of the reference's plain FP64 RKF78 (restart schedule)"},
        "timed_fraction": cb.timed_fraction,
        "timed_fraction_note": "spectra per step actually integrated (a k-subsample of one pulse "
                               "instance); value = timed fractions / timed seconds",
        "k_steps_per_s": ksps,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb.cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def traffic_from_profile(wl_name):
    """Per-launch DRAM bytes of the integration kernel from the committed ncu
    summaries (a line 'traffic_bytes_per_launch[<workload>]: <bytes>' in one
    of profiles/bz_integrate_kernel*.md)."""
    import glob
    key = f"traffic_bytes_per_launch[{wl_name}]:"
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "bz_integrate_kernel*.md"))):
        for line in open(path):
            if line.strip().startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


# ---------------------------------------------------------------------------
# The GPU arm
# ---------------------------------------------------------------------------
def train_proposer(eng, wl_name, wl, api, W):
    """The learned proposer: accept/reject histories of the FP64 carry
    controller at the plain tolerances (hhg_learned_collect), on the workload's
    training sources (TRAIN_SOURCES: configurations 1-3 for the learned-proposer
    workload; otherwise the workload itself), then Adam on the GPU (tcgen05
    training kernels).  Outside the timed region; reported under "training"."""
    names = TRAIN_SOURCES.get(wl_name, (wl_name,))
    t0 = time.perf_counter()
    parts, sources = [], []
    cap = LEARNED_RECORDS // len(names)
    for nm in names:
        src = wl if nm == wl_name else W.ALL[nm]()
        n_int = sum(p.n_measurements for p in src.pulses)
        every = max(1, math.ceil(src.n_k * n_int / cap))
        recs, _ = eng.learned_collect(src.system, src.pulses, src.grid, src.opts(),
                                      hist_every=every, cap=cap)
        parts.append(recs)
        sources.append({"workload": src.name, "records": int(recs.shape[0]), "hist_every": every})
    recs = np.concatenate(parts)
    t1 = time.perf_counter()
    net = api.mlp_init(1, recs)
    loss, train_ms = eng.mlp_train(recs, net, api.train_opts(epochs=LEARNED_EPOCHS))
    t2 = time.perf_counter()
    return net, {"records": int(recs.shape[0]), "sources": sources,
                 "collect_s": t1 - t0, "train_s": t2 - t1, "train_device_ms": train_ms,
                 "epochs": LEARNED_EPOCHS, "loss_first_last": [float(loss[0]), float(loss[-1])],
                 "network": "8-64-64-64-1 SiLU, BF16/FP32, tcgen05 training"}


def variant_opts(name, net, args, api):
    okw = dict(VARIANTS[name])
    if okw.get("proposer") == api.PROPOSER_LEARNED:
        okw["mlp"] = net
        if args.mlp_every:
            okw["mlp_every"] = args.mlp_every
    return okw


def spectrum_intensities(plan, pulse_index, mo=None):
    from higherharmonics_b200.analysis import default_max_order, harmonic_intensities
    fr, re, im = plan.fetch_spectrum(pulse_index)
    if mo is None:
        mo = default_max_order(fr)
    return harmonic_intensities(fr, re, im, mo), mo


class OracleCheck:
    """Harmonic error of a variant against the FP64 oracle on a seeded
    subsample: ORACLE_ROWS k rows spread evenly over the grid and the first
    ORACLE_PULSES pulse instances of batch 0, each over its full pulse.  The
    oracle (strict FP64, -ffp-contract=off) integrates those rows once; a
    variant runs the same rows through an explicit-rows grid."""

    def __init__(self, wl, rows, api):
        from oracle import hhg_oracle as O
        from tests.helpers import harmonics, oracle_args
        stride = max(1, rows.shape[0] // ORACLE_ROWS)
        self.rows = np.ascontiguousarray(rows[::stride][:ORACLE_ROWS])
        self.grid, self._keep = api.grid_explicit(self.rows)
        self.pulses = wl.pulses[:ORACLE_PULSES]
        self.I, self.mo = [], []
        t0 = time.perf_counter()
        for p in self.pulses:
            m, op, tc, s = oracle_args(wl.system, p, wl.opts_kw["abs_tol"], wl.opts_kw["rel_tol"])
            j, _, rc = O.current_density(m, op, tc, s, self.rows, threads=host_cores())
            if rc != 0:
                raise RuntimeError(f"oracle status {rc}")
            I = harmonics(j, p)
            self.I.append(I)
            self.mo.append(I.size)
        self.oracle_s = time.perf_counter() - t0
        self.stride = stride

    def error(self, eng, wl, okw) -> float:
        from higherharmonics_b200.analysis import harmonic_rel_err
        plan = eng.plan(wl.system, self.pulses, self.grid, wl.opts(**okw))
        plan.execute_async()
        plan.spectrum_async()
        plan.fetch(copy_j=False)
        err = 0.0
        for i, I0 in enumerate(self.I):
            I, _ = spectrum_intensities(plan, i, self.mo[i])
            err = max(err, harmonic_rel_err(I, I0, floor_rel=1e-6))
        plan.close()
        return err

    def describe(self) -> str:
        return (f"{self.rows.shape[0]} k rows (every {self.stride}th) x the first "
                f"{len(self.pulses)} pulse instances, full pulses; FP64 oracle "
                f"({self.oracle_s:.1f} s on {host_cores()} threads)")


def time_plan(plan, stream, flush, steps):
    """Mean ms of `steps` graph launches (integration + reduction + spectra),
    CUDA events on the launching stream, L2 flushed before each."""
    import torch
    sptr = stream.cuda_stream
    flush.zero_()
    plan.execute_graph(sptr, with_spectrum=True)  # warm-up (captures the graph)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        a.record(stream)
        plan.execute_graph(sptr, with_spectrum=True)
        b.record(stream)
        torch.cuda.synchronize()
        total += a.elapsed_time(b)
    return total / steps


def compare_variants(args, eng, wl, batch0, api, stream, flush, main_variant, net, ref_I, ocheck):
    """spectra/s of the plain FP64 path and the other variants on batch 0 of
    the workload, same timing method as the headline (CUDA events over graph
    launches, L2 flushed before each), each with its harmonic error against
    the GPU FP64 engine (full grid) and against the FP64 oracle (subsample)."""
    from higherharmonics_b200.analysis import harmonic_rel_err
    out = {}
    names = ["fp64", "mixed_learned", "mixed_lockstep", "magnus4"]
    steps = max(1, min(args.steps, 2))
    for v in names:
        if v == main_variant or (v != "fp64" and args.workload in DEFAULT_VARIANT):
            continue
        okw = variant_opts(v, net, args, api)
        plan = eng.plan(wl.system, batch0, wl.grid, wl.opts(**okw))
        ms = time_plan(plan, stream, flush, steps)
        _, st = plan.fetch(copy_j=False)
        herr = 0.0
        for i in range(len(batch0)):
            I, mo = spectrum_intensities(plan, i, len(ref_I[i]))
            herr = max(herr, harmonic_rel_err(I, ref_I[i], floor_rel=1e-6))
        plan.close()
        out[v] = {"value": len(batch0) / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                  "timed_launches": steps,
                  "k_steps_per_spectrum": st.attempted_steps / len(batch0),
                  "harmonic_err_vs_fp64": herr,
                  "harmonic_err_vs_oracle": ocheck.error(eng, wl, okw) if ocheck else None}
    return out


class JView:
    """A plan's device j buffer seen by torch (zero copy), for the NCCL sum."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 2}


def our_arm(args):
    import torch
    ws, rank, local = dist_env()
    strong = args.scaling == "strong" and ws > 1
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from higherharmonics_b200 import api
    from higherharmonics_b200 import workloads as W
    from higherharmonics_b200.distributed import shard_range

    name = args.workload
    wl = W.ALL[name]()
    pps = args.pulses_per_step or PULSES_PER_STEP.get(name, len(wl.pulses))
    batches = [wl.pulses[i:i + pps] for i in range(0, len(wl.pulses), pps)]
    nb = len(batches)
    eng = api.Engine(dev)
    rows_all = None
    grid = wl.grid
    shard = None
    if strong:
        # this rank's contiguous block of the k rows (jobs_per_rank blocks)
        rows_all = api.grid_rows(wl.system, wl.grid)
        lo, hi = shard_range(rows_all.shape[0], rank, ws)
        grid, _keep_rows = api.grid_explicit(rows_all[lo:hi])
        shard = [lo, hi]

    net = training = None
    if VARIANTS[args.variant].get("proposer") == api.PROPOSER_LEARNED or not args.no_compare:
        net, training = train_proposer(eng, name, wl, api, W)
    okw = variant_opts(args.variant, net, args, api)

    # one plan per batch (the batch a step integrates); weak scaling: rank r
    # takes batch (k ws + r) mod nb at step k
    def batch_of(k):
        return k % nb if strong else (k * ws + rank) % nb

    needed = sorted({batch_of(k) for k in range(args.warmup + args.steps)})
    plans = {}
    t_setup = time.perf_counter()
    for b in needed:
        plans[b] = eng.plan(wl.system, batches[b], grid, wl.opts(**okw))
    setup_s = time.perf_counter() - t_setup
    tune = None
    if args.autotune and not strong and nb == 1:
        tune = plans[needed[0]].autotune(reps=2)
    # a dedicated stream: the legacy default stream has handle 0, which the
    # C ABI reads as "the context's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr != 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(k):
        plan = plans[batch_of(k)]
        flush.zero_()
        if not strong:
            plan.execute_graph(sptr, with_spectrum=True)
            return
        # integrate this rank's rows, sum j over the ranks, then the spectra
        plan.execute_graph(sptr, with_spectrum=False)
        jt = torch.as_tensor(JView(plan.device_j_ptr(), plan.j_len), device="cuda")
        torch.distributed.all_reduce(jt, op=torch.distributed.ReduceOp.SUM)
        plan.spectrum_async(sptr)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        step(args.warmup + k)
        ev[k][1].record(stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    elapsed_ms = e_start.elapsed_time(e_end)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    # attempted k.steps of the timed steps (each plan's counters hold its last run)
    ksteps = 0
    for k in range(args.steps):
        _, st = plans[batch_of(args.warmup + k)].fetch(copy_j=False)
        ksteps += st.attempted_steps
    if ws > 1:
        t = torch.tensor([elapsed_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed_ms = float(t.item())
        kt = torch.tensor([float(ksteps)], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(kt, op=torch.distributed.ReduceOp.SUM)
        ksteps_all = float(kt.item())
    else:
        ksteps_all = float(ksteps)
    spectra_per_step = pps * (1 if strong else ws)
    value = args.steps * spectra_per_step / (elapsed_ms * 1e-3)

    # end to end through the public one-shot API with host buffers: every
    # step a new batch (a plan-cache miss: the host builds and uploads the
    # pulse records and time grids, the device stages the pulses; the k table
    # of the grid is the context's shared one), j back, then each pulse's
    # spectrum from its host j
    e2e = None
    if not args.no_e2e and not strong:
        n_e2e = max(1, min(args.steps, 3))
        e_batches = [(k * ws + rank + args.warmup) % nb for k in range(n_e2e)]
        if nb == 1:
            eng.current_density(wl.system, batches[0], grid, wl.opts(**okw))  # cache warm-up
        # warm-up of the spectrum path (the context's FFT plans and buffers
        # for a length are made on its first call)
        for n_m in sorted({p.n_measurements for b in e_batches for p in batches[b]}):
            eng.spectrum(np.zeros(n_m + 1), n_m, 0.0, 1.0)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        h2d = d2h = 0
        t0 = time.perf_counter()
        for b in e_batches:
            j, st = eng.current_density(wl.system, batches[b], grid, wl.opts(**okw))
            off = 0
            for p in batches[b]:  # every pulse instance's spectrum
                n_s = p.n_measurements + 1
                eng.spectrum(j[off:off + n_s], p.n_measurements, p.window_begin, p.window_end)
                off += n_s
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if ws > 1:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            el = float(t.item())
        # bytes copied per step: in, the pulse records (256 B) and time grids
        # (8 B x samples) of the batch and each pulse's j into its spectrum
        # call (the k rows were uploaded once, by the first plan on the grid);
        # out, j and each spectrum's frequencies, real and imaginary parts
        for p in batches[e_batches[0]]:
            n_s = p.n_measurements + 1
            n_fft = 4 * n_s + 1
            h2d += 256 + 8 * n_s + 8 * n_s
            d2h += 8 * n_s + 3 * 8 * n_fft
        e2e = {"value": ws * n_e2e * pps / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": "Engine.current_density + Engine.spectrum (hhg_gpu_current_density + "
                       "hhg_gpu_spectrum), host buffers, wall clock" +
                       (", a new batch every step (plan built on the grid's shared k table)" if nb > 1 else
                        ", plan cached by the context after the first call")}

    if rank != 0:
        for p in plans.values():
            p.close()
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0

    per_kstep = ALG_FLOPS_PER_KSTEP.get(name, 421)
    magnus = VARIANTS[args.variant].get("stepper", 0) == 1
    if magnus:
        per_kstep = MAGNUS4_FLOPS_PER_KSTEP
    mixed = VARIANTS[args.variant].get("precision", 0) == 1
    peak = eng.fp64_peak_tflops()
    peak32 = eng.fp32_peak_tflops() if mixed else None
    kernel_s = float(np.mean(launch_ms)) * 1e-3
    ksteps_per_launch = ksteps / args.steps
    if mixed:
        # the bound is whichever pipe needs longer for its share of the work:
        # FP32 (13 F_rhs + 330 flops) against the measured FP32 FMA rate
        f32 = per_kstep - FP64_FLOPS_MIXED
        t32, t64 = f32 / peak32, FP64_FLOPS_MIXED / peak
        bound, bpeak, bflops = ("fp32_pipe", peak32, f32) if t32 >= t64 else ("fp64_pipe", peak, FP64_FLOPS_MIXED)
        peak_src = ("measured FP32 FMA throughput (hhg_measure_fp32_peak, burst); the FP64 share "
                    f"({FP64_FLOPS_MIXED} flops/k.step at {peak:.1f} TFLOP/s) needs less time")
    else:
        bound, bpeak, bflops = "fp64_pipe", peak, per_kstep
        peak_src = ("measured FP64 FMA throughput (hhg_measure_fp64_peak, burst); "
                    "MEASURED_PEAKS.json has no FP64 figure")
    achieved = bflops * ksteps_per_launch / kernel_s / 1e12
    roofline = {"bound": bound, "achieved": achieved, "peak": bpeak, "unit": "TFLOP/s",
                "frac": achieved / bpeak, "traffic": traffic_from_profile(name),
                "peak_source": peak_src, "fp64_peak": peak, "fp32_peak": peak32,
                "kernel": "bz_integrate_kernel", "kernel_ms": 1e3 * kernel_s,
                "kernel_ms_source": "mean over the timed steps of CUDA events around each graph "
                                    "launch (integration + reduction + FFTs) on the launching "
                                    "stream (rank 0)",
                "alg_flops_per_kstep": per_kstep, "bound_flops_per_kstep": bflops,
                "special_ops_per_kstep": 2 if magnus else SPECIAL_OPS_PER_KSTEP.get(name, 0)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if strong else "weak", "vs_baseline": None,
        "dtype": "f64" if not mixed else "f32 rhs / f64 state",
        "data": "synthetic (seeded pulse table, splitmix64 seed 20261203)",
        "config": {"workload": wl.name, "k_points": wl.n_k,
                   "n_measurements": wl.pulses[0].n_measurements, "pulses": len(wl.pulses),
                   "pulses_per_step": pps, "batches": nb,
                   "tolerances": "{:g}/{:g}".format(wl.opts(**okw).abs_tol, wl.opts(**okw).rel_tol),
                   "variant": args.variant,
                   "l2": "flushed (256 MiB write) before every timed step",
                   **({"k_rows_of_rank0": shard} if strong else {})},
        "k_steps_per_s": ksteps_all / (elapsed_ms * 1e-3),
        "k_steps_per_spectrum": ksteps / (args.steps * pps),
        "gpu_launches": (4 + 2 * pps) * args.steps if not strong else (3 + 2 * pps) * args.steps,
        "roofline": roofline, "clocks": clocks, "e2e": e2e, "training": training,
        "setup_s": setup_s,
        "path": "plans per batch of pulse instances, one CUDA graph launch per step "
                "(integration + BZ reduction + trapezoidal FFTs)" +
                (", j summed over ranks by NCCL all_reduce between them" if strong else ""),
        "timing": {"device_ms_total": elapsed_ms, "launch_ms": launch_ms},
    }
    if tune is not None:
        line["autotune"] = {"chosen": tune.as_list()[tune.best], "candidates": tune.as_list()}
    if ws == 1:
        # accuracy: batch 0 against the plain FP64 engine (full grid), and the
        # variant against the FP64 oracle (k-subsample)
        ocheck = None
        if not args.no_oracle_check:
            ocheck = OracleCheck(wl, api.grid_rows(wl.system, wl.grid), api)
            line["harmonic_err_vs_oracle"] = ocheck.error(eng, wl, okw)
            line["oracle_check"] = ocheck.describe()
        ref = eng.plan(wl.system, batches[0], wl.grid, wl.opts())
        ref.execute_async(sptr)
        ref.spectrum_async(sptr)
        ref.fetch(copy_j=False)
        ref_I = [spectrum_intensities(ref, i)[0] for i in range(len(batches[0]))]
        ref.close()
        from higherharmonics_b200.analysis import harmonic_rel_err
        p0 = plans.get(0) or eng.plan(wl.system, batches[0], wl.grid, wl.opts(**okw))
        p0.execute_async(sptr)
        p0.spectrum_async(sptr)
        p0.fetch(copy_j=False)
        herr = 0.0
        for i in range(len(batches[0])):
            I, _ = spectrum_intensities(p0, i, len(ref_I[i]))
            herr = max(herr, harmonic_rel_err(I, ref_I[i], floor_rel=1e-6))
        line["harmonic_err_vs_fp64"] = herr
        if not args.no_cpu_baseline:
            rw = ref_workload(name) if _has_ref(name) else engine_ref_workload(wl, api)
            if rw is not None:
                cb = CpuBaseline(rw, target_s=args.cpu_seconds)
                v, _, desc, ksps = cb.run(0)
                line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cb.cores, "kind": "port",
                                        "sample": desc, "k_steps_per_s": ksps}
        if not args.no_compare:
            line["compare"] = compare_variants(args, eng, wl, batches[0], api, stream, flush,
                                               args.variant, net, ref_I, ocheck)
            fp = line["compare"].get("fp64")
            if fp:
                line["speedup_vs_plain_fp64"] = value / fp["value"]
    print(json.dumps(line), flush=True)
    for p in plans.values():
        p.close()
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def _has_ref(name):
    try:
        ref_workload(name)
        return True
    except KeyError:
        return False


# The Dirac workload's unit is one k.interval of the closed-form Magnus step
# (DiracSystem::time_evolution_magnus), counted on the plane/axis form the
# kernel evaluates (only nonzero components): moments and the plane vectors
# (~18 flops), the three first-level cross products (9), their nested
# products and the 13 series terms (~86), the rotation S <- exp(Omega) S
# (~75) and the weighted sample (1): ~190 FP64 flops, plus sqrt, sincos and
# three divisions (special operations).
MAGNUS_FLOPS_PER_KINTERVAL = 190
# Dirac-3D with relaxation under FP64 RKF78: one attempted step = 13
# right-hand sides (m_x, m_z: 4 flops; the rotation part 6; the three
# relaxation terms 6: 16) + the tableau arithmetic (421)
DIRAC_RELAX_FLOPS_PER_KSTEP = 13 * 16 + 421
MAGNUS_SPECIAL_OPS = 5


class DiracCpuBaseline:
    """The oracle's Dirac quadrature (the same adaptive kappa rule, the
    oracle's closed-form Magnus step, OpenMP over trajectories) on an evenly
    spaced subset of the (k_z slice, split) pairs, each split refined to
    convergence; spectra/s scaled by all splits / sampled splits (the splits
    are independent)."""

    def __init__(self, wl, target_s: float):
        from oracle import hhg_oracle as O
        from tests.helpers import oracle_args
        self.O = O
        self.m, self.p, self.tc, self.s = oracle_args(wl.system, wl.pulse, wl.opts.abs_tol,
                                                      wl.opts.rel_tol, stepper=wl.opts.stepper)
        q = wl.quad
        self.q = q
        self.dz = 2 * q.max_k / q.n_z
        self.kz = [(z - q.n_z // 2) * self.dz for z in range(1, q.n_z) if z != q.n_z // 2]
        self.cores = (len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity")
                      else os.cpu_count())
        self.pairs = [(z, sp) for z in range(len(self.kz)) for sp in range(q.n_splits)]
        # calibration: the first splits of the middle slice (the widest kappa range)
        mid = len(self.kz) // 2 * q.n_splits
        t0 = time.perf_counter()
        self._splits(self.pairs[mid:mid + 4])
        per_split = (time.perf_counter() - t0) / 4
        n = int(min(len(self.pairs), max(4, target_s / max(per_split, 1e-9))))
        step = len(self.pairs) / n
        self.sample = sorted({self.pairs[int(i * step)] for i in range(n)})

    def _splits(self, pairs):
        O, q = self.O, self.q
        kz = self.kz
        kmax = [math.sqrt(q.max_k * q.max_k - k * k) for k in kz]
        m, p, tc, s = self.m, self.p, self.tc, self.s

        def contrib(rows):
            out, rc = O.k_resolved(m, p, tc, s, rows, 0, threads=self.cores, fast=True)
            if rc != 0:
                raise RuntimeError(f"oracle status {rc}")
            return out[:, :, 2] * rows[:, 3][None, :]

        _, info = O.adaptive_kappa(contrib, kz, kmax, q.n_kappa, q.threshold, q.n_splits,
                                   q.max_halvings or 12, self.dz, tc.n_measurements + 1,
                                   lambda z, a, H, L: O.kappa_rows(m, kz[z], a, H, L, q.n_kappa),
                                   only=pairs)
        return info

    def run(self):
        """One sample: (spectra/s, seconds, description, k.intervals/s)."""
        t0 = time.perf_counter()
        info = self._splits(self.sample)
        el = time.perf_counter() - t0
        v = self.timed_fraction / el
        kint = info["trajectories"] * self.tc.n_measurements
        desc = (f"{len(self.sample)} of {len(self.pairs)} (k_z slice, kappa split) pairs, evenly "
                f"spaced, each refined to convergence ({info['trajectories']} trajectories, {kint} "
                f"k.intervals) in {el:.2f} s on {self.cores} threads (oracle port, -O3 "
                f"-ffast-math, OpenMP); spectra/s = {self.timed_fraction:.3e} of a spectrum / time")
        return v, el, desc, kint / el

    @property
    def timed_fraction(self) -> float:
        return len(self.sample) / len(self.pairs)


def dirac_config(wl, path):
    q = wl.quad
    return {"workload": wl.name, "n_z": q.n_z, "n_kappa": q.n_kappa, "n_splits": q.n_splits,
            "kappa_threshold": q.threshold, "max_k": q.max_k,
            "n_measurements": wl.pulse.n_measurements,
            "stepper": ("closed-form Magnus (FP64)" if wl.opts.stepper == 2 else
                        "RKF78 with relaxation, reference schedule (FP64)"),
            "l2": "flushed (256 MiB write) before every timed step", "path": path}


def dirac_reference_arm(args):
    """The Dirac quadrature's reference arm: each step one bounded sample of
    (slice, split) pairs; ms_per_step is its measured wall time."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from higherharmonics_b200 import workloads as W
    wl = W.ALL[args.workload]()
    cb = DiracCpuBaseline(wl, max(0.5, args.reference_seconds / (args.steps + args.warmup)))
    secs = []
    desc = None
    for i in range(args.warmup + args.steps):
        _, el, desc, _ = cb.run()
        if i >= args.warmup:
            secs.append(el)
    total_s = float(np.sum(secs))
    value = args.steps * cb.timed_fraction / total_s
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dirac_config(wl, "oracle port"),
            "timed_fraction": cb.timed_fraction,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb.cores, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def dirac_arm(args):
    """One step = one Dirac spectrum through the public API:
    Engine.dirac_current_density (k_z slices x the adaptive kappa rule, every
    refinement round one integration launch over its new nodes, convergence
    read back to the host) and Engine.spectrum.  The call is synchronous and
    host-driven between rounds, so `value` is the wall time of the quadrature
    call and `e2e` adds the spectrum; the roofline uses the integration
    kernels' CUDA-event time summed over the rounds."""
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from higherharmonics_b200 import api
    from higherharmonics_b200 import workloads as W
    wl = W.ALL[args.workload]()
    if ws > 1:  # one pulse instance per rank: weak scaling
        wl.pulse.phase = wl.pulse.phase + 0.1 * rank
    eng = api.Engine(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    p = wl.pulse

    def step():
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        j, qs, st = eng.dirac_current_density(wl.system, p, wl.quad, wl.opts)
        t1 = time.perf_counter()
        eng.spectrum(j, p.n_measurements, p.window_begin, p.window_end)
        t2 = time.perf_counter()
        return t1 - t0, t2 - t0, qs, st

    for _ in range(args.warmup):
        step()
    peak = eng.fp64_peak_tflops()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    quad_s, e2e_s, kern_ms, kint, launches = 0.0, 0.0, 0.0, 0, 0
    qs = st = None
    per_step = []
    for _ in range(args.steps):
        a, b, qs, st = step()
        per_step.append((1e3 * a, 1e3 * b, st.kernel_ms))
        quad_s += a
        e2e_s += b
        kern_ms += st.kernel_ms
        kint += st.attempted_steps
        launches += 3 * qs.launches + 1 + 3  # rows, integration, round; sum; pad, FFT, correction
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    if ws > 1:
        t = torch.tensor([quad_s, e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        quad_s, e2e_s = float(t[0]), float(t[1])
    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0
    kernel_s = kern_ms * 1e-3
    magnus = wl.opts.stepper == 2
    per_unit = MAGNUS_FLOPS_PER_KINTERVAL if magnus else DIRAC_RELAX_FLOPS_PER_KSTEP
    achieved = per_unit * kint / kernel_s / 1e12
    n_s = p.n_measurements + 1
    n_fft = 4 * n_s + 1
    line = {
        "metric": METRIC, "value": ws * args.steps / quad_s, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * quad_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": dirac_config(wl, "hhg_gpu_dirac_current_density (synchronous, host-driven "
                                   "rounds), wall clock"),
        ("k_intervals_per_spectrum" if magnus else "k_steps_per_spectrum"): st.attempted_steps,
        "kappa": qs.as_dict(),
        "gpu_launches": launches,
        "roofline": {"bound": "fp64_pipe", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic_from_profile(args.workload),
                     "traffic_note": "DRAM bytes of the first integration launch (99 % of the "
                                     "k.steps), scaled from the committed ncu capture",
                     "peak_source": "measured FP64 FMA throughput (hhg_measure_fp64_peak, burst)",
                     "kernel": "bz_integrate_kernel (closed-form Magnus, per-trajectory output)",
                     "kernel_ms": kern_ms / args.steps,
                     "kernel_ms_source": "CUDA events around each round's integration launch on "
                                         "the context stream, summed over the rounds",
                     "unit_of_work": "k.interval (Magnus step)" if magnus else "attempted k.step",
                     "alg_flops_per_unit": per_unit,
                     "special_ops_per_unit": MAGNUS_SPECIAL_OPS if magnus else 0},
        "clocks": clocks,
        "timing": {"quadrature_ms": [round(a, 3) for a, _, _ in per_step],
                   "with_spectrum_ms": [round(b, 3) for _, b, _ in per_step],
                   "integration_kernel_ms": [round(k, 3) for _, _, k in per_step]},
        "e2e": {"value": ws * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(8 * n_s + 3 * 8 * n_fft),
                "path": "Engine.dirac_current_density + Engine.spectrum, host buffers, wall "
                        "clock (inputs are descriptors: rows are built on the device)"},
    }
    if ws == 1 and not args.no_cpu_baseline:
        cb = DiracCpuBaseline(wl, args.cpu_seconds)
        v, _, desc, kps = cb.run()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cb.cores, "kind": "port",
                                "sample": desc, "k_intervals_per_s": kps}
    print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def ncu_case(args):
    """A small case of a bench workload for ncu captures (committed so the
    profile summaries name a command that runs committed files only): the
    same grid and pulse shape over --ncu-cycles cycles (default 1: 1024
    intervals) and the first --ncu-pulses pulse instances, two executions of
    the selected variant (the learned variants first collect histories on the
    case itself, one launch, and train 2 epochs); with --variant mlp_train,
    history collection on that case and 2 epochs of proposer training.  Prints one line, no
    timing."""
    from higherharmonics_b200 import api
    from higherharmonics_b200 import workloads as W
    import inspect
    if args.workload.startswith("dirac3d_kappa"):
        wl = W.ALL[args.workload](n_cycles=args.ncu_cycles)
        eng = api.Engine(0)
        for _ in range(2):
            _, qs, st = eng.dirac_current_density(wl.system, wl.pulse, wl.quad, wl.opts)
        print("ok dirac3d_kappa", qs.as_dict(), st.attempted_steps, st.kernel_ms)
        return 0
    make = W.ALL[args.workload]
    wl = (make(n_cycles=args.ncu_cycles) if "n_cycles" in inspect.signature(make).parameters
          else make())
    if args.ncu_pulses:
        wl.pulses = wl.pulses[:args.ncu_pulses]
    eng = api.Engine(0)
    if args.variant == "mlp_train":
        recs, _ = eng.learned_collect(wl.system, wl.pulses, wl.grid, wl.opts(), hist_every=32,
                                      cap=1 << 21)
        net = api.mlp_init(1, recs)
        loss, ms = eng.mlp_train(recs, net, api.train_opts(epochs=2))
        print("ok mlp_train", recs.shape[0], float(loss[-1]), ms)
        return 0
    okw = dict(VARIANTS[args.variant])
    if okw.get("proposer") == api.PROPOSER_LEARNED:
        recs, _ = eng.learned_collect(wl.system, wl.pulses, wl.grid, wl.opts(), hist_every=32,
                                      cap=1 << 21)
        okw["mlp"] = api.mlp_init(1, recs)
        eng.mlp_train(recs, okw["mlp"], api.train_opts(epochs=2))
    plan = eng.plan(wl.system, wl.pulses, wl.grid, wl.opts(**okw))
    for _ in range(2):
        plan.execute_async()
        _, st = plan.fetch(copy_j=False)
    print("ok", args.variant, st.attempted_steps, st.kernel_ms, st.poly_degree)
    return 0


def self_launch(args) -> int:
    """--gpus N without a torchrun environment: re-run this command under
    torch.distributed.run with N ranks on this node (127.0.0.1)."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--variant", default=None, choices=sorted(VARIANTS) + ["mlp_train"],
                    help="default: mixed_learned (fp64 for piflux3d_relax)")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1: every rank its own batches (weak) or every batch's k rows "
                         "split over the ranks with j summed by NCCL (strong)")
    ap.add_argument("--pulses-per-step", type=int, default=None,
                    help="pulse instances per step (default: 8 of the 64 for "
                         "honeycomb_1024x64, all of them otherwise)")
    ap.add_argument("--autotune", action="store_true",
                    help="autotune the work decomposition of a single-batch workload first")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run the small profiling case of the workload (no timing)")
    ap.add_argument("--ncu-cycles", type=int, default=1,
                    help="pulse cycles of the --ncu-case workload (the bench uses the full length)")
    ap.add_argument("--ncu-pulses", type=int, default=None,
                    help="pulse instances of the --ncu-case workload (default: all)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="seconds of the GPU arm's CPU-baseline sample")
    ap.add_argument("--reference-seconds", type=float, default=120.0,
                    help="seconds of CPU work of the whole --impl reference run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--no-oracle-check", action="store_true")
    ap.add_argument("--mlp-every", type=int, default=None,
                    help="intervals between network proposals of the learned variants "
                         "(default: the library's)")
    args = ap.parse_args(argv)
    if args.variant is None:
        args.variant = DEFAULT_VARIANT.get(args.workload, "mixed_learned")
    if args.warmup < 3:
        args.warmup = 3
    if args.ncu_case:
        return ncu_case(args)
    if args.variant == "mlp_train":
        ap.error("--variant mlp_train is a profiling case (--ncu-case)")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return self_launch(args)
    if args.workload.startswith("dirac3d_kappa"):
        return dirac_reference_arm(args) if args.impl == "reference" else dirac_arm(args)
    if args.impl == "reference":
        if not _has_ref(args.workload):
            return reference_arm_engine_inputs(args)
        return reference_arm(args)
    return our_arm(args)


def engine_ref_workload(wl, api) -> RefWorkload:
    """Oracle inputs of a workload whose descriptors come from the engine's
    configuration reader (the production PiFlux runs): the descriptors mapped
    onto the oracle's structs (tests/helpers.oracle_args), the engine's k rows."""
    from tests.helpers import oracle_args
    m, p, tc, _ = oracle_args(wl.system, wl.pulses[0], wl.opts_kw["abs_tol"], wl.opts_kw["rel_tol"])
    rows = api.grid_rows(wl.system, wl.grid)
    return RefWorkload(wl.name, [(m, p, tc)], (wl.opts_kw["abs_tol"], wl.opts_kw["rel_tol"]),
                       lambda: rows)


def reference_arm_engine_inputs(args):
    """Reference arm of the workloads without an oracle-side definition (the
    production PiFlux runs, whose inputs come from the engine's configuration
    reader)."""
    from higherharmonics_b200 import api
    from higherharmonics_b200 import workloads as W
    _REF_OVERRIDE[args.workload] = engine_ref_workload(W.ALL[args.workload](), api)
    try:
        return reference_arm(args)
    finally:
        _REF_OVERRIDE.pop(args.workload, None)


_REF_OVERRIDE = {}


if __name__ == "__main__":
    sys.exit(main())
