#!/usr/bin/env python
"""Benchmark: spectra/s of the per-k-point Bloch integration -> BZ current
sum -> trapezoidal FFT path on the 256x256 PiFlux-2D workload.

One step = one spectrum: integrate all 65 536 k-points over the 8-cycle
pulse (8192 measurement intervals), reduce j(t), FFT it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--variant NAME]
  python bench.py --impl reference ...   # the oracle port on the host cores

Under torchrun (N > 1) every rank integrates its own pulse instance (the
carrier phase differs per rank): weak scaling with no data-path collective;
the only collectives are the barrier and the max-over-ranks timing.
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

METRIC = "spectra/sec at harmonic err <=1e-4 vs FP64"
UNIT = "spectra/s"

# Algorithmic FP64 flops per attempted RKF78 step (one k-point): 13 right-hand
# sides plus the tableau arithmetic 2*3*55 (stages) + 2*3*7 (solution) +
# 2*3*4 (error) + ~25 (norm and control) = 421; the right-hand side of the
# 2D pi-flux model costs 12 flops plus two cosines (counted separately).
# The PiFlux relaxation right-hand side (PiFlux.cpp:113-186 in the kernel's
# form: off-diagonal equilibrium as the normalised perpendicular part of the
# start state, Fermi pair through one reciprocal square root) costs 76 flops:
# cos(kz - A) 3, |u|^2 5, |u| 1, occupation energies 4, Fermi pair 11,
# g_d (a2 - b2)/|u| 2, coherent part with -g_s S + g_d r_d 24, perpendicular
# projection, its norm and the g_o term 26; plus 5 special operations (2 exp,
# 3 rsqrt).
ALG_FLOPS_PER_KSTEP = {"piflux2d_256": 13 * 12 + 421, "dirac2d_64": 13 * 16 + 421,
                       "honeycomb_512": 13 * 30 + 421, "dirac2d_sweep": 13 * 16 + 421,
                       "piflux3d_relax": 13 * 76 + 421, "piflux3d_field": 13 * 12 + 421}
SPECIAL_OPS_PER_KSTEP = {"piflux2d_256": 26, "dirac2d_64": 0, "honeycomb_512": 78,
                         "dirac2d_sweep": 0, "piflux3d_relax": 13 * 5}
# the relaxation workload runs the reference step schedule in FP64 only
DEFAULT_VARIANT = {"piflux3d_relax": "fp64"}
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


def train_proposer(eng, wl, api):
    """Step-size history of a carry run of the same workload at the plain
    tolerances -> the learned proposer, trained on the GPU (outside the timed
    region; reported under "training")."""
    p = wl.pulses[0]
    every = max(1, math.ceil(wl.n_k * p.n_measurements / LEARNED_RECORDS))
    t0 = time.perf_counter()
    recs, cst = eng.learned_collect(wl.system, wl.pulses, wl.grid, wl.opts(), hist_every=every,
                                    cap=LEARNED_RECORDS)
    t1 = time.perf_counter()
    net = api.mlp_init(1, recs)
    loss, train_ms = eng.mlp_train(recs, net, api.train_opts(epochs=LEARNED_EPOCHS))
    t2 = time.perf_counter()
    return net, {"records": int(recs.shape[0]), "hist_every": every,
                 "collect_s": t1 - t0, "train_s": t2 - t1, "train_device_ms": train_ms,
                 "epochs": LEARNED_EPOCHS, "loss_first_last": [float(loss[0]), float(loss[-1])],
                 "network": "8-64-64-64-1 SiLU, BF16/FP32, tcgen05 training"}


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


class CpuBaseline:
    """The oracle port timed on the host cores over a strided k-subsample of
    the workload; spectra/s are extrapolated to the full grid."""

    def __init__(self, wl, rows, target_s: float):
        from oracle import hhg_oracle as O
        from tests.helpers import oracle_args
        self.O = O
        p = wl.pulses[0]
        self.args = oracle_args(wl.system, p, wl.opts_kw["abs_tol"], wl.opts_kw["rel_tol"])
        self.cores = (len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity")
                      else os.cpu_count())
        self.n_k = rows.shape[0]
        m, p, tc, s = self.args
        calib = rows[:: max(1, self.n_k // max(self.cores, 8))][: max(self.cores, 8)]
        t0 = time.perf_counter()
        O.current_density(m, p, tc, s, calib, threads=self.cores, fast=True)
        per_k = (time.perf_counter() - t0) / calib.shape[0]
        n_sample = int(min(self.n_k, max(self.cores, target_s / max(per_k, 1e-9))))
        self.stride = max(1, self.n_k // n_sample)
        self.sample = np.ascontiguousarray(rows[:: self.stride])
        self.n_meas = tc.n_measurements

    def run(self):
        m, p, tc, s = self.args
        t0 = time.perf_counter()
        _, st, rc = self.O.current_density(m, p, tc, s, self.sample, threads=self.cores,
                                           fast=True)
        el = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"oracle status {rc}")
        spectra_per_s = 1.0 / (el * self.n_k / self.sample.shape[0])
        desc = (f"every {self.stride}th k-point ({self.sample.shape[0]} of {self.n_k}) over the "
                f"full {self.n_meas}-interval pulse, {st.attempted} k.steps in {el:.2f} s on "
                f"{self.cores} threads (oracle port, -O3 -ffast-math, OpenMP); spectra/s "
                f"scaled by {self.n_k}/{self.sample.shape[0]}")
        return spectra_per_s, desc, st.attempted / el


def reference_arm(args, wl_name):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from higherharmonics_b200 import workloads as W
    from higherharmonics_b200 import api
    wl = W.ALL[wl_name]()
    rows = api.grid_rows(wl.system, wl.grid)
    cb = CpuBaseline(wl, rows, target_s=args.cpu_seconds)
    per_step = []
    desc = ksps = None
    for i in range(args.warmup + args.steps):
        v, desc, ksps = cb.run()
        if i >= args.warmup:
            per_step.append(1.0 / v)
    t = float(np.mean(per_step))
    value = 1.0 / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_for(wl, "oracle port, plain FP64 RKF78"),
        "k_steps_per_s": ksps,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb.cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_for(wl, variant_desc, okw=None):
    p = wl.pulses[0]
    tol = dict(wl.opts_kw)
    tol.update({k: v for k, v in (okw or {}).items() if k in ("abs_tol", "rel_tol")})
    return {"workload": wl.name, "k_points": wl.n_k, "n_measurements": p.n_measurements,
            "pulses": len(wl.pulses), "tolerances": f"{tol['abs_tol']:g}/{tol['rel_tol']:g}",
            "variant": variant_desc,
            "l2": "flushed (256 MiB write) before every timed step; inputs < L2"}


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


def compare_variants(args, eng, wl, api, stream, flush, main_variant):
    """spectra/s of the plain FP64 path and of the learned mixed-precision
    path on the same workload, same timing method (CUDA events over K graph
    launches, L2 flushed before each): the learned+FP32 vs plain FP64 ratio."""
    import torch
    from higherharmonics_b200.analysis import (default_max_order, harmonic_intensities,
                                               harmonic_rel_err)
    # the plain FP64 spectrum every variant's harmonic error refers to
    ref = eng.plan(wl.system, wl.pulses, wl.grid, wl.opts())
    ref.execute_async()
    ref.spectrum_async()
    ref.fetch(copy_j=False)
    fr0, re0, im0 = ref.fetch_spectrum(0)
    ref.close()
    mo = default_max_order(fr0)
    I0 = harmonic_intensities(fr0, re0, im0, mo)
    out = {}
    for v in ("fp64", "mixed_learned", "mixed_lockstep", "magnus4"):
        if v == main_variant or (v != "fp64" and args.workload in DEFAULT_VARIANT):
            continue
        okw = dict(VARIANTS[v])
        if okw.get("proposer") == api.PROPOSER_LEARNED:
            okw["mlp"], _ = train_proposer(eng, wl, api)
            if args.mlp_every:
                okw["mlp_every"] = args.mlp_every
        plan = eng.plan(wl.system, wl.pulses, wl.grid, wl.opts(**okw))
        plan.autotune(reps=1)
        sptr = stream.cuda_stream
        for _ in range(3):
            flush.zero_()
            plan.execute_graph(sptr, with_spectrum=True)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            plan.execute_graph(sptr, with_spectrum=True)
        b.record(stream)
        torch.cuda.synchronize()
        _, st = plan.fetch(copy_j=False)
        fr, re, im = plan.fetch_spectrum(0)
        out[v] = {"value": args.steps * len(wl.pulses) / (a.elapsed_time(b) * 1e-3), "unit": UNIT,
                  "k_steps_per_spectrum": st.attempted_steps,
                  "harmonic_err_vs_fp64": harmonic_rel_err(harmonic_intensities(fr, re, im, mo), I0,
                                                           floor_rel=1e-6)}
        plan.close()
    return out


def our_arm(args, wl_name):
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
    from higherharmonics_b200.analysis import (default_max_order, harmonic_intensities,
                                               harmonic_rel_err)

    wl = W.ALL[wl_name]()
    if ws > 1:  # one pulse instance per rank: weak scaling
        for p in wl.pulses:
            p.phase = p.phase + 0.1 * rank
    eng = api.Engine(dev)
    okw = dict(VARIANTS[args.variant])
    training = None
    if okw.get("proposer") == api.PROPOSER_LEARNED:
        net, training = train_proposer(eng, wl, api)
        okw["mlp"] = net
        if args.mlp_every:
            okw["mlp_every"] = args.mlp_every
    plan = eng.plan(wl.system, wl.pulses, wl.grid, wl.opts(**okw))
    tune = plan.autotune(reps=2)
    # a dedicated stream: the legacy default stream has handle 0, which the
    # C ABI reads as "the context's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr != 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        flush.zero_()
        plan.execute_graph(sptr, with_spectrum=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    j0, st0 = plan.fetch()
    ksteps = st0.attempted_steps

    # accuracy of this variant against the plain FP64 engine (itself within
    # 1e-9 of the oracle, see tests/test_gpu_parity.py)
    herr = 0.0
    if args.variant != "fp64":
        fr, re, im = plan.fetch_spectrum(0)
        ref = eng.plan(wl.system, wl.pulses, wl.grid, wl.opts())
        ref.execute_async()
        ref.spectrum_async()
        ref.fetch(copy_j=False)
        fr0, re0, im0 = ref.fetch_spectrum(0)
        ref.close()
        mo = default_max_order(fr0)
        herr = harmonic_rel_err(harmonic_intensities(fr, re, im, mo),
                                harmonic_intensities(fr0, re0, im0, mo), floor_rel=1e-6)

    peak = eng.fp64_peak_tflops()
    mixed = VARIANTS[args.variant].get("precision", 0) == 1
    peak32 = eng.fp32_peak_tflops() if mixed else None
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
        flush.zero_()
        ev[k][0].record(stream)
        plan.execute_graph(sptr, with_spectrum=True)
        ev[k][1].record(stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    elapsed_ms = e_start.elapsed_time(e_end)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    step_sum_ms = sum(ev[k][0].elapsed_time(ev[k + 1][0]) for k in range(args.steps - 1))
    if ws > 1:
        t = torch.tensor([elapsed_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    # one step = every pulse instance's spectrum (one graph launch)
    value = ws * args.steps * len(wl.pulses) / (elapsed_ms * 1e-3)

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        n_e2e = max(1, min(args.steps, 3))
        eng.current_density(wl.system, wl.pulses, wl.grid, wl.opts(**okw))
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            j, st = eng.current_density(wl.system, wl.pulses, wl.grid, wl.opts(**okw))
            off = 0
            for p in wl.pulses:  # every pulse instance's spectrum
                n_s = p.n_measurements + 1
                eng.spectrum(j[off:off + n_s], p.n_measurements, p.window_begin, p.window_end)
                off += n_s
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if ws > 1:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            el = float(t.item())
        # k table and pulse records in; per pulse: the staging time grid
        # (2 x samples) and j back into the spectrum call; out: j and the
        # spectrum's three arrays
        h2d = wl.n_k * 64 + 256 * len(wl.pulses)
        d2h = 0
        for p in wl.pulses:
            n_s = p.n_measurements + 1
            n_fft = 4 * n_s + 1
            h2d += 8 * n_s * 2 + 8 * n_s
            d2h += 8 * n_s + 3 * 8 * n_fft
        e2e = {"value": ws * n_e2e * len(wl.pulses) / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": "Engine.current_density + Engine.spectrum (hhg_gpu_current_density + "
                       "hhg_gpu_spectrum), host buffers, wall clock"}

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0
    avg_launch_s = float(np.mean(launch_ms)) * 1e-3
    # the graph launch = integration kernel + BZ reduction + FFT (the
    # integration is >= 98 % of it in the launch list), so this slightly
    # understates the kernel's own throughput
    kernel_s = avg_launch_s
    per_kstep = ALG_FLOPS_PER_KSTEP.get(wl_name, 421)
    if VARIANTS[args.variant].get("stepper", 0) == 1:
        per_kstep = MAGNUS4_FLOPS_PER_KSTEP
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
    achieved = bflops * ksteps / kernel_s / 1e12
    roofline = {"bound": bound, "achieved": achieved, "peak": bpeak, "unit": "TFLOP/s",
                "frac": achieved / bpeak, "traffic": traffic_from_profile(wl_name),
                "peak_source": peak_src, "fp64_peak": peak, "fp32_peak": peak32,
                "kernel": "bz_integrate_kernel", "kernel_ms": 1e3 * kernel_s,
                "kernel_ms_source": "mean over the timed steps of CUDA events around each graph "
                                    "launch (integration + reduction + FFT) on the launching stream",
                "alg_flops_per_kstep": per_kstep, "bound_flops_per_kstep": bflops,
                "special_ops_per_kstep": (2 if VARIANTS[args.variant].get("stepper", 0) == 1
                                          else SPECIAL_OPS_PER_KSTEP.get(wl_name, 0))}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if VARIANTS[args.variant].get("precision", 0) == 0 else "f32 rhs / f64 state",
        "data": "synthetic", "config": config_for(wl, args.variant, VARIANTS[args.variant]),
        "k_steps_per_s": ws * ksteps / kernel_s if ws == 1 else None,
        "fraction_of_fp64_peak_fp64_equivalent": per_kstep * ksteps / kernel_s / 1e12 / peak,
        "k_steps_per_spectrum": ksteps, "harmonic_err_vs_fp64": herr,
        "gpu_launches": 4 * args.steps, "roofline": roofline, "clocks": clocks, "e2e": e2e,
        "training": training,
        "autotune": {"chosen": tune.as_list()[tune.best], "candidates": tune.as_list()},
        "path": "plan with autotuned work decomposition, one CUDA graph launch per spectrum "
                "(integration + BZ reduction + trapezoidal FFT)",
        "timing": {"device_ms_total": elapsed_ms, "launch_ms": launch_ms,
                   "mean_step_ms_between_launch_starts": (step_sum_ms / (args.steps - 1)
                                                          if args.steps > 1 else None)},
    }
    if ws == 1 and not args.no_cpu_baseline:
        rows = api.grid_rows(wl.system, wl.grid)
        cb = CpuBaseline(wl, rows, target_s=args.cpu_seconds)
        v, desc, ksps = cb.run()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cb.cores, "kind": "port",
                                "sample": desc, "k_steps_per_s": ksps}
    if ws == 1 and not args.no_compare:
        line["compare"] = compare_variants(args, eng, wl, api, stream, flush, args.variant)
    print(json.dumps(line), flush=True)
    plan.close()
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


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
        t0 = time.perf_counter()
        info = self._splits(self.sample)
        el = time.perf_counter() - t0
        n_all = len(self.pairs)
        v = 1.0 / (el * n_all / len(self.sample))
        kint = info["trajectories"] * self.tc.n_measurements
        desc = (f"{len(self.sample)} of {n_all} (k_z slice, kappa split) pairs, evenly spaced, "
                f"each refined to convergence ({info['trajectories']} trajectories, {kint} "
                f"k.intervals) in {el:.2f} s on {self.cores} threads (oracle port, -O3 "
                f"-ffast-math, OpenMP); "
                f"spectra/s scaled by {n_all}/{len(self.sample)}")
        return v, desc, kint / el


def dirac_config(wl, path):
    q = wl.quad
    return {"workload": wl.name, "n_z": q.n_z, "n_kappa": q.n_kappa, "n_splits": q.n_splits,
            "kappa_threshold": q.threshold, "max_k": q.max_k,
            "n_measurements": wl.pulse.n_measurements,
            "stepper": ("closed-form Magnus (FP64)" if wl.opts.stepper == 2 else
                        "RKF78 with relaxation, reference schedule (FP64)"),
            "l2": "flushed (256 MiB write) before every timed step", "path": path}


def dirac_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from higherharmonics_b200 import workloads as W
    wl = W.ALL[args.workload]()
    cb = DiracCpuBaseline(wl, args.cpu_seconds)
    per = []
    desc = None
    for i in range(args.warmup + args.steps):
        v, desc, _ = cb.run()
        if i >= args.warmup:
            per.append(1.0 / v)
    t = float(np.mean(per))
    line = {"impl": "reference", "metric": METRIC, "value": 1.0 / t, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dirac_config(wl, "oracle port"),
            "cpu_baseline": {"value": 1.0 / t, "unit": UNIT, "cores": cb.cores, "kind": "port",
                             "sample": desc},
            "e2e": {"value": 1.0 / t, "unit": UNIT, "h2d_bytes_per_step": 0,
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
        v, desc, kps = cb.run()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cb.cores, "kind": "port",
                                "sample": desc, "k_intervals_per_s": kps}
    print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def ncu_case(args):
    """A small case of the bench workload for ncu captures (committed so the
    profile summaries name a command that runs committed files only): the
    same grid and pulse shape over --ncu-cycles cycles (default 1: 1024
    intervals), two executions
    of the selected variant; with --variant mlp_train, history collection on
    that case and 2 epochs of proposer training.  Prints one line, no timing."""
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="piflux2d_256")
    ap.add_argument("--variant", default=None, choices=sorted(VARIANTS) + ["mlp_train"],
                    help="default: mixed_lockstep (fp64 for piflux3d_relax)")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run the small profiling case of the workload (no timing)")
    ap.add_argument("--ncu-cycles", type=int, default=1,
                    help="pulse cycles of the --ncu-case workload (the bench uses the full length)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--mlp-every", type=int, default=None,
                    help="intervals between network proposals of the learned variants "
                         "(default: the library's)")
    args = ap.parse_args()
    if args.variant is None:
        args.variant = DEFAULT_VARIANT.get(args.workload, "mixed_lockstep")
    if args.warmup < 3:
        args.warmup = 3
    if args.ncu_case:
        return ncu_case(args)
    if args.variant == "mlp_train":
        ap.error("--variant mlp_train is a profiling case (--ncu-case)")
    if args.workload.startswith("dirac3d_kappa"):
        return dirac_reference_arm(args) if args.impl == "reference" else dirac_arm(args)
    if args.impl == "reference":
        return reference_arm(args, args.workload)
    return our_arm(args, args.workload)


if __name__ == "__main__":
    sys.exit(main())
