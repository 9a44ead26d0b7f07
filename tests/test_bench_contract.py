"""bench.py on the CPU: the JSON line of its reference arm (`--impl
reference`, tiny samples) with the keys and meanings the benchmark contract
requires, the arm's independence from the engine (it builds its inputs from
the oracle alone and loads no engine library), and the oracle-side workload
definitions against the engine's (the GPU arm itself runs on the GPU)."""
import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_line(*extra):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
           "--warmup", "3", "--reference-seconds", "2", *extra]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["honeycomb_1024x64", "piflux2d_256", "dirac3d_kappa"])
def test_reference_arm_line(workload):
    d = _reference_line("--workload", workload)
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e", "timed_fraction"):
        assert key in d, key
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    assert d["unit"] == "spectra/s" and d["higher_is_better"] is True and d["value"] > 0
    # ms_per_step is the measured wall time of a step: value x time = the
    # fraction of a spectrum a step integrates
    frac = d["value"] * d["ms_per_step"] * 1e-3
    assert abs(frac - d["timed_fraction"]) <= 1e-9 * max(frac, 1e-30) + 1e-15
    assert 0 < d["timed_fraction"] <= 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_loads_no_engine_code():
    """The default workload's reference arm imports nothing of the engine
    package and maps no engine library."""
    code = (
        "import sys; sys.argv = ['bench.py']; import bench; "
        "rc = bench.main(['--impl', 'reference', '--steps', '1', '--warmup', '3', "
        "'--reference-seconds', '1']); "
        "eng = [m for m in sys.modules if m.startswith('higherharmonics_b200')]; "
        "maps = open('/proc/self/maps').read(); "
        "print('ENGINE', eng, 'libhhg_gpu' in maps, rc)")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600, check=True)
    tail = [ln for ln in out.stdout.splitlines() if ln.startswith("ENGINE")][0]
    assert tail == "ENGINE [] False 0", tail


@pytest.mark.parametrize("name", ["dirac2d_64", "piflux2d_256", "honeycomb_512", "dirac2d_sweep",
                                  "honeycomb_1024x64"])
def test_oracle_side_workloads_match_the_engines(name):
    """bench.ref_workload (oracle inputs) describes the same runs as
    higherharmonics_b200.workloads: pulses, time grids, scaled model constants,
    tolerances and (spot-checked) k rows."""
    sys.path.insert(0, ROOT)
    import bench
    from higherharmonics_b200 import api
    from higherharmonics_b200 import workloads as W
    from tests.helpers import oracle_args
    wl = W.ALL[name]()
    rw = bench.ref_workload(name)
    assert len(rw.jobs) == len(wl.pulses)
    assert rw.tol == (wl.opts_kw["abs_tol"], wl.opts_kw["rel_tol"])
    for (m, p, tc), pd in zip(rw.jobs, wl.pulses):
        m2, p2, tc2, _ = oracle_args(wl.system, pd, *rw.tol)
        for f, _ in type(m)._fields_:
            assert getattr(m, f) == getattr(m2, f), (f, getattr(m, f), getattr(m2, f))
        assert (p.amplitude, p.n_cycles, p.t_begin, p.phase) == \
            (p2.amplitude, p2.n_cycles, p2.t_begin, p2.phase)
        for f, _ in type(tc)._fields_:
            assert getattr(tc, f) == getattr(tc2, f), f
    if name in ("honeycomb_1024x64", "dirac2d_sweep"):
        # spot check: the first and last rows and an evenly spaced subset
        rows = api.grid_rows(wl.system, wl.grid)
        sel = np.r_[0:8, np.linspace(0, rows.shape[0] - 1, 64).astype(int)]
        assert np.allclose(rw.rows[sel], rows[sel], rtol=0, atol=1e-15)
    else:
        assert np.allclose(rw.rows, api.grid_rows(wl.system, wl.grid), rtol=0, atol=1e-15)
    assert math.isfinite(rw.rows[:, 3].sum())


def test_gpus_flag_self_launches_ranks():
    """--gpus 2 outside torchrun re-launches bench.py under
    torch.distributed.run with two ranks (127.0.0.1); the reference arm runs on
    rank 0 only and prints one line for the whole job."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--reference-seconds", "1"]
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, check=True,
                         env=env)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout + out.stderr
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["impl"] == "reference"
