"""GPU checks of the batching layer: CUDA-graph execution of a plan and the
work-decomposition autotuner.  Neither changes any trajectory: the graph
replays the same launches, and the autotuner only regroups k tiles into work
items (which changes the order of the partial-row sums, so j may move by a
few units in the last place)."""
import math

import numpy as np
import pytest

from higherharmonics_b200 import api
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _dirac_batch():
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulses = [api.cosine_pulse(0.3 + 0.2 * i, 1.5 + 0.5 * i, 1024 + 512 * i, phase=0.4 * i,
                               energy_scale=1 / (0.06 + 0.02 * i)) for i in range(4)]
    grid = api.grid_tensor(48, 48, -2, 2, -2, 2)
    return sys, pulses, grid


def test_graph_matches_stream_execution(engine):
    sys, pulses, grid = _dirac_batch()
    opts = api.solver(1e-10, 1e-10)
    plan = engine.plan(sys, pulses, grid, opts)
    plan.execute_async()
    plan.spectrum_async()
    j0, st0 = plan.fetch()
    spec0 = [plan.fetch_spectrum(p) for p in range(len(pulses))]
    for rep in range(2):  # capture, then replay
        plan.execute_graph(with_spectrum=True)
        j1, st1 = plan.fetch()
        assert np.array_equal(j0, j1)
        assert st1.attempted_steps == st0.attempted_steps
        assert st1.kernel_ms > 0 and st1.total_ms >= st1.kernel_ms
        for p in range(len(pulses)):
            for a, b in zip(spec0[p], plan.fetch_spectrum(p)):
                assert np.array_equal(a, b)
    # integration-only graph, then back to the spectrum graph
    plan.execute_graph(with_spectrum=False)
    j2, _ = plan.fetch()
    assert np.array_equal(j0, j2)
    plan.close()


def test_graph_on_caller_stream(engine):
    import torch
    sys, pulses, grid = _dirac_batch()
    plan = engine.plan(sys, pulses[:1], grid, api.solver(1e-10, 1e-10))
    plan.execute_async()
    j0, _ = plan.fetch()
    s = torch.cuda.Stream()
    plan.execute_graph(s.cuda_stream, with_spectrum=False)
    s.synchronize()
    j1, _ = plan.fetch()
    assert np.array_equal(j0, j1)
    plan.close()


@pytest.mark.parametrize("proposer", [api.PROPOSER_NONE, api.PROPOSER_LOCKSTEP])
def test_autotune_keeps_results(engine, proposer):
    s = 1 / math.sqrt(2)
    sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
    pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=20.0)
    grid = api.grid_tensor(96, 96, -math.pi, math.pi, -math.pi, math.pi)
    plan = engine.plan(sys, pulse, grid, api.solver(1e-12, 1e-8, proposer=proposer))
    plan.execute_async()
    j0, st0 = plan.fetch()
    rep = plan.autotune(reps=1)
    cands = rep.as_list()
    assert rep.n_candidates >= 4
    assert {c["tile_k"] for c in cands} >= {1, 2, 4}
    assert all(c["kernel_ms"] > 0 for c in cands)
    assert cands[rep.best]["kernel_ms"] == min(c["kernel_ms"] for c in cands)
    plan.execute_graph(with_spectrum=True)
    j1, st1 = plan.fetch()
    assert st1.attempted_steps == st0.attempted_steps
    assert rel_l2(j1, j0) <= 1e-13
    plan.close()


def test_one_shot_plan_cache_has_no_stale_hits(engine):
    """The one-shot entry point reuses plans for repeated descriptors; any
    change of a descriptor (a pulse field, explicit k rows by value, the
    tolerances) must give the freshly computed result."""
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 1, 512, energy_scale=10.0)
    grid = api.grid_tensor(16, 16, -2, 2, -2, 2)
    opts = api.solver(1e-10, 1e-10)
    a, _ = engine.current_density(sys, pulse, grid, opts)
    b, _ = engine.current_density(sys, pulse, grid, opts)
    assert np.array_equal(a, b)
    pulse2 = api.cosine_pulse(1.1, 1, 512, energy_scale=10.0)
    c, _ = engine.current_density(sys, pulse2, grid, opts)
    assert not np.array_equal(a, c)
    # fresh engine: no cache, same answer for pulse2
    e2 = api.Engine(0)
    c2, _ = e2.current_density(sys, pulse2, grid, opts)
    assert np.array_equal(c, c2)
    rows = api.grid_rows(sys, grid)
    g1, keep1 = api.grid_explicit(rows.copy())
    r1, _ = engine.current_density(sys, pulse, g1, opts)
    assert np.array_equal(r1, a)
    rows2 = rows.copy()
    rows2[:, 3] *= 2.0  # weights doubled -> j doubled, same buffer address pattern
    g2, keep2 = api.grid_explicit(rows2)
    r2, _ = engine.current_density(sys, pulse, g2, opts)
    assert np.allclose(r2, 2 * a, rtol=1e-14, atol=0)
    # the restart schedule makes the step sequence tolerance-independent here;
    # the carried proposal changes it
    d, std = engine.current_density(sys, pulse, grid, api.solver(1e-10, 1e-10,
                                                                 proposer=api.PROPOSER_CARRY))
    assert not np.array_equal(a, d)
    e2.close()


def test_plans_share_the_k_table_of_a_grid(engine):
    """Plans built on one context from the same system and generated grid
    share one device k table: the results equal a fresh context's, whichever
    plan is destroyed first, and a plan on another grid (or another system)
    gets its own table."""
    sys, pulses, grid = _dirac_batch()
    opts = api.solver(1e-10, 1e-10)
    p1 = engine.plan(sys, pulses[:1], grid, opts)
    p2 = engine.plan(sys, pulses[1:2], grid, opts)
    p3 = engine.plan(sys, pulses[1:2], api.grid_tensor(40, 40, -2, 2, -2, 2), opts)
    sys_m = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.07)
    p4 = engine.plan(sys_m, pulses[1:2], grid, opts)
    p1.close()  # p2 keeps the shared table alive
    fresh = api.Engine(0)
    try:
        for pl, (s, g) in ((p2, (sys, grid)), (p3, (sys, api.grid_tensor(40, 40, -2, 2, -2, 2))),
                           (p4, (sys_m, grid))):
            pl.execute_async()
            j, _ = pl.fetch()
            ref, _ = fresh.current_density(s, pulses[1:2], g, opts)
            assert np.array_equal(j, ref)
        # a plan built after the others were closed, on the first grid again
        for pl in (p2, p3, p4):
            pl.close()
        p5 = engine.plan(sys, pulses[:1], grid, opts)
        p5.execute_async()
        j, _ = p5.fetch()
        ref, _ = fresh.current_density(sys, pulses[:1], grid, opts)
        assert np.array_equal(j, ref)
        p5.close()
    finally:
        fresh.close()
