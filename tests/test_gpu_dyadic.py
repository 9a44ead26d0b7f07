"""The warp-synchronous dyadic stepping's coarsening bound (opts.coarsen_div).

A strong, coarsely sampled pi-flux pulse (A0 = 2, 64 samples per cycle, 8
cycles: 10-14 RKF78 steps per interval, so the level changes within the
intervals) on a 32 x 32 grid, against the CPU oracle (FP64, the reference's
restart controller at 1e-12 / 1e-8).  In FP64 the default bound is the
controller's growth rule (1/600) and a looser one (1/128) stays within the
tolerance-level distance of the oracle; in mixed precision the default is
1/64, which takes fewer attempts than the growth rule and is as accurate.
Every step is still judged by the embedded error estimate.  Out-of-range
bounds are refused.
"""
import math

import pytest

from higherharmonics_b200 import api
from tests.helpers import harmonic_rel_err, harmonics, oracle_j, rel_l2

pytestmark = pytest.mark.gpu

J_TOL_FP64 = 1e-6   # different step sequences at abs 1e-12 / rel 1e-8
BAR = 1e-4          # the fast variants' harmonic bar (and j(t) relative L2)


def _case(n):
    s = 1.0 / math.sqrt(2.0)
    sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
    pulse = api.cosine_pulse(2.0, 8, 8 * 64, window=(0.0, 2 * math.pi * 9), energy_scale=20.0)
    grid = api.grid_tensor(n, n, -math.pi, math.pi, -math.pi, math.pi)
    j_ref, ost = oracle_j(sys, pulse, api.grid_rows(sys, grid), 1e-12, 1e-8)
    return sys, pulse, grid, j_ref, ost


@pytest.fixture(scope="module")
def strong_piflux():
    return _case(32)


def _runs(engine, case, divs, **kw):
    sys, pulse, grid, j_ref, ost = case
    out = {}
    for div in divs:
        j, st = engine.current_density(sys, pulse, grid,
                                       api.solver(proposer=api.PROPOSER_LOCKSTEP, coarsen_div=div,
                                                  **kw))
        assert st.failed_trajectories == 0
        out[div] = (j, st, rel_l2(j, j_ref),
                    harmonic_rel_err(harmonics(j, pulse), harmonics(j_ref, pulse)))
    return out


def test_fp64_default_is_the_growth_rule(engine, strong_piflux):
    r = _runs(engine, strong_piflux, (0, 600, 128), abs_tol=1e-12, rel_tol=1e-8)
    assert (r[0][0] == r[600][0]).all() and r[0][1].attempted_steps == r[600][1].attempted_steps
    for div, (_, st, jerr, herr) in r.items():
        assert jerr <= J_TOL_FP64, (div, jerr)
        assert herr <= BAR, (div, herr)


def test_mixed_default_bound_takes_fewer_steps(engine, strong_piflux):
    """At the mixed tolerances (1e-8 / 1e-6) this strong pulse's harmonic
    error is set by the tolerance, not the precision (the FP64 restart
    controller at the same tolerances: 4.8e-4); the default bound takes 8 %
    fewer attempts than the growth rule and is no less accurate."""
    r = _runs(engine, strong_piflux, (0, 64, 600), abs_tol=1e-8, rel_tol=1e-6,
              precision=api.PREC_MIXED)
    assert (r[0][0] == r[64][0]).all() and r[0][1].attempted_steps == r[64][1].attempted_steps
    for div, (_, st, jerr, herr) in r.items():
        assert jerr <= 1e-5, (div, jerr)
    assert r[0][3] <= 1.25 * r[600][3], (r[0][3], r[600][3])
    assert r[0][1].attempted_steps < 0.97 * r[600][1].attempted_steps, \
        (r[0][1].attempted_steps, r[600][1].attempted_steps)


@pytest.mark.parametrize("div", [1, -3, 65537])
def test_out_of_range_coarsening_bound_is_refused(engine, strong_piflux, div):
    sys, pulse, grid, _, _ = strong_piflux
    with pytest.raises(api.HHGError, match="coarsen_div"):
        engine.current_density(sys, pulse, grid,
                               api.solver(proposer=api.PROPOSER_LOCKSTEP, coarsen_div=div))
