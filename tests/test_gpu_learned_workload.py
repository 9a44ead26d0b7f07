"""The learned-proposer workload (honeycomb + staggered mass 0.1 on the
rhombic BZ, 64 seeded pulse instances with A0 ~ U[0.5, 2] and random carrier
phase, omega = 0.08, 6 cycles) on a reduced grid, against the CPU oracle.

The first 8 pulse instances of the workload's own pulse table, full 6144-
interval pulses, run as one batched plan (one persistent launch) on a 16 x 16
rhombic grid: the plain FP64 RKF78 path within the parity bar (j(t) relative
L2 <= 1e-9, harmonics <= 1e-6 above the noise floor) pulse by pulse.

The fast variants (mixed precision with the lockstep and learned proposers,
Magnus-4) within the harmonic bar of 1e-4 against the oracle, on 2048 of the
workload's own 1024 x 1024 k rows (every 511th, an explicit-rows grid) and its
first 4 pulse instances.  The FP32 right-hand side's rounding is independent
from k-point to k-point and averages out in the Brillouin-zone sum, so its
harmonic error shrinks with the number of k-points: on 256 k-points (the 16 x
16 grid) it is 3e-4, on the full grid 1e-6 against the FP64 engine.
"""
import numpy as np
import pytest

from higherharmonics_b200 import api
from higherharmonics_b200 import workloads as W
from tests.helpers import harmonic_rel_err, harmonics, oracle_j, rel_l2

pytestmark = pytest.mark.gpu

J_TOL = 1e-9
H_TOL = 1e-6
FAST_H_TOL = 1e-4
N_PULSES = 8


@pytest.fixture(scope="module")
def reduced():
    wl = W.honeycomb_1024x64(n_grid=16)
    pulses = wl.pulses[:N_PULSES]
    rows = api.grid_rows(wl.system, wl.grid)
    refs = [oracle_j(wl.system, p, rows, 1e-12, 1e-8) for p in pulses]
    return wl, pulses, refs


def _split(j, pulses):
    out, off = [], 0
    for p in pulses:
        n = p.n_measurements + 1
        out.append(j[off:off + n])
        off += n
    return out


def test_batched_fp64_parity_with_the_oracle(engine, reduced):
    wl, pulses, refs = reduced
    j, st = engine.current_density(wl.system, pulses, wl.grid, wl.opts())
    assert st.failed_trajectories == 0
    total = 0
    for jp, p, (jr, ost) in zip(_split(j, pulses), pulses, refs):
        assert rel_l2(jp, jr) <= J_TOL, rel_l2(jp, jr)
        assert harmonic_rel_err(harmonics(jp, p), harmonics(jr, p)) <= H_TOL
        total += ost.attempted
    assert abs(st.attempted_steps - total) <= 1e-3 * total


@pytest.fixture(scope="module")
def subsample():
    wl = W.honeycomb_1024x64()
    pulses = wl.pulses[:4]
    rows = np.ascontiguousarray(api.grid_rows(wl.system, wl.grid)[::511][:2048])
    grid, keep = api.grid_explicit(rows)
    refs = [oracle_j(wl.system, p, rows, 1e-12, 1e-8) for p in pulses]
    wl.grid = grid
    return wl, pulses, refs, keep


@pytest.mark.parametrize("variant", ["mixed_lockstep", "mixed_learned", "magnus4"])
def test_fast_variants_within_the_harmonic_bar_of_the_oracle(engine, subsample, variant):
    wl, pulses, refs, _ = subsample
    okw = {"mixed_lockstep": dict(precision=api.PREC_MIXED, proposer=api.PROPOSER_LOCKSTEP,
                                  abs_tol=1e-8, rel_tol=1e-6),
           "mixed_learned": dict(precision=api.PREC_MIXED, proposer=api.PROPOSER_LEARNED,
                                 abs_tol=1e-8, rel_tol=1e-6),
           "magnus4": dict(stepper=api.STEPPER_MAGNUS4, magnus_substeps=1)}[variant]
    if variant == "mixed_learned":
        # a network trained (briefly) on a different configuration's histories
        src = W.honeycomb_512(n_grid=32)
        recs, _ = engine.learned_collect(src.system, src.pulses, src.grid, src.opts(),
                                         hist_every=4, cap=1 << 18)
        net = api.mlp_init(1, recs)
        engine.mlp_train(recs, net, api.train_opts(epochs=3))
        okw["mlp"] = net
    j, st = engine.current_density(wl.system, pulses, wl.grid, wl.opts(**okw))
    assert st.failed_trajectories == 0
    for jp, p, (jr, _) in zip(_split(j, pulses), pulses, refs):
        herr = harmonic_rel_err(harmonics(jp, p), harmonics(jr, p))
        assert herr <= FAST_H_TOL, (variant, herr)
        assert rel_l2(jp, jr) <= FAST_H_TOL, (variant, rel_l2(jp, jr))
