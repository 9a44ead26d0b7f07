"""World-size-2 gloo tests of the k sharding and the j(t) reduction (CPU).

Each rank integrates its contiguous block of k rows (here with the CPU
oracle standing in for the per-rank GPU) and the partial currents are
reduced; the result must equal the single-process sum.
"""
import math
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from higherharmonics_b200.distributed import neumaier_sum, shard_range


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 64, 1001):
        for w in (1, 2, 3, 8):
            got = [shard_range(n, r, w) for r in range(w)]
            idx = [i for lo, hi in got for i in range(lo, hi)]
            assert idx == list(range(n))


def test_neumaier_is_order_robust():
    rng = np.random.default_rng(0)
    parts = [rng.normal(size=16) * 1e8 for _ in range(5)] + [rng.normal(size=16)]
    parts.append(-sum(parts[:5]))
    s = neumaier_sum(parts)
    assert np.allclose(s, parts[5], rtol=0, atol=1e-6)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q, deterministic):
    import torch.distributed as dist

    from higherharmonics_b200.distributed import reduce_current, shard_rows
    from oracle import hhg_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = O.model(O.DIRAC2D, velocity=10.0, mass=0.5)
    rows = O.grid_tensor(m, 10, 10, -2, 2, -2, 2)
    p = O.Pulse(0.9, 1)
    tc = O.time_config(0.0, p.t_end, 256)
    mine = shard_rows(rows, rank, world)
    j, _, rc = O.current_density(m, p, tc, O.solver(1e-10, 1e-10), mine, threads=1)
    total = reduce_current(j, deterministic=deterministic)
    out_q.put((rank, total, j))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("deterministic", [True, False])
def test_two_rank_reduction_matches_single_process(deterministic):
    from oracle import hhg_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, deterministic)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    res.sort(key=lambda r: r[0])
    m = O.model(O.DIRAC2D, velocity=10.0, mass=0.5)
    rows = O.grid_tensor(m, 10, 10, -2, 2, -2, 2)
    p = O.Pulse(0.9, 1)
    tc = O.time_config(0.0, p.t_end, 256)
    full, _, _ = O.current_density(m, p, tc, O.solver(1e-10, 1e-10), rows, threads=1)
    for _, total, _ in res:
        assert np.allclose(total, full, rtol=1e-12, atol=1e-14 * np.max(np.abs(full)))
    # both ranks hold the same reduced current
    assert np.array_equal(res[0][1], res[1][1])


def test_dirac_z_blocks_follow_the_reference_partition():
    from higherharmonics_b200.distributed import dirac_z_block
    for n_z in (3, 4, 7, 51, 60):
        for w in (1, 2, 3, 8):
            zs = []
            for r in range(w):
                zf, zc = dirac_z_block(n_z, r, w)
                # DiracSystem.cpp:288-295
                jobs = -(-(n_z - 1) // w)
                lo = r * jobs + 1
                hi = n_z if lo + jobs > n_z else lo + jobs
                assert (zf, zc) == (lo, max(0, hi - lo))
                zs += list(range(zf, zf + zc))
            assert zs == list(range(1, n_z))


class _OracleDiracEngine:
    """Stands in for one rank's GPU: the oracle's kappa rule on the block of
    slices the quadrature descriptor names."""

    def __init__(self):
        from oracle import hhg_oracle as O
        self.O = O

    def dirac_current_density(self, sys, pulse, quad, opts):
        O = self.O
        m = O.model(O.DIRAC3D)
        p = O.Pulse(pulse.amplitude, pulse.n_cycles, pulse.t_begin)
        tc = O.time_config(pulse.window_begin, pulse.window_end, pulse.n_measurements)
        s = O.solver(stepper=2)
        dz = 2 * quad.max_k / quad.n_z
        zs = range(quad.z_first, quad.z_first + quad.z_count)
        kz = [(z - quad.n_z // 2) * dz for z in zs if z != quad.n_z // 2]
        kmax = [math.sqrt(quad.max_k ** 2 - k * k) for k in kz]

        def contrib(rows):
            out, rc = O.k_resolved(m, p, tc, s, rows, 0, threads=1)
            return out[:, :, 2] * rows[:, 3][None, :]

        j, info = O.adaptive_kappa(contrib, kz, kmax, quad.n_kappa, quad.threshold,
                                   quad.n_splits, quad.max_halvings, dz,
                                   tc.n_measurements + 1,
                                   lambda z, a, H, L: O.kappa_rows(m, kz[z], a, H, L, quad.n_kappa))
        return j, info, None


DIRAC_ARGS = dict(max_k=2.0, n_z=7, n_kappa=3, threshold=1e-5, n_splits=2, max_halvings=6)


def _dirac_worker(rank, world, port, out_q):
    import torch.distributed as dist

    from higherharmonics_b200 import api
    from higherharmonics_b200.distributed import sharded_dirac_current_density
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pulse = api.cosine_pulse(0.6, 1, 64)
    total = sharded_dirac_current_density(_OracleDiracEngine(), None, pulse,
                                          api.kappa_quad(**DIRAC_ARGS), None, rank, world)
    out_q.put((rank, total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_dirac_slices_match_single_process():
    from oracle import hhg_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dirac_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    m = O.model(O.DIRAC3D)
    full, _, rc = O.dirac_kappa_current(m, O.Pulse(0.6, 1, 0.0), O.time_config(0.0, 2 * math.pi, 64),
                                        O.solver(stepper=2), **DIRAC_ARGS)
    assert rc == 0 and np.max(np.abs(full)) > 0
    for _, total in res:
        assert np.allclose(total, full, rtol=1e-12, atol=1e-14 * np.max(np.abs(full)))
