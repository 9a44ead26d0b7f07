"""k-point sharding of one spectrum across ranks.

The reference splits the outer k loop into contiguous blocks per MPI rank
(``jobs_per_rank``, PiFlux.cpp:811-820, Honeycomb.cpp:250-258) and sums the
per-rank j(t) with one MPI_Reduce (sources/hhg.cpp:240-246).  Here each rank
(one process per GPU, torch.distributed) integrates a contiguous block of the
k table and the partial currents are combined either with one all_reduce
(SUM) or, for a bitwise-reproducible result, gathered and summed in rank
order with compensation.
"""
from __future__ import annotations

import numpy as np

from . import api


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of block `rank` when n items are split in `world` contiguous
    blocks of ceil(n / world) (the last block may be short or empty)."""
    jobs = -(-n // world)
    lo = min(rank * jobs, n)
    hi = min(lo + jobs, n)
    return lo, hi


def neumaier_sum(parts) -> np.ndarray:
    """Compensated elementwise sum of equally shaped arrays, in list order."""
    s = np.zeros_like(parts[0], dtype=np.float64)
    c = np.zeros_like(s)
    for v in parts:
        v = np.asarray(v, dtype=np.float64)
        t = s + v
        big = np.abs(s) >= np.abs(v)
        c += np.where(big, (s - t) + v, (v - t) + s)
        s = t
    return s + c


def reduce_current(j_local: np.ndarray, deterministic: bool = True, group=None) -> np.ndarray:
    """Sum per-rank partial currents over the process group."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(j_local, dtype=np.float64)).to(dev)
    if not deterministic:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    return neumaier_sum([p.cpu().numpy() for p in parts])


def shard_rows(rows: np.ndarray, rank: int, world: int) -> np.ndarray:
    lo, hi = shard_range(rows.shape[0], rank, world)
    return rows[lo:hi]


def sharded_current_density(engine, sys, pulses, grid, opts, rank: int, world: int,
                            deterministic: bool = True, group=None):
    """Integrate this rank's block of the k grid on its GPU and reduce j(t)
    over the group; every rank returns the full current."""
    rows = api.grid_rows(sys, grid)
    mine = shard_rows(rows, rank, world)
    if mine.shape[0] == 0:
        n = sum(p.n_measurements + 1 for p in (pulses if isinstance(pulses, list) else [pulses]))
        j = np.zeros(n)
    else:
        g, keep = api.grid_explicit(mine)
        j, _ = engine.current_density(sys, pulses, g, opts)
    return reduce_current(j, deterministic=deterministic, group=group)


def dirac_z_block(n_z: int, rank: int, world: int) -> tuple[int, int]:
    """(z_first, z_count) of `rank`'s block of the Dirac system's z loop
    z = 1 .. n_z - 1, partitioned as the reference does under MPI
    (DiracSystem.cpp:288-295): jobs_per_rank = ceil((n_z - 1) / n_ranks),
    [rank jobs + 1, min(n_z, rank jobs + 1 + jobs))."""
    jobs = (n_z - 1) // world
    if jobs * world < n_z - 1:
        jobs += 1
    lo = rank * jobs + 1
    hi = min(n_z, lo + jobs)
    return lo, max(0, hi - lo)


def sharded_dirac_current_density(engine, sys, pulse, quad, opts, rank: int, world: int,
                                  deterministic: bool = True, group=None):
    """The Dirac-3D current density with the k_z slices split over ranks:
    this rank integrates its block of slices (Engine.dirac_current_density
    with z_first / z_count; each block already carries the factor dz, as the
    reference's per-rank current does) and j(t) is reduced over the group
    (the reference's MPI_Reduce, hhg.cpp:240-246); every rank returns the full
    current."""
    zf, zc = dirac_z_block(quad.n_z, rank, world)
    if zc == 0:
        j = np.zeros(pulse.n_measurements + 1)
    else:
        q = api.kappa_quad(quad.max_k, quad.n_z, quad.n_kappa, quad.threshold, quad.n_splits,
                           quad.max_halvings, z_first=zf, z_count=zc)
        j, _, _ = engine.dirac_current_density(sys, pulse, q, opts)
    return reduce_current(j, deterministic=deterministic, group=group)
