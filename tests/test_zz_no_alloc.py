"""The allocation-free entry point hhg_gpu_current_density_noalloc.

It serves callers that cannot allocate device memory during the call (code
under another framework's allocator, real-time loops that cannot afford
cudaMalloc's implicit synchronisation, jobs that budget a shared GPU byte by
byte): the caller owns the device buffers for the k table and j, and the
integration scratch sits in the library's fixed 64 MiB device array.

Checked through the C ABI against the regular entry point
(hhg_gpu_current_density) on two consecutive calls -- the second call runs on
whatever the first left in the shared scratch array -- within the parity
tolerance of the GPU tests (relative L2 <= 1e-9), for the restart and carry
proposers, the mixed-precision right-hand side and Magnus-4; an asynchronous
call (stats == NULL) whose outcome is read afterwards with hhg_noalloc_status,
including a step-limit status; the asynchronous call captured into a CUDA graph
and replayed.  This file is collected last so a failure here
does not stop the rest of the GPU suite.
"""
import ctypes
import math

import numpy as np
import pytest

from higherharmonics_b200 import api

pytestmark = pytest.mark.gpu

J_TOL = 1e-9


def _noalloc(lib, sys, pulse, d_rows, n_rows, opts, d_j, stats=True, stream=None):
    err = ctypes.create_string_buffer(512)
    st = api.Stats()
    rc = lib.hhg_gpu_current_density_noalloc(ctypes.byref(sys), ctypes.byref(pulse),
                                             ctypes.c_void_p(d_rows), n_rows, ctypes.byref(opts),
                                             ctypes.c_void_p(d_j), ctypes.c_void_p(stream),
                                             ctypes.byref(st) if stats else None, err, len(err))
    return rc, st, err.value.decode()


def _status(lib, stream=None):
    err = ctypes.create_string_buffer(512)
    st = api.Stats()
    rc = lib.hhg_noalloc_status(ctypes.c_void_p(stream), ctypes.byref(st), err, len(err))
    return rc, st, err.value.decode()


def _case(case):
    if case == "piflux2d":
        s = 1 / math.sqrt(2)
        sys = api.system(api.SYS_PIFLUX2D, hopping=1.0, pol=(s, s))
        pulse = api.cosine_pulse(1.0, 2, 2048, window=(0.0, 6 * math.pi), energy_scale=20.0)
        grid = api.grid_tensor(32, 32, -math.pi, math.pi, -math.pi, math.pi)
    else:
        sys = api.system(api.SYS_HONEYCOMB, hopping=1.0, mass=0.1)
        pulse = api.cosine_pulse(1.2, 2, 2048, phase=0.7, window=(0.0, 6 * math.pi),
                                 energy_scale=12.5)
        grid = api.grid_rhombic(24, 24)
    return sys, pulse, grid


OPTIONS = {
    "restart": dict(),
    "carry": dict(proposer=api.PROPOSER_CARRY),
    "mixed_carry": dict(precision=api.PREC_MIXED, proposer=api.PROPOSER_CARRY, abs_tol=1e-8,
                        rel_tol=1e-6),
    "magnus4": dict(stepper=api.STEPPER_MAGNUS4, magnus_substeps=2),
}


@pytest.mark.parametrize("case,option", [("piflux2d", "restart"), ("honeycomb", "restart"),
                                         ("piflux2d", "carry"), ("honeycomb", "mixed_carry"),
                                         ("honeycomb", "magnus4")])
def test_noalloc_matches_regular_entry_point_twice(case, option):
    import torch
    torch.cuda.set_device(0)
    lib = api.load_library()
    eng = api.Engine(0)
    try:
        sys, pulse, grid = _case(case)
        kw = dict(abs_tol=1e-12, rel_tol=1e-8)
        kw.update(OPTIONS[option])
        opts = api.solver(**kw)
        j_ref, st_ref = eng.current_density(sys, pulse, grid, opts)
        rows = api.grid_rows(sys, grid)
        d_rows = torch.from_numpy(rows).cuda()
        d_j = torch.empty(pulse.n_measurements + 1, dtype=torch.float64, device="cuda")
        for call in range(2):
            d_j.fill_(float("nan"))
            torch.cuda.synchronize()
            rc, st, msg = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], opts,
                                   d_j.data_ptr())
            assert rc == api.OK, msg
            torch.cuda.synchronize()
            j = d_j.cpu().numpy()
            err = float(np.linalg.norm(j - j_ref) / np.linalg.norm(j_ref))
            assert err <= J_TOL, (call, err)
            assert st.attempted_steps == st_ref.attempted_steps
            assert st.failed_trajectories == 0
    finally:
        eng.close()


def test_noalloc_async_call_and_status_query():
    """stats == NULL: the call only enqueues; hhg_noalloc_status reports the
    outcome afterwards -- a clean run, then a step limit, then a clean run
    again (the counters are cleared on every call)."""
    import torch
    torch.cuda.set_device(0)
    lib = api.load_library()
    sys, pulse, grid = _case("piflux2d")
    rows = api.grid_rows(sys, grid)
    d_rows = torch.from_numpy(rows).cuda()
    d_j = torch.empty(pulse.n_measurements + 1, dtype=torch.float64, device="cuda")
    opts = api.solver(1e-12, 1e-8)
    rc, st_sync, msg = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], opts,
                                d_j.data_ptr())
    assert rc == api.OK, msg
    j_sync = d_j.cpu().numpy()
    for tight in (False, True, False):
        o = api.solver(1e-12, 1e-8)
        if tight:
            # the restart schedule needs 4 attempts per interval: 2 cannot land
            o.max_attempts_per_interval = 2
        d_j.fill_(float("nan"))
        torch.cuda.synchronize()
        rc, _, msg = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], o,
                              d_j.data_ptr(), stats=False)
        assert rc == api.OK, msg
        rc, st, msg = _status(lib)
        if tight:
            assert rc == api.STEP_LIMIT, (rc, msg)
            assert st.failed_trajectories > 0
        else:
            assert rc == api.OK, msg
            assert st.attempted_steps == st_sync.attempted_steps
            assert st.failed_trajectories == 0
            assert st.k_points == rows.shape[0]
            assert np.array_equal(d_j.cpu().numpy(), j_sync)


def test_noalloc_call_captured_into_a_cuda_graph():
    """After a first call outside any capture, an asynchronous call (stats ==
    NULL) can be captured into a CUDA graph: every replay reproduces the
    direct call's j bit for bit and leaves its outcome for hhg_noalloc_status.
    Under capture, a call with stats != NULL and the status query are refused
    with HHG_UNSUPPORTED without breaking the capture."""
    import torch
    torch.cuda.set_device(0)
    lib = api.load_library()
    sys, pulse, grid = _case("honeycomb")
    rows = api.grid_rows(sys, grid)
    d_rows = torch.from_numpy(rows).cuda()
    d_j = torch.empty(pulse.n_measurements + 1, dtype=torch.float64, device="cuda")
    opts = api.solver(1e-12, 1e-8, proposer=api.PROPOSER_CARRY)
    rc, st_sync, msg = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], opts,
                                d_j.data_ptr())
    assert rc == api.OK, msg
    j_sync = d_j.cpu().numpy()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        sp = stream.cuda_stream
        rc_cap, _, msg_cap = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], opts,
                                      d_j.data_ptr(), stats=False, stream=sp)
        rc_sync, _, msg_sync = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], opts,
                                        d_j.data_ptr(), stats=True, stream=sp)
        rc_stat, _, msg_stat = _status(lib, sp)
    assert rc_cap == api.OK, msg_cap
    assert rc_sync == api.UNSUPPORTED and "capture" in msg_sync, (rc_sync, msg_sync)
    assert rc_stat == api.UNSUPPORTED and "capture" in msg_stat, (rc_stat, msg_stat)
    for _ in range(2):
        d_j.fill_(float("nan"))
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            graph.replay()
        rc, st, msg = _status(lib, stream.cuda_stream)
        assert rc == api.OK, msg
        assert st.attempted_steps == st_sync.attempted_steps
        assert np.array_equal(d_j.cpu().numpy(), j_sync)
    del graph


def test_noalloc_rejects_oversized_problem_and_bad_options():
    import torch
    torch.cuda.set_device(0)
    lib = api.load_library()
    sys = api.system(api.SYS_DIRAC2D, velocity=1.0, mass=0.05)
    pulse = api.cosine_pulse(1.0, 8, 8192, energy_scale=10.0)
    rows = api.grid_rows(sys, api.grid_tensor(256, 256, -2, 2, -2, 2))
    # partial rows alone need 2048 x 8193 x 8 B > 64 MiB; the buffers are
    # full-sized all the same
    d_rows = torch.from_numpy(rows).cuda()
    d_j = torch.zeros(pulse.n_measurements + 1, dtype=torch.float64, device="cuda")
    rc, _, msg = _noalloc(lib, sys, pulse, d_rows.data_ptr(), rows.shape[0], api.solver(),
                          d_j.data_ptr())
    assert rc == api.BAD_CONFIG
    assert "scratch" in msg, msg
    # the regular path's Magnus-4 substep bound applies here too
    small = d_rows[:64]
    rc, _, msg = _noalloc(lib, sys, pulse, small.data_ptr(), 64,
                          api.solver(stepper=api.STEPPER_MAGNUS4, magnus_substeps=5000),
                          d_j.data_ptr())
    assert rc == api.BAD_CONFIG, msg
