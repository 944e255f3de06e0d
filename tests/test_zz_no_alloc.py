"""phi_gpu_rk4_step_noalloc: the RK4 step for callers that cannot allocate
device memory when they step (stream capture, host-owned memory pools,
latency-bound loops).  Called through the C ABI on caller-owned device
buffers, twice in a row, and checked against the allocating entry point
phi_gpu_rk4 with the FP64 tolerance of the other parity tests.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest
import torch

import cases
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
DT = 0.001


def _noalloc_step(h, d_in, d_out):
    stream = torch.cuda.current_stream()
    rc = h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(d_in.data_ptr()),
                                        ctypes.c_void_p(d_out.data_ptr()), DT,
                                        ctypes.c_void_p(stream.cuda_stream))
    capi.check(rc, h.ctx)


@pytest.mark.parametrize("make", [lambda: configs.frenkel7(depth=3), configs.spin_boson,
                                  lambda: cases.random_problem("full", n=3, matsubara=2, truncation=4)],
                         ids=["frenkel7_L3", "spin_boson", "full_n3"])
def test_noalloc_step_matches_allocating_rk4(make):
    p = make()
    with Hierarchy(p) as h:
        s0 = cases.random_hermitian_state(h.num_nodes, p.num_states, seed=5)
        # Allocating entry point: one and two steps from s0.
        h.set_state(s0)
        h.time = 0.0
        h.rk4(DT, DT)
        ref1 = h.get_state()
        h.rk4(DT, 2 * DT)
        ref2 = h.get_state()
        # No-alloc entry point, two calls in a row on caller-owned buffers.
        a = torch.tensor(s0, dtype=torch.float64, device="cuda")
        b = torch.empty_like(a)
        c = torch.empty_like(a)
        _noalloc_step(h, a, b)
        _noalloc_step(h, b, c)
        torch.cuda.synchronize()
        got1, got2 = b.cpu().numpy(), c.cpu().numpy()
        assert np.array_equal(a.cpu().numpy(), s0)  # input untouched
    scale = max(np.abs(ref2).max(), 1e-300)
    assert np.abs(got1 - ref1).max() <= FP64_TOL * scale
    assert np.abs(got2 - ref2).max() <= FP64_TOL * scale


def _time_local():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=2)
    p.use_time_local_truncation = True
    return p


def _filtered():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=5, seed=2)
    p.filter_tolerance = 1e-3
    return p


@pytest.mark.parametrize("make", [_time_local, _filtered], ids=["time_local_n3", "filtered_n3"])
def test_noalloc_steps_carry_context_matrices_and_flags(make):
    """A time-local or filtered context: each call advances the context's
    truncation matrices and filter flags like one phi_gpu_rk4 step, so two
    calls from set_state(s0) equal two allocating steps from s0."""
    p = make()
    with Hierarchy(p) as h:
        s0 = h.get_state()
        s0 = s0 + 1e-4 * cases.random_hermitian_state(h.num_nodes, p.num_states, seed=7)
        h.set_state(s0)
        h.time = 0.0
        h.rk4(DT, 2 * DT)
        ref, act_ref, q_ref = h.get_state(), h.active(), h.time_local()
        h.set_state(s0)  # matrices and flags back to their start
        h.time = 0.0
        a = torch.tensor(s0, dtype=torch.float64, device="cuda")
        b, c = torch.empty_like(a), torch.empty_like(a)
        _noalloc_step(h, a, b)
        _noalloc_step(h, b, c)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert h.lib.phi_gpu_check_device_flag(h.ctx, stream) == capi.PHI_OK
        torch.cuda.synchronize()
        got, act, q = c.cpu().numpy(), h.active(), h.time_local()
    if p.filter_tolerance > 0:
        assert np.array_equal(act, act_ref) and 0 < int(act.sum()) < len(act)
    if p.use_time_local_truncation:
        assert np.abs(q - q_ref).max() <= 1e-14 * np.abs(q_ref).max()
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()


def test_noalloc_rejects_states_beyond_its_scratch():
    p = configs.frenkel7()  # 38,760 nodes: 30.4 MB of state > 8 MiB
    with Hierarchy(p) as h:
        a = torch.zeros(16, dtype=torch.float64, device="cuda")
        b = torch.zeros(16, dtype=torch.float64, device="cuda")
        rc = h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(a.data_ptr()),
                                            ctypes.c_void_p(b.data_ptr()), DT, None)
        assert rc == capi.PHI_E_INVALID
        assert "exceeds" in capi.last_error(h.ctx)
