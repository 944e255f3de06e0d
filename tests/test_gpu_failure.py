"""Failure paths of the device integrators, none of which faults or hangs the
GPU: an RKF45 run that hits its step limit (PHI_E_STEP_COLLAPSE), a
Hamiltonian whose scale overflows the stage values (PHI_E_NUMERIC), and a
bounded device wait that gives up (PHI_E_TIMEOUT) -- made to give up at
once through the test hook phi_gpu_debug_set_wait_limit, after which the
kernel drains its own bulk copies with the built-in limit and returns, and
the context stays usable."""
import ctypes

import numpy as np
import pytest

import cases
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu


def test_rkf45_step_limit_is_reported():
    p = configs.frenkel7(depth=2)
    with Hierarchy(p) as h:
        with pytest.raises(capi.PhiError) as e:
            h.rkf45(0.001, 1.0, 1e-6, 1e-6, max_steps=3)
        assert e.value.code == capi.PHI_E_STEP_COLLAPSE
        assert "step limit" in capi.last_error(h.ctx)
        assert 0 < h.time < 1.0
        # The context continues from where the limit stopped it.
        st = h.rkf45(0.001, 0.02, 1e-6, 1e-6)
        assert st["final_time"] == pytest.approx(0.02)


def test_overflowing_hamiltonian_is_reported_as_numeric():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=0)
    p.time_indepenent_hamiltonian = p.time_indepenent_hamiltonian * 1e300
    with Hierarchy(p) as h:
        with pytest.raises(capi.PhiError) as e:
            h.rkf45(0.001, 0.01, 1e-6, 1e-6)
        assert e.value.code == capi.PHI_E_NUMERIC
        assert "non-finite" in capi.last_error(h.ctx)


def test_nan_hamiltonian_is_rejected_at_create():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=0)
    H = p.time_indepenent_hamiltonian.copy()
    H[0, 1] = np.nan
    p.time_indepenent_hamiltonian = H
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p)
    assert e.value.code == capi.PHI_E_INVALID


@pytest.mark.parametrize("precision", [capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED], ids=["fp64", "mixed"])
def test_device_wait_that_gives_up_is_reported_and_context_recovers(precision):
    p = configs.frenkel7(depth=3)  # tiled stage kernel (7 sites, K+1 = 2)
    with Hierarchy(p, precision=precision) as ref:
        s0 = ref.get_state()
        ref.rk4(0.001, 0.004)
        want = ref.get_state()
    with Hierarchy(p, precision=precision) as h:
        assert h.lib.phi_gpu_debug_set_wait_limit(h.ctx, -1) == capi.PHI_OK
        with pytest.raises(capi.PhiError) as e:
            h.rk4(0.001, 0.004)
        assert e.value.code == capi.PHI_E_TIMEOUT
        assert "gave up" in capi.last_error(h.ctx)
        # The flag was cleared by the report; the built-in limit is back.
        assert h.lib.phi_gpu_debug_set_wait_limit(h.ctx, 0) == capi.PHI_OK
        assert h.lib.phi_gpu_check_device_flag(h.ctx, None) == capi.PHI_OK
        h.set_state(s0)
        h.time = 0.0
        h.rk4(0.001, 0.004)
        got = h.get_state()
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()


def test_noalloc_step_timeout_is_reported_by_the_flag_query():
    import torch
    p = configs.frenkel7(depth=3)
    with Hierarchy(p) as h:
        a = torch.tensor(h.get_state(), dtype=torch.float64, device="cuda")
        b = torch.empty_like(a)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert h.lib.phi_gpu_debug_set_wait_limit(h.ctx, -1) == capi.PHI_OK
        rc = h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(a.data_ptr()),
                                            ctypes.c_void_p(b.data_ptr()), 0.001, stream)
        assert rc == capi.PHI_OK  # the call does not synchronise
        assert h.lib.phi_gpu_check_device_flag(h.ctx, stream) == capi.PHI_E_TIMEOUT
        assert h.lib.phi_gpu_debug_set_wait_limit(h.ctx, 0) == capi.PHI_OK
        rc = h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(a.data_ptr()),
                                            ctypes.c_void_p(b.data_ptr()), 0.001, stream)
        assert rc == capi.PHI_OK
        assert h.lib.phi_gpu_check_device_flag(h.ctx, stream) == capi.PHI_OK
