"""Annealing Hamiltonians on the GPU: H = f_x(t/T) H_X + f_z(t/T) H_Z set on
the device before every RK4 / RKF45 stage (UpdateTimeDependentHamiltonian,
hierarchy_integrator.cc:1618-1673), against the reference build's rho_0
(tests/golden/ref_anneal.json) and the oracle (whole state and final H), on
the tiled kernel (real and complex H_X), the generic kernel (diagonal and
full baths) and with time-local truncation.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_anneal.json")))["cases"]
FP64_TOL = 1e-10    # max-abs error relative to the largest element
RHO0_TOL = 1e-6     # mixed precision against FP64


def build(case):
    b = case["builder"]
    if b.startswith("config:"):
        p = getattr(configs, b.split(":", 1)[1])(**case["kwargs"])
    else:
        p = getattr(cases, b)(**case["kwargs"])
    p = cases.annealed(p, case["t_end"], **case["anneal"])
    p.use_time_local_truncation = case["time_local"]
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def run_gpu(h, case):
    if case["method"] == "rk4":
        h.rk4(case["timestep"], case["t_end"])
    else:
        h.rkf45(case["timestep"], case["t_end"], 1e-6, 1e-6)


def run_oracle(o, case):
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    return s


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_rho0_matches_reference(case):
    p = build(case)
    with Hierarchy(p) as h:
        run_gpu(h, case)
        rho = h.rho0()
    ref = np.array([complex(a, b) for a, b in case["rho0_colmajor"]]).reshape(p.num_states, p.num_states).T
    assert np.abs(rho - ref).max() <= FP64_TOL * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_state_and_hamiltonian_match_oracle(case):
    p = build(case)
    o = O.Oracle(p)
    ref = run_oracle(o, case)
    with Hierarchy(p) as h:
        run_gpu(h, case)
        got, H = h.get_state(), h.hamiltonian()
    H_ref = o.hamiltonian()
    assert np.abs(H - H_ref).max() <= 1e-14 * np.abs(H_ref).max()
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()


def _problem(**kw):
    return cases.annealed(cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=2), 0.05,
                          seed=1, **kw)


def test_mixed_precision_annealed_rho0():
    p = cases.annealed(configs.frenkel7(depth=2), 0.1, seed=1)
    p.fix_incompatible_combinations("rkf45")
    out = {}
    for prec in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        with Hierarchy(p, precision=prec) as h:
            h.rkf45(0.001, 0.1, 1e-6, 1e-6)
            out[prec] = h.rho0()
    assert np.abs(out[capi.PHI_PREC_MIXED] - out[capi.PHI_PREC_FP64]).max() <= RHO0_TOL


def test_chunked_rk4_follows_the_ramp():
    """13 then 37 steps equal one 50-step call: the step time and the gate
    state carry over between calls."""
    p = _problem()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        one, H1 = h.get_state(), h.hamiltonian()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.013)
        h.rk4(0.001, 0.05)
        two, H2 = h.get_state(), h.hamiltonian()
    assert np.abs(H1 - H2).max() == 0
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_chunked_rkf45_follows_the_ramp():
    p = _problem()
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p) as h:
        st = h.rkf45(0.001, 0.05, 1e-6, 1e-6)
        one = h.get_state()
    with Hierarchy(p) as h:
        done = h.rkf45_advance(0.001, 0.05, 1e-6, 1e-6, 7)["steps"]
        while h.time < 0.05:
            done += h.rkf45_advance(0.0, 0.05, 1e-6, 1e-6, 5)["steps"]
        two = h.get_state()
    assert done == st["steps"]
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_parameter_file_annealing(tmp_path):
    p = _problem()
    path = tmp_path / "params.txt"
    path.write_text(O.param_file_text(p, timestep=0.001, t_end=0.05))
    with Hierarchy.from_file(str(path), "rk4") as h:
        h.rk4(0.001, 0.05)
        a = h.get_state()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        b = h.get_state()
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


def test_reset_and_refusals():
    import torch
    p = _problem()
    with Hierarchy(p) as h:
        assert np.abs(h.hamiltonian()).max() == 0  # zero until the first stage
        s0 = h.get_state()
        h.rk4(0.001, 0.01)
        assert np.abs(h.hamiltonian()).max() > 0
        h.set_state(s0)
        assert np.abs(h.hamiltonian()).max() == 0
        with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
            h.steady_state(tol=1e-10)
        a = torch.tensor(s0, dtype=torch.float64, device="cuda")
        b = torch.empty_like(a)
        rc = h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                            0.001, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == capi.PHI_E_INVALID
