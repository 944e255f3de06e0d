"""Mixed precision (PHI_PREC_MIXED): complex64 stage inputs and derivatives,
FP32 Liouvillian arithmetic, FP64 state / combines / error norm / control.

Tolerances stated here:
* one apply: max-abs error <= 2e-6 of the output scale (FP32 arithmetic on
  complex64 inputs; the FP64 oracle is the reference);
* propagated rho_0: max-abs error <= 1e-6 against the FP64 GPU path (the
  accuracy target of the mixed mode).
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

APPLY_RTOL = 2e-6
RHO0_TOL = 1e-6


@pytest.mark.parametrize("make", [lambda: configs.frenkel7(depth=3), lambda: configs.chain4(depth=3),
                                  lambda: configs.ring24(depth=2),
                                  lambda: cases.random_problem("independent", n=5, matsubara=3, truncation=4,
                                                               complex_h=True)],
                         ids=["frenkel7_L3", "chain4_L3", "ring24_L2", "indep_n5_K2"])
def test_mixed_apply_close_to_oracle(make):
    p = make()
    o = O.Oracle(p)
    s = cases.random_hermitian_state(o.M, p.num_states, seed=3)
    ref = o.apply(s)
    with Hierarchy(p, precision=capi.PHI_PREC_MIXED) as h:
        got = h.apply(s)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= APPLY_RTOL, err


@pytest.mark.parametrize("make,t_end", [(lambda: configs.frenkel7(depth=4), 0.3),
                                        (lambda: configs.chain4(depth=4), 0.3),
                                        (lambda: configs.ring24(depth=2), 0.1)],
                         ids=["frenkel7_L4", "chain4_L4", "ring24_L2"])
def test_mixed_rkf45_rho0_within_1e6_of_fp64(make, t_end):
    p = make()
    p.fix_incompatible_combinations("rkf45")
    out = {}
    for prec in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        with Hierarchy(p, precision=prec) as h:
            st = h.rkf45(0.001, t_end, 1e-6, 1e-6)
            out[prec] = (h.rho0(), st)
    s64, s32 = out[capi.PHI_PREC_FP64][1], out[capi.PHI_PREC_MIXED][1]
    # PHI's step control clamps the last step on the step size before its
    # growth (hierarchy_integrator.cc:2434-2437), so a run may end up to one
    # grown step past t_end; the two arithmetics can take different
    # accept/reject decisions when an error estimate sits within rounding of
    # tol.
    for st in (s64, s32):
        assert t_end <= st["final_time"] < t_end + 0.02
    if (s64["steps"], s64["accepted"]) == (s32["steps"], s32["accepted"]) and \
            s64["final_time"] == s32["final_time"]:
        err = np.abs(out[capi.PHI_PREC_MIXED][0] - out[capi.PHI_PREC_FP64][0]).max()
        assert err <= RHO0_TOL, (err, s64, s32)
    # Each run against a fine fixed-step FP64 RK4 reference at its own final
    # time: mixed must be as accurate as FP64 at the same tolerance, to 1e-6.
    errs = {}
    for prec, (rho, st) in out.items():
        n = int(round(st["final_time"] / 1e-4))
        dt = st["final_time"] / n
        with Hierarchy(p) as h:
            h.rk4(dt, (n - 0.5) * dt)
            errs[prec] = np.abs(rho - h.rho0()).max()
    assert errs[capi.PHI_PREC_MIXED] <= errs[capi.PHI_PREC_FP64] + RHO0_TOL, (errs, s64, s32)


def test_mixed_rk4_rho0_within_1e6_of_fp64():
    p = configs.frenkel7(depth=4)
    res = {}
    for prec in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        with Hierarchy(p, precision=prec) as h:
            steps, times, rows = h.rk4(0.001, 0.2, 0.01, capacity=32)
            res[prec] = (h.rho0(), rows, steps)
    assert res[0][2] == res[1][2] == 200
    assert np.abs(res[1][0] - res[0][0]).max() <= RHO0_TOL
    assert np.abs(res[1][1] - res[0][1]).max() <= RHO0_TOL


def test_mixed_state_stays_hermitian_and_trace_one():
    p = configs.chain4(depth=4)
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p, precision=capi.PHI_PREC_MIXED) as h:
        h.rkf45(0.001, 0.2, 1e-6, 1e-6)
        rho = h.rho0()
    assert np.allclose(rho, rho.conj().T, atol=1e-12)
    assert abs(np.trace(rho).real - 1.0) < 1e-6


def test_mixed_rejected_where_not_built():
    p = configs.spin_boson()  # diagonal coupling: FP64 only
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p, precision=capi.PHI_PREC_MIXED)
    assert e.value.code == capi.PHI_E_INVALID
