"""Time-local truncation (PHI's TimeLocal) in the oracle, pinned to the
reference build (CPU), and the library's scope checks for it.

tests/golden/ref_timelocal.json holds, per case, rho_0 printed with %.17g by
the reference build, the whole final state from the restart file the same
run wrote (6 significant digits, small hierarchies) and, for RKF45, the sums
over k of the stored Q_{m,k} that file ends with.  PHI advances
Q_{m,k} <- d_k U^+ (Q_{m,k} + h c_{m,k} |m><m|) U with U = I - i H h
(hierarchy.cc:229-341) along the stage times (with diag(V_m) or V_m in place
of |m><m| for diagonal and full couplings), and the deepest tier adds
-sum_m [V_m, Q_m rho - rho Q_m^+] in place of its next terms
(hierarchy_updater.cc:28-44, :93-104, :171-190).
"""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Batch, Hierarchy

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_timelocal.json")))["cases"]


def build(case):
    b = case["builder"]
    if b.startswith("config:"):
        p = getattr(configs, b.split(":", 1)[1])(**case["kwargs"])
    else:
        p = getattr(cases, b)(**case["kwargs"])
    p.use_time_local_truncation = True
    p.filter_tolerance = case["filter_tolerance"]
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def run_oracle(o, case):
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    return s


def to_complex(v):
    return np.array([complex(a, b) for a, b in v])


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_oracle_rho0_matches_reference(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case)
    ref = to_complex(case["rho0_colmajor"]).reshape(p.num_states, p.num_states).T
    assert np.abs(o.rho0(s) - ref).max() <= 1e-13


@pytest.mark.parametrize("case", [c for c in FIX if "state_6_digits" in c],
                         ids=[c["id"] for c in FIX if "state_6_digits" in c])
def test_oracle_state_matches_reference_restart_file(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case).view(np.complex128)
    ref = to_complex(case["state_6_digits"])
    assert ref.size == s.size
    np.testing.assert_allclose(s, ref, rtol=6e-6, atol=1e-300)


@pytest.mark.parametrize("case", [c for c in FIX if "q_sums_6_digits" in c],
                         ids=[c["id"] for c in FIX if "q_sums_6_digits" in c])
def test_oracle_time_local_matrices_match_reference(case):
    """After an accepted RKF45 step the stored Q_{m,k} equal the current ones;
    their sums over k are the Q_m the oracle reports (6 digits as printed,
    summed here, so the bound is on the scale of the terms)."""
    p = build(case)
    o = O.Oracle(p)
    run_oracle(o, case)
    got = o.time_local().reshape(-1)
    ref = to_complex(case["q_sums_6_digits"])
    assert np.abs(got).max() > 0
    assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_time_local_changes_the_result(case):
    p = build(case)
    o = O.Oracle(p)
    run_oracle(o, case)
    p.use_time_local_truncation = False
    o2 = O.Oracle(p)
    s2 = run_oracle(o2, case)
    ref = to_complex(case["rho0_colmajor"]).reshape(p.num_states, p.num_states).T
    assert np.abs(o2.rho0(s2) - ref).max() > 1e-7


def test_chunked_rk4_keeps_time_local_state():
    """Two RK4 calls with continue_run equal one call: Q carries over."""
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=2)
    p.use_time_local_truncation = True
    o = O.Oracle(p)
    one, n1, *_ = o.rk4(o.initial_state(), 0.001, 0.05)
    q1 = o.time_local()
    a, na, *_ = o.rk4(o.initial_state(), 0.001, 0.013)
    b, nb, *_ = o.rk4(a, 0.001, 0.05, start_time=0.013, continue_run=True)
    assert n1 == na + nb
    assert np.abs(o.time_local() - q1).max() <= 1e-14 * np.abs(q1).max()
    assert np.abs(b - one).max() <= 1e-14 * np.abs(one).max()


def test_time_local_outside_identity_map_is_rejected():
    """Independent baths on another site map: PHI adds c at (b, b) whatever
    site bath b couples to (hierarchy.cc:298-300), so the library refuses the
    input instead of guessing.  (Diagonal and full couplings are built.)"""
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=1)
    p.bath_sites = np.array([0, 2, 1], np.int32)
    p.use_time_local_truncation = True
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy(p)


def test_batch_rejects_time_local():
    p = configs.frenkel7(depth=2)
    p.use_time_local_truncation = True
    with pytest.raises(capi.PhiError, match="time-local"):
        Batch([p])
