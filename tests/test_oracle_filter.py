"""Adaptive hierarchy filtering (PHI's FilterTolerance) in the oracle, pinned
to the reference build (CPU).

tests/golden/ref_filter.json holds, per case, rho_0 printed with %.17g by the
reference build and, for small hierarchies, the whole final state from the
restart file the same run wrote (6 significant digits).  PHI's effective
filtering (hierarchy_updater.h:36-52 calls the non-virtual Get, so only the
virtual DoNext / DoPrevious overrides of IndependentBathAdaptiveTruncation,
hierarchy_updater.cc:256-303, take effect) keeps every node's own terms and
drops the terms fed by inactive neighbours; flags follow every RK4 step and
every accepted RKF45 step (hierarchy_integrator.cc:2827-2850, :2359-2384).
"""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import configs

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_filter.json")))["cases"]


def build(case):
    b = case["builder"]
    if b.startswith("config:"):
        p = getattr(configs, b.split(":", 1)[1])(**case["kwargs"])
    else:
        p = getattr(cases, b)(**case["kwargs"])
    p.filter_tolerance = case["filter_tolerance"]
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def run_oracle(o, case, filtered=True):
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    return s


def colmajor_to_matrix(v, n):
    z = np.array([complex(a, b) for a, b in v])
    return z.reshape(n, n).T


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_oracle_rho0_matches_reference(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case)
    ref = colmajor_to_matrix(case["rho0_colmajor"], p.num_states)
    assert np.abs(o.rho0(s) - ref).max() <= 1e-13


@pytest.mark.parametrize("case", [c for c in FIX if "state_6_digits" in c],
                         ids=[c["id"] for c in FIX if "state_6_digits" in c])
def test_oracle_state_matches_reference_restart_file(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case).view(np.complex128)
    ref = np.array([complex(a, b) for a, b in case["state_6_digits"]])
    assert ref.size == s.size == o.M * p.num_states ** 2
    # 6 significant digits as PHI prints them
    np.testing.assert_allclose(s, ref, rtol=6e-6, atol=1e-300)


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_filtering_changes_the_result(case):
    """Each fixture case is one where filtering matters: the unfiltered run
    differs from the reference's filtered rho_0 by far more than FP64 noise,
    and some nodes end inactive."""
    p = build(case)
    o = O.Oracle(p)
    run_oracle(o, case)
    assert (~o.active()).sum() > 0
    p.filter_tolerance = 0.0
    o2 = O.Oracle(p)
    s2 = run_oracle(o2, case)
    ref = colmajor_to_matrix(case["rho0_colmajor"], p.num_states)
    assert np.abs(o2.rho0(s2) - ref).max() > 1e-7
    assert o2.active().all()


def test_filter_is_ignored_for_diagonal_and_full_baths():
    """FixIncompatibleCombinations drops FilterTolerance for correlated and
    full bath couplings (phi_parameters.cc:847-851)."""
    for kind in ("diagonal", "full"):
        p = cases.random_problem(kind, n=3, matsubara=2, truncation=4, seed=1)
        o = O.Oracle(p)
        a, *_ = o.rk4(o.initial_state(), 0.001, 0.02)
        p.filter_tolerance = 1e-2
        o2 = O.Oracle(p)
        b, *_ = o2.rk4(o2.initial_state(), 0.001, 0.02)
        assert np.array_equal(a, b)


def test_flags_reactivate():
    """Hysteresis both ways: a deep node that drops below the tolerance in the
    first step is fed by its active neighbours and comes back above it."""
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=2)
    p.filter_tolerance = 1e-3
    o = O.Oracle(p)
    s, *_ = o.rk4(o.initial_state(), 0.001, 0.001)
    first = o.active()
    s, *_ = o.rk4(s, 0.001, 0.05, start_time=0.001, continue_run=True)
    last = o.active()
    assert (~first).sum() > 0
    assert (last & ~first).sum() > 0, "no node came back"


def test_chunked_rk4_keeps_flags():
    """Two calls with keep_filter equal one call (the flags carry over)."""
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    o = O.Oracle(p)
    one, n1, *_ = o.rk4(o.initial_state(), 0.001, 0.05)
    a, na, *_ = o.rk4(o.initial_state(), 0.001, 0.013)
    b, nb, *_ = o.rk4(a, 0.001, 0.05, start_time=0.013, continue_run=True)
    assert n1 == na + nb
    assert np.abs(b - one).max() <= 1e-14


def test_batch_rejects_filtering():
    """Filtering runs on single hierarchies; a batch refuses it before any
    device work."""
    from phi_b200 import capi
    from phi_b200.heom import Batch
    p = configs.frenkel7(depth=2)
    p.filter_tolerance = 1e-3
    with pytest.raises(capi.PhiError, match="filtering"):
        Batch([p])


def test_negative_filter_tolerance_is_rejected():
    from phi_b200 import capi
    from phi_b200.heom import Hierarchy
    p = configs.frenkel7(depth=2)
    p.filter_tolerance = -1.0
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy(p)
