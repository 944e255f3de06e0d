"""Adaptive hierarchy filtering (PHI's FilterTolerance) on the GPU: the tiled
kernel (identity site map, K+1 <= 3) and the generic kernel (K+1 > 3), RK4
and RKF45, against the oracle (whole state and the active flags) and against
the reference build's rho_0 (tests/golden/ref_filter.json).

A node's flag follows its largest |element| after every RK4 step and every
accepted RKF45 step (hierarchy_integrator.cc:2827-2850, :2359-2384); an
inactive node keeps its own terms but feeds no neighbour
(hierarchy_updater.cc:256-303).
"""
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
FIX = json.load(open(os.path.join(HERE, "golden", "ref_filter.json")))["cases"]
FP64_TOL = 1e-10    # max-abs error relative to max |state|
RHO0_TOL = 1e-6     # mixed precision against FP64


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


def run_gpu(h, method, dt, t_end):
    if method == "rk4":
        h.rk4(dt, t_end)
    else:
        h.rkf45(dt, t_end, 1e-6, 1e-6)


def run_oracle(o, method, dt, t_end):
    s0 = o.initial_state()
    if method == "rk4":
        s, *_ = o.rk4(s0, dt, t_end)
    else:
        s, _ = o.rkf45(s0, dt, t_end, 1e-6, 1e-6)
    return s


# Fixture cases run on the tiled kernel; the generic kernel serves K+1 = 4.
GENERIC = [
    {"id": "generic_n3_k4_t4/rk4/1e-3", "builder": "random_problem",
     "kwargs": dict(kind="independent", n=3, matsubara=4, truncation=4, seed=4),
     "method": "rk4", "timestep": 0.001, "t_end": 0.05, "filter_tolerance": 1e-3},
    {"id": "generic_n3_k4_t4/rkf45/1e-3", "builder": "random_problem",
     "kwargs": dict(kind="independent", n=3, matsubara=4, truncation=4, seed=4),
     "method": "rkf45", "timestep": 0.001, "t_end": 0.05, "filter_tolerance": 1e-3},
]
ALL = FIX + GENERIC


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_rho0_matches_reference(case):
    p = build(case)
    with Hierarchy(p) as h:
        run_gpu(h, case["method"], case["timestep"], case["t_end"])
        rho = h.rho0()
    ref = np.array([complex(a, b) for a, b in case["rho0_colmajor"]]).reshape(p.num_states, p.num_states).T
    assert np.abs(rho - ref).max() <= 1e-11


@pytest.mark.parametrize("case", ALL, ids=[c["id"] for c in ALL])
def test_state_and_flags_match_oracle(case):
    p = build(case)
    o = O.Oracle(p)
    ref = run_oracle(o, case["method"], case["timestep"], case["t_end"])
    with Hierarchy(p) as h:
        run_gpu(h, case["method"], case["timestep"], case["t_end"])
        got = h.get_state()
        act = h.active()
    assert np.array_equal(act, o.active())
    assert (~act).sum() > 0
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()


def test_chunked_rk4_carries_flags():
    """13 steps (no graph, odd: the flags end in the second buffer) then 37
    (two 16-step graphs and a tail) equal one 50-step call, state and flags."""
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        one, act1 = h.get_state(), h.active()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.013)
        h.rk4(0.001, 0.05)
        two, act2 = h.get_state(), h.active()
    assert np.array_equal(act1, act2)
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_chunked_rkf45_carries_flags():
    """rkf45_advance in chunks continues the flags of the accepted state."""
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p) as h:
        st = h.rkf45(0.001, 0.05, 1e-6, 1e-6)
        one, act1 = h.get_state(), h.active()
    with Hierarchy(p) as h:
        a = h.rkf45_advance(0.001, 0.05, 1e-6, 1e-6, 7)
        done = a["steps"]
        while h.time < 0.05:
            b = h.rkf45_advance(0.0, 0.05, 1e-6, 1e-6, 5)
            done += b["steps"]
        two, act2 = h.get_state(), h.active()
    assert done == st["steps"]
    assert np.array_equal(act1, act2)
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_set_state_and_reset_restore_all_active():
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    with Hierarchy(p) as h:
        s0 = h.get_state()
        h.rk4(0.001, 0.02)
        assert not h.active().all()
        h.set_state(s0)
        assert h.active().all()
        h.time = 0.0
        h.rk4(0.001, 0.02)
        assert not h.active().all()
        capi.check(h.lib.phi_gpu_reset(h.ctx, 0.0), h.ctx)
        assert h.active().all()


def test_filtering_off_is_unchanged():
    """filter_tolerance 0 and a diagonal bath with a tolerance (dropped as
    FixIncompatibleCombinations does) give the unfiltered state exactly."""
    for make in (lambda: configs.frenkel7(depth=3),
                 lambda: cases.random_problem("diagonal", n=3, matsubara=2, truncation=4, seed=1)):
        p = make()
        with Hierarchy(p) as h:
            h.rk4(0.001, 0.02)
            a = h.get_state()
        p.filter_tolerance = 1e-2 if p.bath_kind != capi.PHI_BATH_INDEPENDENT else 0.0
        with Hierarchy(p) as h:
            h.rk4(0.001, 0.02)
            b = h.get_state()
            assert h.active().all()
        assert np.array_equal(a, b)


def test_steady_state_ignores_flags_of_a_fresh_context():
    """BiCGSTAB never updates the flags (PHI updates them only in RK4 /
    RKF45), so on a fresh context the filtered and unfiltered solves agree."""
    p = configs.frenkel7(depth=2)
    p.fix_incompatible_combinations("bicgstab")
    with Hierarchy(p) as h:
        h.steady_state(tol=1e-12, ell=2)
        a = h.get_state()
    p.filter_tolerance = 1e-3
    with Hierarchy(p) as h:
        h.steady_state(tol=1e-12, ell=2)
        b = h.get_state()
    assert np.abs(a - b).max() <= 1e-14


def test_mixed_precision_filtered_rho0():
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    out = {}
    for prec in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        with Hierarchy(p, precision=prec) as h:
            h.rk4(0.001, 0.1)
            out[prec] = (h.rho0(), h.active())
    assert np.abs(out[capi.PHI_PREC_MIXED][0] - out[capi.PHI_PREC_FP64][0]).max() <= RHO0_TOL
    assert (out[capi.PHI_PREC_MIXED][1] != out[capi.PHI_PREC_FP64][1]).mean() < 0.01


def test_parameter_file_filter_tolerance(tmp_path):
    """FilterTolerance read from a PHI parameter file reaches the kernels."""
    p = configs.frenkel7(depth=3)
    p.filter_tolerance = 1e-3
    path = tmp_path / "params.txt"
    path.write_text(O.param_file_text(p, timestep=0.001, t_end=0.05))
    with Hierarchy.from_file(str(path), "rk4") as h:
        h.rk4(0.001, 0.05)
        a, act = h.get_state(), h.active()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        b = h.get_state()
    assert not act.all()
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
