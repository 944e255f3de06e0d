"""BiCGSTAB(ell) steady state on the GPU (PrepForSteadyState followed by
BicgstabLSteadyState / BicgstabSteadyState, hierarchy_integrator.cc:1471-1613,
:3112-3441, :3495-3783).

The reference's steady-state runs give no output to pin against (its test
suite has no steady-state case), so parity is with the oracle's dense solve of
the same eliminated system, within the solver tolerance times the condition
number of that system, and with long-time propagation.
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-12  # relative residual asked of the device solver

SMALL = [
    ("indep_n3_K2_L4", lambda: cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)),
    ("indep_n2_K1_L6", lambda: cases.random_problem("independent", n=2, matsubara=1, truncation=6, seed=5)),
    ("indep_n4_K1_L3_complexH", lambda: cases.random_problem("independent", n=4, matsubara=1, truncation=3,
                                                             seed=6, complex_h=True)),
    ("diag_n3_b2_K1_L4", lambda: cases.random_problem("diagonal", n=3, matsubara=1, truncation=4, baths=2, seed=3)),
    ("full_n2_b2_K2_L4", lambda: cases.random_problem("full", n=2, matsubara=2, truncation=4, baths=2, seed=3)),
    ("frenkel7_L2", lambda: configs.frenkel7(depth=2)),
]


@pytest.mark.parametrize("ell", [1, 2, 4])
@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_steady_state_matches_dense_solve(name, make, ell):
    p = make()
    o = O.Oracle(p)
    A = o.liouvillian_matrix()
    ref = o.steady_state(A)
    cond = np.linalg.cond(A[1:, 1:])
    with Hierarchy(p) as h:
        st = h.steady_state(tol=SOLVE_TOL, ell=ell, max_steps=20000, check=False)
        got = h.get_state()
    if ell == 1 and not st["converged"]:
        # BiCGSTAB (ell = 1) may break down on oscillatory spectra, as it does
        # in the reference; BiCGSTAB(ell >= 2) must not.
        assert st["status"] == capi.PHI_E_NO_CONVERGENCE
        return
    assert st["converged"] and st["status"] == capi.PHI_OK
    assert st["residual"] <= SOLVE_TOL
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max()
    assert err <= max(1e-10, 10 * SOLVE_TOL * cond) * scale, (err, cond, st)
    rho = o.rho0(got)
    assert abs(np.trace(rho) - 1) <= 1e-14
    assert np.allclose(rho, rho.conj().T, rtol=0, atol=1e-15)


@pytest.mark.parametrize("make", [lambda: configs.frenkel7(depth=5), lambda: configs.chain4(depth=5)],
                         ids=["frenkel7_L5", "chain4_L5"])
def test_steady_state_residual_at_size(make):
    """Size-independent check: L(rho_ss) ~ 0 through the device apply, trace 1,
    Hermitian, populations in [0, 1]."""
    p = make()
    with Hierarchy(p) as h:
        e00 = np.zeros(h.state_len)
        e00[0] = 1.0
        bnorm = np.linalg.norm(h.apply(e00)[2:])
        st = h.steady_state(tol=1e-12, max_steps=20000)
        x = h.get_state()
        r = h.apply(x)
        rho = h.rho0()
    assert st["converged"], st
    # The solution is divided by tr rho_0, so the residual scales by 1/x00.
    assert np.linalg.norm(r) <= 1e-9 * bnorm, (np.linalg.norm(r), bnorm)
    assert abs(np.trace(rho) - 1) <= 1e-13
    assert np.allclose(rho, rho.conj().T, rtol=0, atol=1e-14)
    pop = np.diag(rho).real
    assert np.all(pop > 0) and np.all(pop < 1)


def test_long_time_propagation_reaches_steady_state():
    """RK4 for 10 ps (slowest relaxation rate 2.8/ps) lands on the solver's state."""
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)
    with Hierarchy(p) as h:
        h.rk4(0.001, 10.0)
        rho_t = h.rho0()
        h.steady_state(tol=SOLVE_TOL)
        rho_ss = h.rho0()
    assert np.abs(rho_t - rho_ss).max() <= 1e-9


def test_c4_family_propagation_reaches_the_solver_state():
    """The c4 family (4-site chain, K = 2) at depth 2: RKF45 -- the
    propagator pinned to the reference build -- run for 700 ps, far past the
    slowest relaxation (0.046 per ps: population transfer along the chain),
    lands on the BiCGSTAB(2) steady state (the oracle, on the same run: 181,860
    attempted steps, rho_0 within 1.3e-13 of its dense steady-state solve)."""
    p = configs.chain4(seed=1000, depth=2)
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p) as h:
        h.rkf45(0.001, 700.0, 1e-10, 1e-9)
        rho_t = h.rho0()
        st = h.steady_state(tol=SOLVE_TOL, ell=2)
        rho_ss = h.rho0()
    assert st["converged"]
    assert np.abs(rho_t - rho_ss).max() <= 1e-8


def test_guess_at_solution_converges_immediately():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)
    with Hierarchy(p) as h:
        h.steady_state(tol=1e-12)
        x = h.get_state()
        st = h.steady_state(tol=1e-10, guess=3.0 * x)  # guesses are rescaled to rho_0[0,0] = 1
        y = h.get_state()
    assert st["converged"] and st["steps"] == 0
    assert np.abs(y - x).max() <= 1e-14 * np.abs(x).max()


def test_step_limit_reports_no_convergence():
    p = configs.frenkel7(depth=3)
    with Hierarchy(p) as h:
        st = h.steady_state(tol=1e-14, ell=2, max_steps=4, check=False)
    assert st["status"] == capi.PHI_E_NO_CONVERGENCE
    assert not st["converged"] and st["steps"] == 4


@pytest.mark.parametrize("mode", [capi.PHI_TOL_ABSOLUTE, capi.PHI_TOL_ABS_SQUARED])
def test_absolute_tolerance_modes(mode):
    """The reference's rules: ||r|| <= tol (BiCGSTAB(ell)) and ||r||^2 <= tol
    (BiCGSTAB); the reported residual is the compared quantity."""
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)
    with Hierarchy(p) as h:
        st = h.steady_state(tol=1e-6, tol_mode=mode)
        x = h.get_state()
        e00 = np.zeros(h.state_len)
        e00[0] = 1.0
        b = -h.apply(e00)
    assert st["converged"] and 0 < st["residual"] <= 1e-6
    # the solution is divided by tr rho_0; undo that to get the solver's residual
    raw = x / x[0]
    raw[:2] = 0
    with Hierarchy(p) as h:
        r = b - h.apply(raw)
    r[:2] = 0
    rn = np.linalg.norm(r)
    measured = rn * rn if mode == capi.PHI_TOL_ABS_SQUARED else rn
    assert measured <= 1e-6 * 1.01 + 1e-12, (measured, st)


def test_invalid_arguments_are_rejected():
    p = cases.random_problem("independent", n=2, matsubara=1, truncation=3, seed=1)
    with Hierarchy(p) as h:
        for kw in (dict(ell=0), dict(ell=9), dict(tol=0.0), dict(tol_mode=7)):
            st = h.steady_state(check=False, **kw)
            assert st["status"] == capi.PHI_E_INVALID, kw
