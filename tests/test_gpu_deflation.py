"""Deflated steady-state solves (the ADOs of the lowest tiers as the
deflation space; heom_deflate.cu): the same solution as PHI's undeflated
BiCGSTAB(ell) and as the oracle's dense solve of the eliminated system, in
fewer iterations."""
import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

TOL = 1e-12

PROBLEMS = [
    # tiled kernel (fused inner products) and generic kernel (diagonal and full baths)
    ("chain4_L3", lambda: configs.chain4(seed=1000, depth=3)),
    ("indep_n3_K2_L4", lambda: cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)),
    ("diag_n3_b2_K1_L4", lambda: cases.random_problem("diagonal", n=3, matsubara=1, truncation=4, baths=2, seed=3)),
    ("full_n2_b2_K2_L4", lambda: cases.random_problem("full", n=2, matsubara=2, truncation=4, baths=2, seed=3)),
    # 36 coordinates per ADO: first-tier blocks inverted by the whole CTA instead of one warp each
    ("indep_n6_K1_L3", lambda: cases.random_problem("independent", n=6, matsubara=1, truncation=3, seed=4)),
]


def _solve(p, tiers, **kw):
    with Hierarchy(p) as h:
        h.set_steady_deflation(tiers)
        st = h.steady_state(tol=TOL, ell=2, max_steps=20000, **kw)
        return st, h.get_state()


@pytest.mark.parametrize("name,make", PROBLEMS, ids=[s[0] for s in PROBLEMS])
def test_deflated_solution_matches_dense_solve(name, make):
    p = make()
    o = O.Oracle(p)
    A = o.liouvillian_matrix()
    ref = o.steady_state(A)
    cond = np.linalg.cond(A[1:, 1:])
    scale = np.abs(ref).max()
    plain, x0 = _solve(p, 0)
    assert plain["deflated_tiers"] == 0 and plain["deflation_size"] == 0
    for tiers in (1, 2):
        st, x = _solve(p, tiers)
        E = p.num_states ** 2
        T = o.T
        assert st["deflated_tiers"] == tiers
        assert st["deflation_size"] == (1 if tiers == 1 else 1 + T) * E - 1
        assert st["converged"] and st["residual"] <= TOL
        err = np.abs(x - ref).max()
        assert err <= max(1e-10, 10 * TOL * cond) * scale, (tiers, err, cond, st)
        assert np.abs(o.rho0(x) - o.rho0(x0)).max() <= max(1e-10, 20 * TOL * cond) * scale


def test_deflation_cuts_iterations_on_the_chain4_family():
    """c4-family draws: the slow population modes sit in rho_0 and the first
    tier; deflating them at least halves the BiCG steps."""
    for seed in (1000, 1001):
        p = configs.chain4(seed=seed, depth=4)
        plain, x0 = _solve(p, 0)
        defl, x2 = _solve(p, 2)
        assert defl["deflated_tiers"] == 2 and defl["deflation_size"] == 207
        assert defl["steps"] <= 0.5 * plain["steps"], (seed, plain["steps"], defl["steps"])
        assert np.abs(x2 - x0).max() <= 1e-8 * np.abs(x0).max()


def test_true_residual_of_the_deflated_solution():
    """b - A x of the returned state (undivided by tr rho_0) meets the
    tolerance: the deflated residual is the true one."""
    p = configs.chain4(seed=1002, depth=3)
    with Hierarchy(p) as h:
        h.set_steady_deflation(2)
        st = h.steady_state(tol=1e-10, ell=2)
        x = h.get_state()
        e00 = np.zeros(h.state_len)
        e00[0] = 1.0
        b = -h.apply(e00)
        raw = x / x[0]
        raw[:2] = 0
        r = b - h.apply(raw)
    b[:2] = 0
    r[:2] = 0
    assert st["converged"] and st["deflated_tiers"] == 2
    assert np.linalg.norm(r) <= 1.05e-10 * np.linalg.norm(b), (np.linalg.norm(r) / np.linalg.norm(b), st)


def test_automatic_choice_and_refusals():
    # frenkel7: 14 terms, 49 coordinates per ADO -> tiers 0..1 have 734 > 256
    p = configs.frenkel7(depth=2)
    with Hierarchy(p) as h:
        st = h.steady_state(tol=1e-10)
        assert st["deflated_tiers"] == 1 and st["deflation_size"] == 48
        st = h.steady_state(tol=1e-10, ell=4)  # automatic deflation is for ell <= 2
        assert st["converged"] and st["deflated_tiers"] == 0
        with pytest.raises(capi.PhiError) as e:
            h.set_steady_deflation(2)
        assert e.value.code == capi.PHI_E_INVALID
        for bad in (-2, 3):
            with pytest.raises(capi.PhiError):
                h.set_steady_deflation(bad)
    q = configs.chain4(seed=1000, depth=3)
    with Hierarchy(q) as h:
        st = h.steady_state(tol=1e-10)
        assert st["deflated_tiers"] == 2 and st["deflation_size"] == 207


def test_deflation_with_guesses():
    p = configs.chain4(seed=1003, depth=3)
    ref_st, ref = _solve(p, 0)
    rho = np.eye(4, dtype=np.complex128) / 4
    st, x = _solve(p, 2, rho0_guess=rho + 0.01 * np.diag([1, -1, 1, -1]))
    assert st["converged"]
    assert np.abs(x - ref).max() <= 1e-8 * np.abs(ref).max()
    # a guess at the solution: no step, the coarse correction leaves it in place
    with Hierarchy(p) as h:
        h.set_steady_deflation(2)
        st = h.steady_state(tol=1e-10, guess=2.0 * x)
        y = h.get_state()
    assert st["converged"] and st["steps"] == 0
    assert np.abs(y - x).max() <= 1e-12 * np.abs(x).max()
