"""The oracle pinned against the reference (CPU only).

1. The C restatement reproduces the rho_0 vectors hard-coded in the
   reference's own tests (src/hierarchy_integrator_test.cc:350-509) with the
   reference's tolerances: 1e-6 for RK4, 1e-3 for RKF45 (:316-340).
2. It reproduces rho_0 printed with %.17g by the reference build, case by
   case (tests/golden/ref_outputs.json), to 1e-12.
3. Its node order equals the reference ConstructI order
   (tests/golden/ref_order.json).
"""
import numpy as np
import pytest

import cases
import golden_data
from oracle import oracle as O

REF_VECTORS = golden_data.reference_test_vectors()


def _run_oracle(p, method, run):
    o = O.Oracle(p)
    s0 = o.initial_state()
    dt = run.get("timestep", p.timestep)
    t_end = run.get("t_end", p.integration_time)
    if method == "rk4":
        s, *_ = o.rk4(s0, dt, t_end)
    else:
        s, _ = o.rkf45(s0, dt, t_end, p.rkf45_tolerance, p.rkf45_minimum_timestep)
    return o.rho0(s)


def _physical(rho):
    """The reference's assertValidDensityMatrix (hierarchy_integrator_test.cc:253-282)."""
    n = rho.shape[0]
    assert np.all(np.abs(np.diag(rho).imag) < 1e-9)
    assert np.all(np.diag(rho).real >= 0)
    assert np.all(np.diag(rho).real < 1.00001)
    assert np.allclose(rho, rho.conj().T, atol=1e-9)
    tr = np.trace(rho).real
    assert 0 <= tr < 1.00001


@pytest.mark.parametrize("name", list(cases.REFERENCE_CASES))
@pytest.mark.parametrize("method", ["rk4", "rkf45"])
def test_oracle_matches_reference_test_vectors(name, method):
    key, _ = cases.REFERENCE_CASES[name]
    p = cases.reference_fixture_case(name)
    rho = _run_oracle(p, method, {})
    _physical(rho)
    tol = cases.RK4_TOL if method == "rk4" else cases.RKF45_TOL
    np.testing.assert_allclose(rho, REF_VECTORS[key], rtol=0, atol=tol)


REF_CASES = [c for c in golden_data.ref_outputs() if c[2] is not None]


@pytest.mark.parametrize("case", REF_CASES, ids=[c[0]["id"] for c in REF_CASES])
def test_oracle_matches_reference_build(case):
    c, p, rho_ref = case
    rho = _run_oracle(p, c["method"], c["run"])
    err = np.abs(rho - rho_ref).max()
    assert err <= 1e-12, err


@pytest.mark.parametrize("order", golden_data.ref_orders(), ids=lambda o: f"T{o[0]}_trunc{o[1]}")
def test_oracle_node_order_matches_reference(order):
    T, trunc, mi_ref = order
    mi = O.build_hierarchy(T, trunc)
    assert mi.shape == mi_ref.shape
    assert np.array_equal(mi, mi_ref)


def test_oracle_node_count_formula():
    for T in range(1, 9):
        for trunc in range(1, 7):
            from math import comb
            assert O.node_count(T, trunc) == comb(T + trunc - 1, trunc - 1)


def test_oracle_neighbour_symmetry():
    """next(prev(n)) = n for every link, and tiers differ by one."""
    p = cases.random_problem("independent", n=4, matsubara=2, truncation=4, seed=3)
    o = O.Oracle(p)
    mi, nx, pv = o.tables()
    tier = mi.sum(1)
    for i in range(o.M):
        for t in range(o.T):
            if nx[i, t] >= 0:
                assert pv[nx[i, t], t] == i and tier[nx[i, t]] == tier[i] + 1
            if pv[i, t] >= 0:
                assert nx[pv[i, t], t] == i and tier[pv[i, t]] == tier[i] - 1
            assert (pv[i, t] >= 0) == (mi[i, t] > 0)


def test_oracle_keeps_ados_hermitian():
    """PHI's formulation keeps every ADO Hermitian (all bath kinds)."""
    for kind in ("independent", "diagonal", "full"):
        p = cases.random_problem(kind, n=3, matsubara=2, truncation=3, seed=11)
        o = O.Oracle(p)
        s = cases.random_hermitian_state(o.M, 3, seed=2)
        d = o.apply(s).view(np.complex128).reshape(o.M, 3, 3)
        assert np.allclose(d, np.conj(np.transpose(d, (0, 2, 1))), atol=1e-9)
