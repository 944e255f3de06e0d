"""The oracle's dense steady-state solve (the checker of the device BiCGSTAB):
Hermitian coordinates round-trip, L(rho_ss) = 0 including the dropped
equation, tr rho_0 = 1, and agreement with long-time propagation."""
import numpy as np

import cases
from oracle import oracle as O


def test_hermitian_coordinates_round_trip():
    p = cases.random_problem("independent", n=4, matsubara=1, truncation=3, seed=2)
    o = O.Oracle(p)
    s = cases.random_hermitian_state(o.M, 4, seed=5)
    assert np.array_equal(o._from_coords(o._to_coords(s)), s)


def test_liouvillian_matrix_matches_apply():
    p = cases.random_problem("full", n=2, matsubara=2, truncation=3, baths=2, seed=1)
    o = O.Oracle(p)
    A = o.liouvillian_matrix()
    s = cases.random_hermitian_state(o.M, 2, seed=7)
    np.testing.assert_allclose(A @ o._to_coords(s), o._to_coords(o.apply(s)), rtol=0, atol=1e-12 * np.abs(A).max())


def test_dense_steady_state_is_stationary():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)
    o = O.Oracle(p)
    x = o.steady_state()
    r = o.apply(x)
    assert np.abs(r).max() <= 1e-12 * np.abs(o.apply(o.initial_state())).max()
    rho = o.rho0(x)
    assert abs(np.trace(rho) - 1) <= 1e-14
    assert np.allclose(rho, rho.conj().T, rtol=0, atol=1e-15)


def test_dense_steady_state_is_long_time_limit():
    p = cases.random_problem("independent", n=2, matsubara=1, truncation=4, seed=5)
    o = O.Oracle(p)
    s, *_ = o.rk4(o.initial_state(), 0.001, 6.0)
    assert np.abs(o.rho0(s) - o.rho0(o.steady_state())).max() <= 1e-8
