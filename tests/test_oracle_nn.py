"""The CPU oracle of the learned guess's network: analytic gradients equal
central finite differences."""
import numpy as np

from oracle import nn_oracle


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    widths = [5, 7, 6, 3]
    layers = [(rng.normal(size=(widths[i + 1], widths[i])) * 0.5, rng.normal(size=widths[i + 1]) * 0.1)
              for i in range(3)]
    X = rng.normal(size=(9, 5))
    T = rng.normal(size=(9, 3))
    loss, gw, gb = nn_oracle.loss_and_grads(layers, X, T)
    h = 1e-6
    for li, (W, b) in enumerate(layers):
        for idx in [(0, 0), (1, 2), (widths[li + 1] - 1, widths[li] - 1)]:
            W[idx] += h
            lp = nn_oracle.loss_and_grads(layers, X, T)[0]
            W[idx] -= 2 * h
            lm = nn_oracle.loss_and_grads(layers, X, T)[0]
            W[idx] += h
            assert abs((lp - lm) / (2 * h) - gw[li][idx]) <= 1e-6 * max(1.0, abs(gw[li][idx]))
        b[0] += h
        lp = nn_oracle.loss_and_grads(layers, X, T)[0]
        b[0] -= 2 * h
        lm = nn_oracle.loss_and_grads(layers, X, T)[0]
        b[0] += h
        assert abs((lp - lm) / (2 * h) - gb[li][0]) <= 1e-6 * max(1.0, abs(gb[li][0]))


def test_rho_coordinates_round_trip():
    from phi_b200 import learned
    rng = np.random.default_rng(3)
    A = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    rho = A + A.conj().T
    c = learned.rho_to_coords(rho)
    assert c.shape == (16,)
    assert np.allclose(learned.coords_to_rho(c, 4), rho, rtol=0, atol=1e-15)
