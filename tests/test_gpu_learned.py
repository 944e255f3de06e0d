"""The learned steady-state initial guess on the GPU.

* The library's forward and backward kernels (phi_nn_*) equal the CPU
  oracle's FP64 restatement on the same BF16-rounded weights (FP32
  accumulation: relative 1e-4).
* Adam matches its formula; training with the library's kernels fits.
* The trained network's rho_0 is closer to the steady state than the
  thermal and I/N guesses on held-out draws, and BiCGSTAB(2) started from it
  reaches the same steady state.
"""
import os

import numpy as np
import pytest
import torch

from oracle import nn_oracle
from phi_b200 import capi, configs, learned, train_guess

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def test_forward_and_gradients_match_cpu_oracle():
    m = learned.MLP([7, 32, 24, 16], seed=5)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(64, 7)).astype(np.float32)
    T = rng.normal(size=(64, 16)).astype(np.float32)
    Xd = torch.tensor(X, device="cuda")
    Td = torch.tensor(T, device="cuda")
    loss, gw, gb = m.loss_and_grads(Xd, Td)
    layers = m.host_weights()
    loss_o, gw_o, gb_o = nn_oracle.loss_and_grads(layers, X.astype(np.float64), T.astype(np.float64))
    assert abs(float(loss.item()) - loss_o) <= 1e-5 * loss_o
    for i in range(3):
        assert _rel(gw[i].cpu().numpy(), gw_o[i]) <= 1e-4, i
        assert _rel(gb[i].cpu().numpy(), gb_o[i]) <= 1e-4, i
    acts = nn_oracle.forward(layers, X.astype(np.float64))
    out = m._forward(Xd)[-1].cpu().numpy()
    assert _rel(out, acts[-1]) <= 1e-5


def test_adam_step_matches_formula():
    lib = capi.load()
    rng = np.random.default_rng(2)
    n = 1000
    w = rng.normal(size=n).astype(np.float32)
    g = rng.normal(size=n).astype(np.float32)
    m0 = rng.normal(size=n).astype(np.float32) * 0.1
    v0 = np.abs(rng.normal(size=n)).astype(np.float32) * 0.1
    wd, gd, md, vd = (torch.tensor(a, device="cuda") for a in (w, g, m0, v0))
    w16 = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    capi.check(lib.phi_nn_adam(wd.data_ptr(), w16.data_ptr(), gd.data_ptr(), md.data_ptr(), vd.data_ptr(), n,
                               1e-2, 0.9, 0.999, 1e-8, 3, None))
    torch.cuda.synchronize()
    m1 = 0.9 * m0 + 0.1 * g
    v1 = 0.999 * v0 + 0.001 * g * g
    w1 = w - 1e-2 * (m1 / (1 - 0.9 ** 3)) / (np.sqrt(v1 / (1 - 0.999 ** 3)) + 1e-8)
    assert np.allclose(wd.cpu().numpy(), w1, rtol=1e-5, atol=1e-6)
    assert np.allclose(w16.float().cpu().numpy(), w1, rtol=1e-2, atol=1e-2)


def test_training_with_library_kernels_fits_a_smooth_map():
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, size=(512, 3))
    Y = np.stack([np.sin(2 * X[:, 0]) * X[:, 1], np.cos(X[:, 2]) + X[:, 0] ** 2], axis=1)
    m = learned.MLP([3, 64, 64, 2], seed=1)
    hist = m.fit(X, Y, steps=1500, lr=3e-3, lr_final=1e-4)
    assert hist[-1] < 0.01 * hist[0], hist[::5]
    err = np.abs(m.predict(X) - Y).max()
    assert err < 0.1, err


def test_trained_guess_beats_thermal_and_identity_guesses_on_held_out_draws():
    """What the trained network gains: on held-out draws its rho_0 is closer
    to the steady state than the thermal state (the reference's eigen guess)
    and than I/N, and BiCGSTAB(2) started from it reaches the same steady
    state (within the solve's conditioning) without more failures."""
    assert os.path.exists(learned.WEIGHTS), "committed weights missing"
    res = train_guess.evaluate(6, seed0=train_guess.EVAL_SEED0 + 200)
    assert res["learned_failed"] == 0
    assert res["guess_err_median"] < 0.5 * res["thermal_err_median"] < res["identity_err_median"], res
    assert res["max_rho0_diff"] <= 1e-4, res
