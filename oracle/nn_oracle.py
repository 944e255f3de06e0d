"""CPU restatement of the learned initial guess's network -- TEST
INFRASTRUCTURE ONLY (the checker of phi_nn_* in phi_b200/csrc/nn_kernels.cu).

FP64 numpy forward and backward of the same layers (Y = tanh(X W^T + b) on
hidden layers, identity on the last) and loss (sum of squares / B), on the
BF16-rounded weights the device uses.
"""
from __future__ import annotations

import numpy as np


def forward(layers, X):
    acts = [np.asarray(X, dtype=np.float64)]
    for i, (W, b) in enumerate(layers):
        Z = acts[-1] @ W.T + b
        acts.append(np.tanh(Z) if i < len(layers) - 1 else Z)
    return acts


def loss_and_grads(layers, X, T):
    acts = forward(layers, X)
    B = X.shape[0]
    D = acts[-1] - T
    loss = float((D * D).sum() / B)
    dY = 2.0 * D / B
    gw, gb = [None] * len(layers), [None] * len(layers)
    for i in reversed(range(len(layers))):
        if i < len(layers) - 1:
            dY = dY * (1.0 - acts[i + 1] ** 2)
        gw[i] = dY.T @ acts[i]
        gb[i] = dY.sum(0)
        dY = dY @ layers[i][0]
    return loss, gw, gb
