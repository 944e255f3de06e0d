"""Learned initial guess for the steady state.

A small multilayer perceptron maps the parameters of a problem family (the
4-site chain of chain4: site energies and nearest-neighbour couplings) to the
steady-state system density matrix rho_0, in Hermitian coordinates (N*N
reals: (i,i) -> Re, (i<j) -> Re X_ij, (i>j) -> Im X_ji).  It predicts the
difference between the steady state and the thermal state
exp(-H/kT)/Z of the system Hamiltonian -- the guess PrepForSteadyState
builds from eigen data (hierarchy_integrator.cc:1547-1588) -- which is about
ten times smaller and smoother than rho_0 itself.  BiCGSTAB(ell)
starts from that rho_0 with every other node zero
(phi_gpu_steady_state_rho0); the solver alone decides the error, so a poor
prediction costs iterations, never accuracy.

Training data are steady states the method itself produced (BiCGSTAB(2) to a
relative residual of 1e-10).  Forward, backward, loss and Adam run in the
library's own kernels (phi_nn_*); torch only holds the device buffers.
Weights are BF16 for the products, with FP32 master copies; accumulation is
FP32.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "chain4_rho0_mlp.npz")
DATASET = os.path.join(HERE, "data", "chain4_steady_states.npz")


# ---- features and targets ---------------------------------------------------

def chain_features(p) -> np.ndarray:
    """Site energies / 300 and nearest-neighbour couplings / 60 of a chain."""
    H = np.asarray(p.time_indepenent_hamiltonian).real
    n = H.shape[0]
    return np.concatenate([np.diag(H) / 300.0, np.array([H[i, i + 1] for i in range(n - 1)]) / 60.0])


def rho_to_coords(rho: np.ndarray) -> np.ndarray:
    """Hermitian N x N -> N*N reals in column-major element order."""
    rho = np.asarray(rho)
    n = rho.shape[0]
    c = np.empty((n, n))
    for j in range(n):
        for i in range(n):
            c[i, j] = rho[i, i].real if i == j else (rho[i, j].real if i < j else rho[j, i].imag)
    return c.T.reshape(-1)


def thermal_rho0(p) -> np.ndarray:
    """exp(-H / k_B T) / Z of the system Hamiltonian (eigen decomposition on
    the host; the reference's guess when eigen data is present)."""
    H = np.asarray(p.time_indepenent_hamiltonian, dtype=np.complex128)
    w, V = np.linalg.eigh(H)
    pop = np.exp(-(w - w.min()) / (p.boltzmann_constant * p.temperature))
    pop /= pop.sum()
    return (V * pop) @ V.conj().T


def coords_to_rho(c: np.ndarray, n: int) -> np.ndarray:
    c = np.asarray(c, dtype=np.float64).reshape(n, n).T  # c[i, j]
    rho = np.zeros((n, n), np.complex128)
    for i in range(n):
        rho[i, i] = c[i, i]
        for j in range(i + 1, n):
            rho[i, j] = c[i, j] + 1j * c[j, i]
            rho[j, i] = np.conj(rho[i, j])
    return rho


# ---- the network ------------------------------------------------------------

class MLP:
    """Layers widths[0] -> ... -> widths[-1]; tanh on hidden layers."""

    def __init__(self, widths, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.lib = capi.load()
        self.widths = list(widths)
        self.device = torch.device("cuda", device)
        rng = np.random.default_rng(seed)
        self.w, self.b = [], []
        for i in range(len(widths) - 1):
            fan_in, fan_out = widths[i], widths[i + 1]
            lim = np.sqrt(6.0 / (fan_in + fan_out))
            self.w.append(torch.tensor(rng.uniform(-lim, lim, size=(fan_out, fan_in)), dtype=torch.float32,
                                       device=self.device))
            self.b.append(torch.zeros(fan_out, dtype=torch.float32, device=self.device))
        self.w16 = [torch.empty(w.shape, dtype=torch.bfloat16, device=self.device) for w in self.w]
        self._sync_bf16()
        self.adam = None
        self.step = 0
        self.x_mean = np.zeros(widths[0], np.float32)
        self.x_std = np.ones(widths[0], np.float32)
        self.y_mean = np.zeros(widths[-1], np.float32)
        self.y_std = np.ones(widths[-1], np.float32)

    @property
    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _sync_bf16(self):
        for w, w16 in zip(self.w, self.w16):
            capi.check(self.lib.phi_nn_to_bf16(w.data_ptr(), w16.data_ptr(), w.numel(), self.stream))

    def _forward(self, X):
        """X: (B, in) float32 device tensor, normalised.  Returns the
        activations of every layer (input first)."""
        torch = self.torch
        acts = [X.contiguous()]
        L = len(self.w)
        for i in range(L):
            B = acts[-1].shape[0]
            Y = torch.empty((B, self.widths[i + 1]), dtype=torch.float32, device=self.device)
            capi.check(self.lib.phi_nn_linear_forward(acts[-1].data_ptr(), self.w16[i].data_ptr(),
                                                      self.b[i].data_ptr(), Y.data_ptr(), B, self.widths[i],
                                                      self.widths[i + 1], 1 if i < L - 1 else 0, self.stream))
            acts.append(Y)
        return acts

    def loss_and_grads(self, X, T):
        """MSE loss of the normalised outputs and its gradients (dW, db per
        layer), from the library's backward kernels."""
        torch = self.torch
        acts = self._forward(X)
        B = X.shape[0]
        dY = torch.empty_like(acts[-1])
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        capi.check(self.lib.phi_nn_mse(acts[-1].data_ptr(), T.data_ptr(), dY.data_ptr(), loss.data_ptr(),
                                       acts[-1].numel(), B, self.stream))
        gw, gb = [None] * len(self.w), [None] * len(self.w)
        L = len(self.w)
        for i in reversed(range(L)):
            dX = torch.empty_like(acts[i]) if i > 0 else None
            gw[i] = torch.empty_like(self.w[i])
            gb[i] = torch.empty_like(self.b[i])
            capi.check(self.lib.phi_nn_linear_backward(
                dY.data_ptr(), acts[i + 1].data_ptr(), acts[i].data_ptr(), self.w16[i].data_ptr(),
                dX.data_ptr() if dX is not None else None, gw[i].data_ptr(), gb[i].data_ptr(), B,
                self.widths[i], self.widths[i + 1], 1 if i < L - 1 else 0, self.stream))
            dY = dX
        return loss, gw, gb

    def train_step(self, X, T, lr: float, b1=0.9, b2=0.999, eps=1e-8):
        torch = self.torch
        if self.adam is None:
            self.adam = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.w + self.b]
        loss, gw, gb = self.loss_and_grads(X, T)
        self.step += 1
        params = self.w + self.b
        grads = gw + gb
        w16 = self.w16 + [None] * len(self.b)
        for p, g, (m, v), p16 in zip(params, grads, self.adam, w16):
            capi.check(self.lib.phi_nn_adam(p.data_ptr(), p16.data_ptr() if p16 is not None else None,
                                            g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), lr, b1, b2, eps,
                                            self.step, self.stream))
        return loss

    def fit(self, features, targets, steps=4000, lr=3e-3, lr_final=3e-5):
        """Full-batch Adam on (features, targets) numpy arrays; inputs and
        outputs standardised per column.  Returns the loss history."""
        torch = self.torch
        self.x_mean = features.mean(0).astype(np.float32)
        self.x_std = (features.std(0) + 1e-8).astype(np.float32)
        self.y_mean = targets.mean(0).astype(np.float32)
        self.y_std = (targets.std(0) + 1e-8).astype(np.float32)
        X = torch.tensor((features - self.x_mean) / self.x_std, dtype=torch.float32, device=self.device)
        T = torch.tensor((targets - self.y_mean) / self.y_std, dtype=torch.float32, device=self.device)
        hist = []
        for k in range(steps):
            lr_k = lr * (lr_final / lr) ** (k / max(steps - 1, 1))
            loss = self.train_step(X, T, lr_k)
            if k % 100 == 0 or k == steps - 1:
                hist.append(float(loss.item()))
        return hist

    def predict(self, features) -> np.ndarray:
        torch = self.torch
        X = torch.tensor((np.atleast_2d(features) - self.x_mean) / self.x_std, dtype=torch.float32,
                         device=self.device)
        Y = self._forward(X)[-1].cpu().numpy()
        return Y * self.y_std + self.y_mean

    def save(self, path: str = WEIGHTS):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        arrays = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        arrays.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        np.savez(path, widths=np.array(self.widths), x_mean=self.x_mean, x_std=self.x_std, y_mean=self.y_mean,
                 y_std=self.y_std, **arrays)

    @classmethod
    def load(cls, path: str = WEIGHTS, device: int = 0) -> "MLP":
        import torch
        z = np.load(path)
        m = cls([int(x) for x in z["widths"]], device=device)
        for i in range(len(m.w)):
            m.w[i] = torch.tensor(z[f"w{i}"], dtype=torch.float32, device=m.device)
            m.b[i] = torch.tensor(z[f"b{i}"], dtype=torch.float32, device=m.device)
        m._sync_bf16()
        m.x_mean, m.x_std, m.y_mean, m.y_std = z["x_mean"], z["x_std"], z["y_mean"], z["y_std"]
        return m

    def host_weights(self):
        """(W rounded to BF16 as float64, b) per layer, for the CPU oracle."""
        out = []
        for w16, b in zip(self.w16, self.b):
            out.append((w16.float().cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64)))
        return out


def training_target(p, rho_ss) -> np.ndarray:
    """What the network learns: coordinates of rho_ss minus the thermal state."""
    return rho_to_coords(rho_ss) - rho_to_coords(thermal_rho0(p))


def predict_rho0(model: MLP, p) -> np.ndarray:
    """Network estimate of the steady-state rho_0 of problem p (trace 1):
    the thermal state plus the predicted correction."""
    c = model.predict(chain_features(p))[0] + rho_to_coords(thermal_rho0(p))
    rho = coords_to_rho(c, p.num_states)
    tr = np.trace(rho).real
    return rho / tr if abs(tr) > 1e-12 else rho
