"""The deflated steady-state method on the CPU, with the oracle's apply as
the operator: BiCGSTAB(2) on P A y = P b, P = I - A Z (Z^T A Z)^-1 Z^T with Z
the real coordinates of the ADOs of tiers 0..1, then
x = y + Z (Z^T A Z)^-1 Z^T (b - A y).  It reaches the oracle's dense
steady state with the same residual and far fewer steps: the algebra the
device solver (heom_deflate.cu) implements, checked without a GPU."""
import numpy as np

from oracle import oracle as O
from phi_b200 import configs


def _bicgstab2(A, b, proj, tol=1e-10, maxit=4000):
    """BiCGSTAB(2) (Sleijpen and Fokkema) with every operator product
    followed by proj; returns (x, BiCG steps)."""
    ell = 2
    Ap = lambda v: proj(A(v))
    x = np.zeros_like(b)
    r = [proj(b - A(x)), None, None]
    u = [np.zeros_like(b), None, None]
    rh = r[0].copy()
    rho0, alpha, om, nb, steps = 1.0, 0.0, 1.0, np.linalg.norm(b), 0
    while steps < maxit and np.linalg.norm(r[0]) > tol * nb:
        rho0 = -om * rho0
        for j in range(ell):
            rho1 = rh @ r[j]
            beta = alpha * rho1 / rho0
            rho0 = rho1
            for i in range(j + 1):
                u[i] = r[i] - beta * u[i]
            u[j + 1] = Ap(u[j])
            alpha = rho0 / (rh @ u[j + 1])
            for i in range(j + 1):
                r[i] = r[i] - alpha * u[i + 1]
            r[j + 1] = Ap(r[j])
            x = x + alpha * u[0]
        G = np.array([[r[i] @ r[k] for k in (1, 2)] for i in (1, 2)])
        g = np.linalg.solve(G, np.array([r[1] @ r[0], r[2] @ r[0]]))
        om = g[-1]
        for i in range(ell):
            u[0] = u[0] - g[i] * u[i + 1]
            x = x + g[i] * r[i]
            r[0] = r[0] - g[i] * r[i + 1]
        steps += ell
    return x, steps


def test_low_tier_deflation_reaches_the_dense_solution_in_fewer_steps():
    p = configs.chain4(seed=1000, depth=3)
    o = O.Oracle(p)
    mi, _, _ = o.tables()
    E = o.n * o.n
    tier = np.repeat(mi.sum(1), E)
    D = o.M * E

    def A(v):  # the eliminated operator: coordinate 0 pinned, its equation dropped
        w = v.copy()
        w[0] = 0.0
        out = o._to_coords(o.apply(o._from_coords(w)))
        out[0] = 0.0
        return out

    e0 = np.zeros(D)
    e0[0] = 1.0
    b = -o._to_coords(o.apply(o._from_coords(e0)))  # minus the column of rho_0[0,0]
    b[0] = 0.0
    dense = o._to_coords(o.steady_state())          # x with x[0] = rho_0[0,0] / tr rho_0
    ref = dense / dense[0]
    ref[0] = 0.0                                     # the eliminated unknown

    idx = np.where(tier <= 1)[0][1:]                 # tiers 0..1 without element (0,0)
    assert len(idx) == (1 + o.T) * E - 1 == 207
    AZ = np.empty((D, len(idx)))
    for j, q in enumerate(idx):
        v = np.zeros(D)
        v[q] = 1.0
        AZ[:, j] = A(v)
    Einv = np.linalg.inv(AZ[idx, :])
    P = lambda v: v - AZ @ (Einv @ v[idx])

    x_plain, n_plain = _bicgstab2(A, b, lambda v: v)
    y, n_defl = _bicgstab2(A, b, P)
    x = y.copy()
    x[idx] += Einv @ (b - A(y))[idx]                 # the coarse correction

    for got in (x_plain, x):
        assert np.linalg.norm(b - A(got)) <= 1.01e-10 * np.linalg.norm(b)
        assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
    assert n_defl <= 0.6 * n_plain, (n_plain, n_defl)
