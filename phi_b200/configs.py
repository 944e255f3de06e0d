"""Seeded synthetic workloads (the benchmark configurations of this path).

Units follow PHI's defaults: energies in cm^-1, times in ps, temperatures in
K, hbar = 5.3088354 cm^-1 ps, k_B = 0.6950344 cm^-1/K.  A Drude bath with
response time tau has Gamma = 1/tau (100 fs -> 10 ps^-1).  Every random draw
uses numpy.random.default_rng(seed) with the seed recorded in the returned
parameters' `seed` attribute.
"""
from __future__ import annotations

import numpy as np

from .heom import PhiParameters


def _basis_state(n: int, k: int) -> np.ndarray:
    r = np.zeros((n, n), np.complex128)
    r[k, k] = 1.0
    return r


def spin_boson(seed: int = 0) -> PhiParameters:
    """Spin-boson qubit: H = (eps/2) sigma_z + Delta sigma_x with eps = 100,
    Delta = 50 cm^-1; one Drude bath on sigma_z (diagonal coupling 1, -1),
    lambda = 20 cm^-1, 1/gamma = 100 fs, T = 300 K, K = 0, depth L = 10
    (HierarchyTruncation = 11); rho(0) = |0><0|; RK4 dt = 1 fs to 2 ps,
    output every 10 fs."""
    p = PhiParameters(
        num_states=2,
        time_indepenent_hamiltonian=np.array([[50.0, 50.0], [50.0, -50.0]], np.complex128),
        num_bath_couplings=1, num_matsubara_terms=1, hierarchy_truncation_level=11,
        gamma=np.array([10.0]), lambda_=np.array([20.0]),
        bath_coupling_op=np.array([[1.0, -1.0]]), is_diagonal_bath_coupling=True,
        initial_density_matrix=_basis_state(2, 0), temperature=300.0,
        timestep=0.001, integration_time=2.0, output_minimum_timestep=0.01)
    p.seed = seed
    p.name = "spin_boson_L10"
    return p


def frenkel7(seed: int = 7, depth: int = 6) -> PhiParameters:
    """7-site Frenkel exciton: site energies U[0, 600] cm^-1, symmetric
    off-diagonal couplings N(0, 50 cm^-1); one Drude bath per site (site
    projector), lambda = 35 cm^-1, 1/gamma = 50 fs, T = 300 K, K = 1, depth
    L = 6 (38,760 nodes of 7x7); rho(0) = |1><1|; RKF45 tol 1e-6 to 1 ps."""
    rng = np.random.default_rng(seed)
    n = 7
    H = np.zeros((n, n))
    H[np.diag_indices(n)] = rng.uniform(0.0, 600.0, size=n)
    off = rng.normal(0.0, 50.0, size=(n, n))
    iu = np.triu_indices(n, 1)
    H[iu] = off[iu]
    H = np.triu(H) + np.triu(H, 1).T
    p = PhiParameters(
        num_states=n, time_indepenent_hamiltonian=H.astype(np.complex128),
        num_bath_couplings=n, num_matsubara_terms=2, hierarchy_truncation_level=depth + 1,
        gamma=np.full(n, 20.0), lambda_=np.full(n, 35.0),
        initial_density_matrix=_basis_state(n, 1), temperature=300.0,
        timestep=0.001, integration_time=1.0, rkf45_tolerance=1e-6,
        rkf45_minimum_timestep=1e-6)
    p.seed = seed
    p.name = f"frenkel7_K1_L{depth}"
    return p


def chain4(seed: int = 4, depth: int = 8) -> PhiParameters:
    """4-site chain for the steady state: site energies U[0, 300] cm^-1,
    nearest-neighbour couplings N(0, 60 cm^-1), 4 Drude baths lambda = 50,
    1/gamma = 50 fs, T = 300 K, K = 2, depth L = 8 (125,970 nodes of 4x4)."""
    rng = np.random.default_rng(seed)
    n = 4
    H = np.diag(rng.uniform(0.0, 300.0, size=n))
    J = rng.normal(0.0, 60.0, size=n - 1)
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = J[i]
    p = PhiParameters(
        num_states=n, time_indepenent_hamiltonian=H.astype(np.complex128),
        num_bath_couplings=n, num_matsubara_terms=3, hierarchy_truncation_level=depth + 1,
        gamma=np.full(n, 20.0), lambda_=np.full(n, 50.0),
        initial_density_matrix=_basis_state(n, 0), temperature=300.0,
        timestep=0.001, integration_time=1.0, bicgstab_tolerance=1e-10)
    p.seed = seed
    p.name = f"chain4_K2_L{depth}"
    return p


def ring24(seed: int = 24, depth: int = 4) -> PhiParameters:
    """24-site ring: site energies N(0, 100 cm^-1), nearest-neighbour
    coupling 300 cm^-1 and next-nearest 30 cm^-1 (periodic); 24 Drude baths
    lambda = 40, 1/gamma = 100 fs, T = 300 K, K = 0, depth L = 4 (20,475
    nodes of 24x24); RKF45 tol 1e-6 to 500 fs."""
    rng = np.random.default_rng(seed)
    n = 24
    H = np.diag(rng.normal(0.0, 100.0, size=n))
    for i in range(n):
        for d, J in ((1, 300.0), (2, 30.0)):
            j = (i + d) % n
            H[i, j] = H[j, i] = J
    p = PhiParameters(
        num_states=n, time_indepenent_hamiltonian=H.astype(np.complex128),
        num_bath_couplings=n, num_matsubara_terms=1, hierarchy_truncation_level=depth + 1,
        gamma=np.full(n, 10.0), lambda_=np.full(n, 40.0),
        initial_density_matrix=_basis_state(n, 0), temperature=300.0,
        timestep=0.001, integration_time=0.5, rkf45_tolerance=1e-6,
        rkf45_minimum_timestep=1e-6)
    p.seed = seed
    p.name = f"ring24_K0_L{depth}"
    return p


BATCH_DIMS = (2, 3, 4, 6, 8, 12, 16)
BATCH_BUDGET_BYTES = 256 * 2**20


def hierarchy_nodes(terms: int, depth: int) -> int:
    """Nodes of a hierarchy with `terms` exponentials truncated at tier
    `depth`: C(terms + depth, depth)."""
    from math import comb
    return comb(terms + depth, depth)


def batched(seed: int = 3, count: int = 512, budget_bytes: int = BATCH_BUDGET_BYTES,
            depth_range=(4, 10)) -> list:
    """Uneven independent instances: N uniform in {2,3,4,6,8,12,16}; a chain
    with site energies U[0, 400] cm^-1 and nearest-neighbour couplings
    N(0, 80 cm^-1); one Drude bath per site with lambda U[10, 100] cm^-1 and
    1/gamma U[20, 200] fs; T U[77, 300] K; K in {0, 1}; depth L uniform in
    depth_range.  Budget rule: while the FP64 state M*N^2*16 B exceeds
    budget_bytes, L is decremented (floor 1); each instance records
    `depth_drawn` and `depth`.  rho(0) = |0><0|; RK4 dt = 0.5 fs, 1000 steps.
    N = 2 instances are dimers with one bath per site."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(BATCH_DIMS))
        k = int(rng.integers(0, 2))
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        H = np.diag(rng.uniform(0.0, 400.0, size=n))
        J = rng.normal(0.0, 80.0, size=n - 1)
        for s in range(n - 1):
            H[s, s + 1] = H[s + 1, s] = J[s]
        lam = rng.uniform(10.0, 100.0, size=n)
        tau_fs = rng.uniform(20.0, 200.0, size=n)
        temp = float(rng.uniform(77.0, 300.0))
        drawn = depth
        terms = n * (k + 1)
        while depth > 1 and hierarchy_nodes(terms, depth) * n * n * 16 > budget_bytes:
            depth -= 1
        p = PhiParameters(
            num_states=n, time_indepenent_hamiltonian=H.astype(np.complex128),
            num_bath_couplings=n, num_matsubara_terms=k + 1, hierarchy_truncation_level=depth + 1,
            gamma=1000.0 / tau_fs, lambda_=lam,
            initial_density_matrix=_basis_state(n, 0), temperature=temp,
            timestep=0.0005, integration_time=0.5)
        p.seed = seed
        p.index = i
        p.depth_drawn = drawn
        p.depth = depth
        p.nodes = hierarchy_nodes(terms, depth)
        p.name = f"batch{seed}_{i}_N{n}_K{k}_L{depth}"
        out.append(p)
    return out


def batch_summary(problems) -> dict:
    """Histogram of effective depths, drawn-vs-effective depth changes and
    the total FP64 state of a batched() draw."""
    hist = {}
    for p in problems:
        hist[p.depth] = hist.get(p.depth, 0) + 1
    return {
        "instances": len(problems),
        "depth_histogram": dict(sorted(hist.items())),
        "depth_reduced": sum(1 for p in problems if p.depth != p.depth_drawn),
        "total_nodes": int(sum(p.nodes for p in problems)),
        "state_bytes_fp64": int(sum(p.nodes * p.num_states ** 2 * 16 for p in problems)),
    }
