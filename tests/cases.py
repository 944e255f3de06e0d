"""Problem builders shared by the tests.

`reference_fixture_case(name)` restates the problems of the reference's own
golden tests (src/hierarchy_integrator_test.cc): the fixture of :27-44 (hbar =
k_B = 1, T = 2, run to t = 1), the two-state Hamiltonian of :46-54, the weak
bath of :143-151 (gamma = 1, lambda = 0.01 for every term: the reference's
`1.0 + i/10` is integer division), the coupling operators of :163-229 and
rho(0) = |0><0| (:231-239).  Only the cases in scope for this path are listed
(static Hamiltonian, untruncated Hilbert space, no time-local closure).
"""
from __future__ import annotations

import numpy as np

from phi_b200.heom import PhiParameters

# name -> (golden vector key, builder kwargs)
REFERENCE_CASES = {
    "TestVacuum": ("kVacuumSoln", dict(baths=1, truncation=1)),
    "TestWeakIndependentBath": ("kWeakIndependentCouplingSoln", dict(baths=2, truncation=2)),
    "TestWeakIndependentDiagonalBath": ("kWeakIndependentCouplingSoln",
                                        dict(baths=2, truncation=2, coupling="diag_identity")),
    "WeakIndependentFullBath": ("kWeakIndependentCouplingSoln",
                                dict(baths=2, truncation=2, coupling="full_identity")),
    "TestWeakDiagonalBath": ("kWeakDiagonalCouplingSoln",
                             dict(baths=2, truncation=2, coupling="diag_alternating")),
    "TestWeakFullDiagonalBath": ("kWeakDiagonalCouplingSoln",
                                 dict(baths=2, truncation=2, coupling="full_diag_alternating")),
    "TestWeakFullBath": ("kWeakFullCouplingSoln",
                         dict(baths=2, truncation=2, coupling="full_alternating")),
    "TestWeakIndependentBathMatsubara": ("kWeakIndependentCouplingMatsubaraSoln",
                                         dict(baths=2, truncation=3, matsubara=3, temperature=0.5)),
    "TestWeakDiagonalBathMatsubara": ("kWeakIndependentCouplingMatsubaraSoln",
                                      dict(baths=2, truncation=3, matsubara=3, temperature=0.5,
                                           coupling="diag_identity")),
    "TestWeakFullBathMatsubara": ("kWeakIndependentCouplingMatsubaraSoln",
                                  dict(baths=2, truncation=3, matsubara=3, temperature=0.5,
                                       coupling="full_identity")),
}

# Tolerances of the reference's assertions (hierarchy_integrator_test.cc:316-340).
RK4_TOL = 1e-6
RKF45_TOL = 1e-3


def reference_fixture_case(name: str) -> PhiParameters:
    _, kw = REFERENCE_CASES[name]
    n = 2
    nb = kw["baths"]
    p = PhiParameters(
        num_states=n,
        time_indepenent_hamiltonian=np.array([[0.5, 0.5], [0.5, -0.5]], np.complex128),
        num_bath_couplings=nb, num_matsubara_terms=kw.get("matsubara", 1),
        hierarchy_truncation_level=kw["truncation"],
        gamma=np.full(nb, 1.0), lambda_=np.full(nb, 0.01),
        temperature=kw.get("temperature", 2.0), hbar=1.0, boltzmann_constant=1.0,
        integration_time=1.0, timestep=0.001, rkf45_tolerance=1e-6, rkf45_minimum_timestep=1e-6)
    rho = np.zeros((n, n), np.complex128)
    rho[0, 0] = 1.0
    p.initial_density_matrix = rho
    c = kw.get("coupling")
    if c == "diag_identity":
        p.bath_coupling_op = np.eye(n)[:nb]
        p.is_diagonal_bath_coupling = True
    elif c == "full_identity":
        V = np.zeros((nb, n, n))
        for i in range(nb):
            V[i, i, i] = 1.0
        p.bath_coupling_op = V
        p.is_full_bath_coupling = True
    elif c == "diag_alternating":
        p.bath_coupling_op = np.array([[(-1.0) ** (i + j) for j in range(n)] for i in range(nb)])
        p.is_diagonal_bath_coupling = True
    elif c == "full_diag_alternating":
        V = np.zeros((nb, n, n))
        for i in range(nb):
            for j in range(n):
                V[i, j, j] = (-1.0) ** (i + j)
        p.bath_coupling_op = V
        p.is_full_bath_coupling = True
    elif c == "full_alternating":
        V = np.array([[[(-1.0) ** (i + j + k) for k in range(n)] for j in range(n)]
                      for i in range(nb)])
        p.bath_coupling_op = V
        p.is_full_bath_coupling = True
    return p


def random_problem(kind: str = "independent", n: int = 3, matsubara: int = 2, truncation: int = 3,
                   baths: int | None = None, seed: int = 0, normalized: bool = True,
                   complex_h: bool = False, scale: float = 50.0) -> PhiParameters:
    """Seeded random problem in PHI's units (cm^-1, ps, K)."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) + (1j * rng.normal(size=(n, n)) if complex_h else 0)
    H = (A + np.conj(A).T) / 2 * scale
    p = PhiParameters(num_states=n, time_indepenent_hamiltonian=np.asarray(H, np.complex128),
                      num_matsubara_terms=matsubara, hierarchy_truncation_level=truncation,
                      temperature=300.0, is_rho_normalized=normalized)
    rho = np.zeros((n, n), np.complex128)
    rho[0, 0] = 0.7
    rho[n - 1, n - 1] += 0.3
    if n > 1:
        rho[0, n - 1] = 0.1 + 0.05j
        rho[n - 1, 0] = 0.1 - 0.05j
    p.initial_density_matrix = rho
    if kind == "independent":
        nb = n
    elif kind == "diagonal":
        nb = baths or 2
        p.is_diagonal_bath_coupling = True
        p.bath_coupling_op = rng.normal(size=(nb, n))
    elif kind == "full":
        nb = baths or 2
        p.is_full_bath_coupling = True
        V = rng.normal(size=(nb, n, n))
        p.bath_coupling_op = (V + V.transpose(0, 2, 1)) / 2
    else:
        raise ValueError(kind)
    p.num_bath_couplings = nb
    p.gamma = rng.uniform(5.0, 20.0, size=nb)
    p.lambda_ = rng.uniform(10.0, 40.0, size=nb)
    return p


def random_hermitian_state(M: int, n: int, seed: int = 1) -> np.ndarray:
    """(M, N, N) random Hermitian ADOs, node-major interleaved doubles."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(M, n, n)) + 1j * rng.normal(size=(M, n, n))
    A = (A + np.conj(np.transpose(A, (0, 2, 1)))) / 2
    return np.ascontiguousarray(np.transpose(A, (0, 2, 1))).view(np.float64).reshape(-1).copy()


def annealed(p: PhiParameters, t_end: float, seed: int = 0, samples: int = 5, complex_x: bool = False,
             min_field_change: float = 0.01) -> PhiParameters:
    """The same problem with an annealing Hamiltonian: H_X = the off-diagonal
    part of H (times a phase when complex_x), H_Z = its diagonal, seeded field
    samples ramping f_x 1 -> 0 and f_z 0 -> 1 over integration_time = t_end."""
    rng = np.random.default_rng(seed)
    H = np.asarray(p.time_indepenent_hamiltonian, np.complex128)
    off = H - np.diag(np.diag(H))
    if complex_x:
        ph = np.exp(1j * rng.uniform(0, np.pi, size=off.shape))
        off = np.triu(off * ph, 1)
        off = off + off.conj().T
    p.time_indepenent_hamiltonian = None
    p.transverse_hamiltonian = off
    p.longitudinal_hamiltonian = np.diag(np.diag(H)).astype(np.complex128)
    p.transverse_field = np.linspace(1.0, 0.0, samples) + 0.1 * rng.normal(size=samples)
    p.longitudinal_field = np.linspace(0.0, 1.0, samples) + 0.1 * rng.normal(size=samples)
    p.integration_time = t_end
    p.minimum_field_change = min_field_change
    return p


def truncated_problem(full: int = 4, k: int = 3, baths: int = 2, matsubara: int = 2, truncation: int = 3,
                      seed: int = 0, time_local: bool = False) -> PhiParameters:
    """Hilbert-space truncated problem (PHI's HilbertSpaceSize > NumStates):
    a real symmetric full x full Hamiltonian whose lowest k eigenvalues sit
    apart from the rest, full bath coupling operators (real symmetric), a
    full-space initial density matrix; the hierarchy keeps the lowest k
    eigenvectors."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(full, full)))
    e = np.concatenate([np.sort(rng.uniform(-60.0, 60.0, size=k)), np.sort(rng.uniform(250.0, 400.0, size=full - k))])
    H = (Q * e) @ Q.T
    H = (H + H.T) / 2
    V = rng.normal(size=(baths, full, full))
    V = (V + np.transpose(V, (0, 2, 1))) / 2
    A = rng.normal(size=(full, full)) + 1j * rng.normal(size=(full, full))
    rho = A @ np.conj(A.T)
    rho /= np.trace(rho).real
    p = PhiParameters(num_states=k, time_indepenent_hamiltonian=np.asarray(H, np.complex128),
                      num_bath_couplings=baths, num_matsubara_terms=matsubara, hierarchy_truncation_level=truncation,
                      temperature=300.0, is_full_bath_coupling=True, bath_coupling_op=V,
                      initial_density_matrix=rho, hilbert_space_size=full)
    p.gamma = rng.uniform(5.0, 20.0, size=baths)
    p.lambda_ = rng.uniform(10.0, 40.0, size=baths)
    p.use_time_local_truncation = time_local
    return p


def truncated_annealed(full: int = 4, k: int = 2, baths: int = 2, matsubara: int = 2, truncation: int = 3,
                       seed: int = 0, time_local: bool = False, t_end: float = 0.05, samples: int = 5,
                       min_field_change: float = 0.01, mix: float = 0.3) -> PhiParameters:
    """Hilbert-space truncated annealing problem: H_X and H_Z real symmetric
    full x full with their lowest k eigenvalues 190 or more below the rest,
    H_Z's eigenbasis that of H_X turned by exp(mix A) (A random
    antisymmetric), so the kept subspace of H(t) = f_x H_X + f_z H_Z turns
    along the anneal; positive field samples (f_x 1 -> 0.2, f_z 0.2 -> 1 plus
    seeded noise), full bath coupling operators and a full-space initial
    density matrix."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(full, full)))
    A = rng.normal(size=(full, full))
    A = (A - A.T) / 2
    w, U = np.linalg.eigh(1j * mix * A)  # exp(mix A) through the Hermitian i mix A
    Rm = np.real((U * np.exp(-1j * w)) @ U.conj().T)
    def spectrum():
        return np.concatenate([np.sort(rng.uniform(-60.0, 60.0, size=k)),
                               np.sort(rng.uniform(250.0, 400.0, size=full - k))])
    HX = (Q * spectrum()) @ Q.T
    Qz = Q @ Rm
    HZ = (Qz * spectrum()) @ Qz.T
    HX, HZ = (HX + HX.T) / 2, (HZ + HZ.T) / 2
    V = rng.normal(size=(baths, full, full))
    V = (V + np.transpose(V, (0, 2, 1))) / 2
    B = rng.normal(size=(full, full)) + 1j * rng.normal(size=(full, full))
    rho = B @ np.conj(B.T)
    rho /= np.trace(rho).real
    p = PhiParameters(num_states=k, time_indepenent_hamiltonian=None, num_bath_couplings=baths,
                      num_matsubara_terms=matsubara, hierarchy_truncation_level=truncation, temperature=300.0,
                      is_full_bath_coupling=True, bath_coupling_op=V, initial_density_matrix=rho,
                      hilbert_space_size=full)
    p.gamma = rng.uniform(5.0, 20.0, size=baths)
    p.lambda_ = rng.uniform(10.0, 40.0, size=baths)
    p.use_time_local_truncation = time_local
    p.transverse_hamiltonian = np.asarray(HX, np.complex128)
    p.longitudinal_hamiltonian = np.asarray(HZ, np.complex128)
    p.transverse_field = np.linspace(1.0, 0.2, samples) + 0.02 * rng.normal(size=samples)
    p.longitudinal_field = np.linspace(0.2, 1.0, samples) + 0.02 * rng.normal(size=samples)
    p.integration_time = t_end
    p.minimum_field_change = min_field_change
    return p


def reference_truncated_anneal(test: str) -> PhiParameters:
    """The problems of the reference's truncated annealing tests
    (src/hierarchy_integrator_test.cc:569-580, :613-623, :642-655,
    :702-714), as PhiParameters: hbar = kB = 1, T = 2, integration time 1
    (10 for the time-local ones), default annealing fields, start in |0><0|
    of a three-state space.

      vacuum                 two-state sigma_x / sigma_z embedded with a third
                             level at 9.9, one medium bath, one tier
      medium_full_indep      the same H, three medium baths, full couplings
                             |m><m|, three tiers
      weak_full_indep_tl     the same H, three weak baths, |m><m|, three tiers,
                             time-local truncation (RKF45 only)
      weak_full_tl           the 3 x 3 annealing H of
                             SetTruncatedAnnealingHamiltonian(3, 2), two weak
                             baths with couplings (-1)^(m+j+k), three tiers,
                             time-local truncation (RKF45 only)
    """
    F = 3
    HX = np.zeros((F, F), np.complex128)
    HZ = np.zeros((F, F), np.complex128)
    if test == "weak_full_tl":
        for i in range(F):
            HZ[i, i] = 1 + i
            HX[i, i] = -1 - i
            for j in range(i):
                HX[i, j] = HX[j, i] = 1 + i
                HZ[i, j] = HZ[j, i] = -1 - j
    else:
        HX[0, 1] = HX[1, 0] = 1.0
        HZ[0, 0], HZ[1, 1] = 1.0, -1.0
        HX[2, 2] = HZ[2, 2] = 9.9
    baths, medium, tiers, tl = {"vacuum": (1, True, 1, False), "medium_full_indep": (3, True, 3, False),
                                "weak_full_indep_tl": (3, False, 3, True), "weak_full_tl": (2, False, 3, True)}[test]
    rho = np.zeros((F, F), np.complex128)
    rho[0, 0] = 1.0
    p = PhiParameters(num_states=2, time_indepenent_hamiltonian=None, num_bath_couplings=baths,
                      num_matsubara_terms=1, hierarchy_truncation_level=tiers, temperature=2.0,
                      initial_density_matrix=rho, hilbert_space_size=F)
    p.hbar = 1.0
    p.boltzmann_constant = 1.0
    # SetMediumBathParameters / SetWeakBathParameters (:143-161): i/10 and
    # i/1000 are integer divisions there.
    p.gamma = np.array([(0.5 if medium else 1.0) for _ in range(baths)], np.float64)
    p.lambda_ = np.array([(0.5 if medium else 0.01) for _ in range(baths)], np.float64)
    if test != "vacuum":
        V = np.zeros((baths, F, F))
        for m in range(baths):
            if test == "weak_full_tl":
                V[m] = np.fromfunction(lambda j, k: (-1.0) ** (m + j + k), (F, F))
            else:
                V[m, m, m] = 1.0
        p.is_full_bath_coupling = True
        p.bath_coupling_op = V
    p.use_time_local_truncation = tl
    p.transverse_hamiltonian = HX
    p.longitudinal_hamiltonian = HZ
    p.transverse_field = np.array([1.0, 0.0])
    p.longitudinal_field = np.array([0.0, 1.0])
    p.integration_time = 10.0 if tl else 1.0
    p.minimum_field_change = 0.01
    return p
