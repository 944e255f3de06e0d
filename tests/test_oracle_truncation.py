"""Hilbert-space truncation (PHI's HilbertSpaceSize > NumStates), CPU side.

tests/golden/ref_truncation.json holds rho_0 in the full space, printed with
%.17g by the reference built in BLAS mode (its -DNOBLAS loops flip signs in
the truncator).  PHI keeps the lowest k eigenvectors V of the full
Hamiltonian and runs the hierarchy on V^+ H V, V^+ rho(0) V and V^+ B_b V
(hilbert_space_truncator.cc:34-134; hierarchy_integrator.cc:915-918,
:1073-1075, :1179-1186), returning V rho_0 V^+ (:177-191).  Restated here
with numpy's eigenbasis and the oracle's k-dimensional integrator, the
result must equal the reference's within 1e-10: it does not depend on the
phases or order of the kept eigenvectors."""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi
from phi_b200.heom import Hierarchy, PhiParameters

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_truncation.json")))["cases"]
TOL = 1e-10


def _rho(case, n):
    v = np.array(case["rho0_colmajor"])
    return (v[:, 0] + 1j * v[:, 1]).reshape(n, n).T


def truncated_restatement(p):
    """The k-dimensional problem of a truncated one, and its basis V."""
    F, k = p.hilbert_space_size, p.num_states
    w, U = np.linalg.eigh(np.asarray(p.time_indepenent_hamiltonian).real)
    V = U[:, :k]
    q = PhiParameters(num_states=k, time_indepenent_hamiltonian=(V.T @ p.time_indepenent_hamiltonian @ V),
                      num_bath_couplings=p.num_bath_couplings, num_matsubara_terms=p.num_matsubara_terms,
                      hierarchy_truncation_level=p.hierarchy_truncation_level, temperature=p.temperature,
                      is_full_bath_coupling=True,
                      bath_coupling_op=np.stack([V.T @ b @ V for b in np.asarray(p.bath_coupling_op)]),
                      initial_density_matrix=V.T @ p.initial_density_matrix @ V,
                      is_rho_normalized=p.is_rho_normalized)
    q.gamma, q.lambda_ = p.gamma, p.lambda_
    q.use_time_local_truncation = p.use_time_local_truncation
    return q, V


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_restatement_matches_reference_truncation(case):
    p = cases.truncated_problem(**case["kwargs"])
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    q, V = truncated_restatement(p)
    o = O.Oracle(q)
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    rho_k = o.rho0(s)
    got = V @ rho_k @ V.T
    ref = _rho(case, p.hilbert_space_size)
    assert np.abs(got - ref).max() <= TOL


def test_truncation_scope_checks_need_no_gpu():
    p = cases.truncated_problem(full=4, k=3, baths=2, matsubara=1, truncation=3, seed=0)
    p.is_full_bath_coupling = False
    p.bath_coupling_op = None  # independent baths with more than one tier
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy(p)
    p = cases.truncated_problem(full=4, k=3, baths=2, matsubara=1, truncation=3, seed=0)
    H = np.array(p.time_indepenent_hamiltonian)
    H[0, 1] += 1j
    H[1, 0] -= 1j  # complex Hermitian: not built
    p.time_indepenent_hamiltonian = H
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy(p)
