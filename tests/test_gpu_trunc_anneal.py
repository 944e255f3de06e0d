"""Hilbert-space truncation of an annealing Hamiltonian on the GPU.  Before
every stage the device re-diagonalises H(t) (one warp, cyclic Jacobi),
truncates it into the lowest k eigenvectors, rotates the full bath operators
and every live ADO (anneal_rotate_kernel), as PHI's UpdateWith / Truncate /
Rotate do (hilbert_space_truncator.cc:34-113, hierarchy_integrator.cc
:1618-1673); rho_0 comes back in the full space with the current basis.

Against rho_0 of the reference built in BLAS mode
(tests/golden/ref_trunc_anneal.json): FP64 within 1e-10.  With time-local
truncation PHI does not rotate its Q matrices, so its result depends on the
signs LAPACK gives the eigenvectors (they flip between updates); those cases
are held to the oracle, which signs the eigenvectors the same way as the
device, within 1e-10, and to the reference within its own RKF45 test
tolerance of 1e-3."""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_trunc_anneal.json")))["cases"]
TOL = 1e-10
TL_TOL = 1e-3


def _rho(case):
    v = np.array(case["rho0_colmajor"])
    F = int(round(len(v) ** 0.5))
    return (v[:, 0] + 1j * v[:, 1]).reshape(F, F).T


def _problem(case):
    p = getattr(cases, case["builder"])(**case["kwargs"])
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def _run_gpu(h, case, p):
    if case["method"] == "rk4":
        h.rk4(case["timestep"], case["t_end"])
    else:
        h.rkf45(case["timestep"], case["t_end"], p.rkf45_tolerance, p.rkf45_minimum_timestep)
    return h.rho0_full()


def _run_oracle(case, p):
    o = O.Oracle(p)
    if case["method"] == "rk4":
        s, *_ = o.rk4(o.initial_state(), case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(o.initial_state(), case["timestep"], case["t_end"], p.rkf45_tolerance,
                       p.rkf45_minimum_timestep)
    return o.rho0_full(s)


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_truncated_annealing_matches_reference(case):
    p = _problem(case)
    with Hierarchy(p) as h:
        assert h.n == p.num_states
        got = _run_gpu(h, case, p)
    ref = _rho(case)
    assert got.shape == ref.shape
    if p.use_time_local_truncation:
        assert np.abs(got - _run_oracle(case, p)).max() <= TOL
        assert np.abs(got - ref).max() <= TL_TOL
    else:
        assert np.abs(got - ref).max() <= TOL


def test_truncated_annealing_chunks_and_reset():
    """RKF45 in chunks of attempted steps equals one call (the basis, H and
    the update state carry over); set_state puts the basis, H and the bath
    operators back to their initial values, so a second run from rho(0)
    repeats the first."""
    case = next(c for c in FIX if c["id"] == "ta_f4_k2_t3/rkf45")
    p = _problem(case)
    tol, mindt, t_end = p.rkf45_tolerance, p.rkf45_minimum_timestep, case["t_end"]
    with Hierarchy(p) as h:
        s0 = h.get_state()
        st = h.rkf45(case["timestep"], t_end, tol, mindt)
        one = h.rho0_full()
        h.set_state(s0)
        h.time = 0.0
        done = h.rkf45_advance(case["timestep"], t_end, tol, mindt, 7)["steps"]
        while h.time < t_end:
            done += h.rkf45_advance(0.0, t_end, tol, mindt, 5)["steps"]
        two = h.rho0_full()
    assert done == st["steps"]
    assert np.abs(two - one).max() <= 1e-14
    assert np.abs(one - _rho(case)).max() <= TOL


def test_truncated_annealing_refuses_state_files(tmp_path):
    case = next(c for c in FIX if c["id"] == "ta_f4_k2_t3/rk4")
    p = _problem(case)
    with Hierarchy(p) as h:
        with pytest.raises(capi.PhiError) as e:
            h.save_state(str(tmp_path / "s.bin"))
        assert e.value.code == capi.PHI_E_INVALID
