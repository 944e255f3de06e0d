"""Annealing Hamiltonians (PHI's TransverseHamiltonian / LongitudinalHamiltonian
with their fields) in the oracle, pinned to the reference build (CPU).

tests/golden/ref_anneal.json holds, per case, rho_0 printed with %.17g by the
reference build and, for small hierarchies, the whole final state from its
restart file.  PHI sets H = f_x(t/T) H_X + f_z(t/T) H_Z before every stage
(UpdateTimeDependentHamiltonian, hierarchy_integrator.cc:1618-1673), f_x and
f_z its cubic splines (cubic_spline.cc), and only when a field moved by the
minimum relative change.
"""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Batch, Hierarchy

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_anneal.json")))["cases"]


def build(case):
    b = case["builder"]
    if b.startswith("config:"):
        p = getattr(configs, b.split(":", 1)[1])(**case["kwargs"])
    else:
        p = getattr(cases, b)(**case["kwargs"])
    p = cases.annealed(p, case["t_end"], **case["anneal"])
    p.use_time_local_truncation = case["time_local"]
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def run_oracle(o, case):
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    return s


def to_complex(v):
    return np.array([complex(a, b) for a, b in v])


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_oracle_rho0_matches_reference(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case)
    ref = to_complex(case["rho0_colmajor"]).reshape(p.num_states, p.num_states).T
    assert np.abs(o.rho0(s) - ref).max() <= 1e-13


@pytest.mark.parametrize("case", [c for c in FIX if "state_6_digits" in c],
                         ids=[c["id"] for c in FIX if "state_6_digits" in c])
def test_oracle_state_matches_reference_restart_file(case):
    p = build(case)
    o = O.Oracle(p)
    s = run_oracle(o, case).view(np.complex128)
    ref = to_complex(case["state_6_digits"])
    np.testing.assert_allclose(s, ref, rtol=6e-6, atol=1e-300)


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_annealing_changes_the_result(case):
    """Against the static Hamiltonian at the end of the ramp, f_x(1) H_X +
    f_z(1) H_Z: the annealed run differs by far more than FP64 noise."""
    p = build(case)
    fx = O.Oracle(p)
    x1 = float(np.asarray(p.transverse_field)[-1])
    z1 = float(np.asarray(p.longitudinal_field)[-1])
    q = build(case)
    q.time_indepenent_hamiltonian = x1 * q.transverse_hamiltonian + z1 * q.longitudinal_hamiltonian
    q.transverse_hamiltonian = None
    o2 = O.Oracle(q)
    s2 = run_oracle(o2, case)
    ref = to_complex(case["rho0_colmajor"]).reshape(p.num_states, p.num_states).T
    assert np.abs(o2.rho0(s2) - ref).max() > 1e-7
    del fx


def test_hamiltonian_follows_the_fields():
    """With no gate the last update is at the end of the ramp (RK4 stage 3 of
    the last step, t = T), where PHI's spline returns the last samples: H is
    f_x(1) H_X + f_z(1) H_Z."""
    p = cases.annealed(cases.random_problem("independent", n=3, matsubara=2, truncation=2, seed=2), 0.05,
                       seed=1, min_field_change=0.0)
    o = O.Oracle(p)
    o.rk4(o.initial_state(), 0.001, 0.05)
    x1 = float(np.asarray(p.transverse_field)[-1])
    z1 = float(np.asarray(p.longitudinal_field)[-1])
    want = x1 * p.transverse_hamiltonian + z1 * p.longitudinal_hamiltonian
    assert np.abs(o.hamiltonian() - want).max() <= 1e-12 * np.abs(want).max()


def test_batch_refuses_annealing():
    p = cases.annealed(configs.frenkel7(depth=2), 0.05, seed=1)
    with pytest.raises(capi.PhiError, match="annealing"):
        Batch([p])
