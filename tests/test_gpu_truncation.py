"""Hilbert-space truncation on the GPU: rho_0 in the full space (V rho_0
V^+, phi_gpu_get_rho0_full) against the reference built in BLAS mode
(tests/golden/ref_truncation.json, %.17g), FP64 within 1e-10; the basis is
the library's own Jacobi eigenbasis, whose phases and order need not match
LAPACK's."""
import json
import os

import numpy as np
import pytest

import cases
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_truncation.json")))["cases"]
TOL = 1e-10


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_truncated_rho0_matches_reference(case):
    p = cases.truncated_problem(**case["kwargs"])
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    F = p.hilbert_space_size
    with Hierarchy(p) as h:
        assert h.n == p.num_states
        if case["method"] == "rk4":
            h.rk4(case["timestep"], case["t_end"])
        else:
            h.rkf45(case["timestep"], case["t_end"], 1e-6, 1e-6)
        got = h.rho0_full()
    v = np.array(case["rho0_colmajor"])
    ref = (v[:, 0] + 1j * v[:, 1]).reshape(F, F).T
    assert got.shape == (F, F)
    assert np.abs(got - ref).max() <= TOL
