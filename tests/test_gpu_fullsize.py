"""Parity at the benchmarked sizes: rho_0 of the device integrators against
rho_0 printed with %.17g by the reference build for the same full-size
configurations (tests/golden/ref_fullsize.json, written by
tests/golden/make_golden.py fullsize):

  frenkel7 L = 6 (38,760 nodes of 7x7)  RKF45 tol 1e-6 to 1 ps, RK4 300 steps
  ring24   L = 4 (20,475 nodes of 24x24) RKF45 tol 1e-6 to 500 fs
  chain4   L = 8 (125,970 nodes of 4x4)  RK4 100 steps

FP64 must match within 1e-10 max-abs on rho_0; the mixed mode (complex64
stages, FP64 state and control) within 1e-6 of the reference, the stated
tolerance of that mode.  RKF45 runs must also take the reference's number of
attempted and accepted steps."""
import json
import os

import numpy as np
import pytest

from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = json.load(open(os.path.join(HERE, "golden", "ref_fullsize.json")))
CASES = {c["id"]: c for c in FIXTURE["cases"]}
FP64_TOL = 1e-10
MIXED_TOL = 1e-6


def _rho(c):
    v = np.array(c["rho0_colmajor"])
    n = int(round(len(v) ** 0.5))
    return (v[:, 0] + 1j * v[:, 1]).reshape(n, n).T


def _run(c, precision):
    p = getattr(configs, c["builder"])(**c["kwargs"])
    assert int(p.seed) == c["seed"]
    p.fix_incompatible_combinations(c["method"])
    with Hierarchy(p, precision=precision) as h:
        if c["method"] == "rk4":
            steps, _, _ = h.rk4(c["timestep"], c["t_end"])
            st = {"steps": steps, "accepted": None}
        else:
            st = h.rkf45(c["timestep"], c["t_end"], c["rkf45_tolerance"], c["rkf45_mindt"])
        return h.rho0(), st


@pytest.mark.parametrize("cid", sorted(CASES))
@pytest.mark.parametrize("precision", [capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED], ids=["fp64", "mixed"])
def test_fullsize_rho0_matches_reference(cid, precision):
    c = CASES[cid]
    rho, st = _run(c, precision)
    ref = _rho(c)
    err = float(np.abs(rho - ref).max())
    tol = FP64_TOL if precision == capi.PHI_PREC_FP64 else MIXED_TOL
    print(f"{cid} {'fp64' if precision == capi.PHI_PREC_FP64 else 'mixed'}: rho_0 max-abs {err:.3e}, "
          f"steps {st['steps']} (reference {c['steps']})")
    assert err <= tol
    if c["method"] == "rkf45" and precision == capi.PHI_PREC_FP64:
        assert st["steps"] == c["steps"] and st["accepted"] == c["accepted_steps"]
    else:
        assert st["steps"] > 0
