"""Restart files of time-local runs (CPU): PHI's layout puts the stored
Q_{m,k} after the nodes (restart_helper.cc:40-50).  Pinned by a file the
reference build wrote (tests/golden/ref_restart_timelocal_n3.txt; its
step-size line set to the run's timestep because PHI writes the clamped 0)."""
import ctypes
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_restart_timelocal_n3.txt")
META = json.load(open(os.path.join(HERE, "golden", "ref_restart_timelocal_n3.json")))


def _problem():
    p = getattr(cases, META["builder"])(**META["kwargs"])
    p.use_time_local_truncation = True
    p.fix_incompatible_combinations("rkf45")
    return p


def _read_ex(path, n, M, nmat):
    lib = capi.load()
    st = np.zeros(2 * M * n * n)
    q = np.zeros(max(1, 2 * nmat * n * n))
    t, dt = ctypes.c_double(), ctypes.c_double()
    rc = lib.phi_restart_read_file_ex(str(path).encode(), n, M, st.ctypes.data, ctypes.byref(t), ctypes.byref(dt),
                                      q.ctypes.data, nmat)
    return rc, st, q[:2 * nmat * n * n], t.value, dt.value


def test_reads_reference_time_local_restart_file():
    p = _problem()
    n, M, nmat = p.num_states, O.node_count(p.num_bath_couplings * p.num_matsubara_terms,
                                            p.hierarchy_truncation_level), META["num_matrices"]
    rc, st, q, t, dt = _read_ex(FIX, n, M, nmat)
    assert rc == capi.PHI_OK
    assert (t, dt) == (META["t1"], META["timestep"])
    # Without the matrices the file has values left over, which is an error.
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        capi.restart_read(FIX, n, M)
    # One matrix too many: the file ends early.
    rc2, *_ = _read_ex(FIX, n, M, nmat + 1)
    assert rc2 == capi.PHI_E_INVALID


def test_reference_matrices_match_oracle():
    """The file's Q_{m,k} are the stored copies after the last accepted RKF45
    step; summed over k they are the oracle's Q_m at t1 (6 digits)."""
    p = _problem()
    o = O.Oracle(p)
    s, _ = o.rkf45(o.initial_state(), META["timestep"], META["t1"], 1e-6, 1e-6)
    n, nb, K1 = p.num_states, p.num_bath_couplings, p.num_matsubara_terms
    rc, st, q, _, _ = _read_ex(FIX, n, o.M, nb * K1)
    assert rc == capi.PHI_OK
    q = q.view(np.complex128).reshape(nb, K1, n * n).sum(axis=1)
    want = o.time_local().reshape(nb, n * n)  # already in storage (column-major) order per bath
    assert np.abs(q - want).max() <= 2e-5 * np.abs(want).max()
    np.testing.assert_allclose(st.view(np.complex128), s.view(np.complex128), rtol=6e-6, atol=1e-300)


def test_ex_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    n, M, nmat = 3, 5, 4
    st = rng.normal(size=2 * M * n * n)
    q = rng.normal(size=2 * nmat * n * n)
    lib = capi.load()
    path = tmp_path / "r.txt"
    assert lib.phi_restart_write_file_ex(str(path).encode(), n, M, st.ctypes.data, 0.25, 1e-3, q.ctypes.data,
                                         nmat) == capi.PHI_OK
    rc, st2, q2, t, dt = _read_ex(path, n, M, nmat)
    assert rc == capi.PHI_OK and (t, dt) == (0.25, 1e-3)
    assert np.array_equal(st, st2) and np.array_equal(q, q2)
    assert len(path.read_text().splitlines()) == 2 + M + nmat
