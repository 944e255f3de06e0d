"""Restart files on the host (no GPU): PHI's layout (restart_helper.cc:30-84)
read from a file the reference build wrote at the end of an RK4 run
(tests/golden/ref_restart_indep_n3.txt), checked against the run's own
rho_0 and against the oracle's whole hierarchy at that time (which also pins
the node order of the file); exact write/read round trip; malformed files."""
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_restart_indep_n3.txt")
META = json.load(open(os.path.join(HERE, "golden", "ref_restart_indep_n3.json")))


def _problem():
    return getattr(cases, META["builder"])(**META["kwargs"])


def _dims(p):
    T = int(p.num_bath_couplings) * int(p.num_matsubara_terms)
    return int(p.num_states), configs.hierarchy_nodes(T, int(p.hierarchy_truncation_level) - 1)


def test_reads_reference_restart_file():
    p = _problem()
    n, M = _dims(p)
    st, t, dt = capi.restart_read(FIX, n, M)
    assert t == pytest.approx(META["t_end"]) and dt == pytest.approx(META["timestep"])
    rho_ref = np.array([complex(a, b) for a, b in META["rho0_colmajor"]])
    rho = st[:2 * n * n].view(np.complex128)
    # the file holds 6 significant digits
    assert np.abs(rho - rho_ref).max() <= 5e-6 * np.abs(rho_ref).max()


def test_reference_restart_matches_oracle_hierarchy():
    p = _problem()
    n, M = _dims(p)
    st, _, _ = capi.restart_read(FIX, n, M)
    o = O.Oracle(p)
    s, steps, _, _ = o.rk4(o.initial_state(), META["timestep"], META["t_end"])
    assert steps == 10
    z, w = st.view(np.complex128), s.view(np.complex128)
    assert np.abs(z - w).max() <= 1e-5 * np.abs(w).max()


def test_write_read_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(0)
    n, M = 4, 37
    st = rng.normal(size=2 * M * n * n) * 10.0 ** rng.integers(-12, 3, size=2 * M * n * n)
    path = tmp_path / "r.txt"
    capi.restart_write(path, n, M, st, 0.123456789012345, 1e-3)
    got, t, dt = capi.restart_read(path, n, M)
    assert np.array_equal(got, st) and t == 0.123456789012345 and dt == 1e-3


@pytest.mark.parametrize("edit", ["truncate", "extra", "garbage"])
def test_malformed_restart_files_are_rejected(tmp_path, edit):
    p = _problem()
    n, M = _dims(p)
    text = open(FIX).read()
    if edit == "truncate":
        text = text[: len(text) // 2]
    elif edit == "extra":
        text += "(1,2)\n"
    else:
        text = "0.01\nabc\n"
    path = tmp_path / "bad.txt"
    path.write_text(text)
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        capi.restart_read(path, n, M)


def test_restart_error_text_is_per_thread(tmp_path):
    """A failed restart call on one thread leaves another thread's error text alone."""
    import ctypes
    import threading

    lib = capi.load()

    def last_error():
        buf = ctypes.create_string_buffer(1024)
        assert lib.phi_restart_last_error(buf, 1024) == 0
        return buf.value.decode()

    n, M = _dims(_problem())
    missing = tmp_path / "missing.txt"
    with pytest.raises(capi.PhiError):
        capi.restart_read(missing, n, M)
    mine = last_error()
    assert mine
    seen = {}

    def other():
        seen["before"] = last_error()
        with pytest.raises(capi.PhiError):
            capi.restart_read(tmp_path / "also_missing.txt", n, M)
        seen["after"] = last_error()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen["before"] == ""
    assert "also_missing" in seen["after"] or seen["after"] != mine
    assert last_error() == mine
