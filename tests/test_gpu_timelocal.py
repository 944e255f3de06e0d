"""Time-local truncation (PHI's TimeLocal) on the GPU: the tiled kernel
(identity site map, K+1 <= 3) and the generic kernel (K+1 > 3), RK4 and
RKF45, against the reference build's rho_0 (tests/golden/ref_timelocal.json)
and the oracle (whole state and the matrices Q_m).

The deepest tier adds -sum_m [V_m, Q_m rho - rho Q_m^+] in place of its next
terms (hierarchy_updater.cc:171-190); the Q_{m,k} advance along the stage
times, with RKF45's restore before stage 5 and store/restore on
accept/reject (hierarchy_integrator.cc:1675-1733, :2028-2247, :2388, :2479).
"""
import ctypes
import json
import os

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_timelocal.json")))["cases"]
FP64_TOL = 1e-10    # max-abs error relative to the largest element
RHO0_TOL = 1e-6     # mixed precision against FP64


def build(case):
    b = case["builder"]
    if b.startswith("config:"):
        p = getattr(configs, b.split(":", 1)[1])(**case["kwargs"])
    else:
        p = getattr(cases, b)(**case["kwargs"])
    p.use_time_local_truncation = True
    p.filter_tolerance = case["filter_tolerance"]
    if case["method"] == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def run_gpu(h, case):
    if case["method"] == "rk4":
        h.rk4(case["timestep"], case["t_end"])
    else:
        h.rkf45(case["timestep"], case["t_end"], 1e-6, 1e-6)


def run_oracle(o, case):
    s0 = o.initial_state()
    if case["method"] == "rk4":
        s, *_ = o.rk4(s0, case["timestep"], case["t_end"])
    else:
        s, _ = o.rkf45(s0, case["timestep"], case["t_end"], 1e-6, 1e-6)
    return s


GENERIC = [
    {"id": "generic_n3_k4_t3/rk4", "builder": "random_problem",
     "kwargs": dict(kind="independent", n=3, matsubara=4, truncation=3, seed=4),
     "method": "rk4", "timestep": 0.001, "t_end": 0.05, "filter_tolerance": 0.0},
    {"id": "generic_n3_k4_t3/rkf45", "builder": "random_problem",
     "kwargs": dict(kind="independent", n=3, matsubara=4, truncation=3, seed=4),
     "method": "rkf45", "timestep": 0.001, "t_end": 0.05, "filter_tolerance": 0.0},
    {"id": "generic_n3_k4_t1/rkf45", "builder": "random_problem",
     "kwargs": dict(kind="independent", n=3, matsubara=4, truncation=1, seed=4),
     "method": "rkf45", "timestep": 0.001, "t_end": 0.05, "filter_tolerance": 0.0},
]
ALL = FIX + GENERIC


@pytest.mark.parametrize("case", FIX, ids=[c["id"] for c in FIX])
def test_rho0_matches_reference(case):
    p = build(case)
    with Hierarchy(p) as h:
        run_gpu(h, case)
        rho = h.rho0()
    ref = np.array([complex(a, b) for a, b in case["rho0_colmajor"]]).reshape(p.num_states, p.num_states).T
    assert np.abs(rho - ref).max() <= FP64_TOL * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("case", ALL, ids=[c["id"] for c in ALL])
def test_state_and_matrices_match_oracle(case):
    p = build(case)
    o = O.Oracle(p)
    ref = run_oracle(o, case)
    q_ref = o.time_local()
    with Hierarchy(p) as h:
        run_gpu(h, case)
        got = h.get_state()
        q = h.time_local()
    assert np.abs(q_ref).max() > 0
    assert np.abs(q - q_ref).max() <= FP64_TOL * np.abs(q_ref).max()
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()


def test_mixed_precision_time_local_rho0():
    p = configs.frenkel7(depth=2)
    p.use_time_local_truncation = True
    p.fix_incompatible_combinations("rkf45")
    out = {}
    for prec in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        with Hierarchy(p, precision=prec) as h:
            h.rkf45(0.001, 0.1, 1e-6, 1e-6)
            out[prec] = h.rho0()
    assert np.abs(out[capi.PHI_PREC_MIXED] - out[capi.PHI_PREC_FP64]).max() <= RHO0_TOL


def _tl_problem():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=2)
    p.use_time_local_truncation = True
    return p


def test_chunked_rk4_carries_matrices():
    """13 then 37 steps (graph path and tail) equal one 50-step call."""
    p = _tl_problem()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        one, q1 = h.get_state(), h.time_local()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.013)
        h.rk4(0.001, 0.05)
        two, q2 = h.get_state(), h.time_local()
    assert np.abs(q1 - q2).max() <= 1e-14 * np.abs(q1).max()
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_chunked_rkf45_carries_matrices():
    p = _tl_problem()
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p) as h:
        st = h.rkf45(0.001, 0.05, 1e-6, 1e-6)
        one, q1 = h.get_state(), h.time_local()
    with Hierarchy(p) as h:
        a = h.rkf45_advance(0.001, 0.05, 1e-6, 1e-6, 7)
        done = a["steps"]
        while h.time < 0.05:
            done += h.rkf45_advance(0.0, 0.05, 1e-6, 1e-6, 5)["steps"]
        two, q2 = h.get_state(), h.time_local()
    assert done == st["steps"]
    assert np.abs(q1 - q2).max() <= 1e-14 * np.abs(q1).max()
    assert np.abs(one - two).max() <= 1e-14 * np.abs(one).max()


def test_noalloc_step_advances_matrices():
    """The no-allocation RK4 step runs the same updates as phi_gpu_rk4."""
    import torch
    p = _tl_problem()
    dt = 0.001
    with Hierarchy(p) as h:
        h.rk4(dt, 2 * dt)
        ref, q_ref = h.get_state(), h.time_local()
    with Hierarchy(p) as h:
        a = torch.tensor(h.get_state(), dtype=torch.float64, device="cuda")
        b, c = torch.empty_like(a), torch.empty_like(a)
        stream = torch.cuda.current_stream()
        for src, dst in ((a, b), (b, c)):
            capi.check(h.lib.phi_gpu_rk4_step_noalloc(h.ctx, ctypes.c_void_p(src.data_ptr()),
                                                      ctypes.c_void_p(dst.data_ptr()), dt,
                                                      ctypes.c_void_p(stream.cuda_stream)), h.ctx)
        torch.cuda.synchronize()
        got, q = c.cpu().numpy(), h.time_local()
    assert np.abs(q - q_ref).max() <= 1e-14 * np.abs(q_ref).max()
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()


def test_set_state_resets_matrices_and_refusals(tmp_path):
    p = _tl_problem()
    with Hierarchy(p) as h:
        s0 = h.get_state()
        h.rk4(0.001, 0.01)
        assert np.abs(h.time_local()).max() > 0
        h.set_state(s0)
        assert np.abs(h.time_local()).max() == 0
        # PHI turns time-local truncation off for steady states.
        with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
            h.steady_state(tol=1e-10)


def test_parameter_file_time_local(tmp_path):
    p = _tl_problem()
    path = tmp_path / "params.txt"
    path.write_text(O.param_file_text(p, timestep=0.001, t_end=0.05))
    with Hierarchy.from_file(str(path), "rk4") as h:
        h.rk4(0.001, 0.05)
        a = h.get_state()
    with Hierarchy(p) as h:
        h.rk4(0.001, 0.05)
        b = h.get_state()
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


RST = os.path.join(HERE, "golden", "ref_restart_timelocal_n3.txt")
RST_META = json.load(open(os.path.join(HERE, "golden", "ref_restart_timelocal_n3.json")))


def _rst_problem():
    p = getattr(cases, RST_META["builder"])(**RST_META["kwargs"])
    p.use_time_local_truncation = True
    p.fix_incompatible_combinations("rkf45")
    return p


def test_continue_from_reference_restart_file():
    """Read the reference's time-local restart file (nodes and stored Q_{m,k},
    restored as PHI's Initialize does) and continue RKF45 to t2: rho_0 equals
    the reference restarted from the same file."""
    p = _rst_problem()
    with Hierarchy(p) as h:
        dt = h.read_restart(RST)
        assert h.time == RST_META["t1"] and dt == RST_META["timestep"]
        n, nb, K1 = p.num_states, p.num_bath_couplings, p.num_matsubara_terms
        st = np.zeros(2 * h.num_nodes * n * n)
        q = np.zeros(2 * nb * K1 * n * n)
        t, d = ctypes.c_double(), ctypes.c_double()
        assert h.lib.phi_restart_read_file_ex(RST.encode(), n, h.num_nodes, st.ctypes.data, ctypes.byref(t),
                                              ctypes.byref(d), q.ctypes.data, nb * K1) == capi.PHI_OK
        q_sum = q.view(np.complex128).reshape(nb, K1, n, n).sum(axis=1)
        assert np.abs(h.time_local() - q_sum).max() <= 1e-15 * np.abs(q_sum).max()
        h.rkf45(dt, RST_META["t2"], 1e-6, 1e-6)
        rho = h.rho0()
    ref = np.array([complex(a, b) for a, b in RST_META["rho0_t2_colmajor"]]).reshape(n, n).T
    assert np.abs(rho - ref).max() <= FP64_TOL * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("fmt", ["text", "binary"])
def test_restart_round_trip_keeps_matrices(tmp_path, fmt):
    """A time-local context's restart (17 digits) or state file carries the
    stored Q_{m,k}; a context loaded from it continues exactly as the one
    that wrote it (after an accepted RKF45 step the stored and the current
    matrices agree)."""
    p = _rst_problem()
    path = str(tmp_path / ("r.txt" if fmt == "text" else "r.bin"))
    with Hierarchy(p) as a:
        st = a.rkf45(0.001, 0.02, 1e-6, 1e-6)
        (a.write_restart if fmt == "text" else a.save_state)(path, 0.001)
        qa = a.time_local()
        a.rkf45(0.001, 0.04, 1e-6, 1e-6)
        end_a = a.get_state()
    with Hierarchy(p) as b:
        (b.read_restart if fmt == "text" else b.load_state)(path)
        assert np.abs(b.time_local() - qa).max() <= 1e-15 * np.abs(qa).max()
        b.rkf45(0.001, 0.04, 1e-6, 1e-6)
        end_b = b.get_state()
    assert st["accepted"] > 0
    assert np.abs(end_a - end_b).max() <= 1e-13 * np.abs(end_a).max()
