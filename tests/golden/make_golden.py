"""Generates the golden fixtures under tests/golden/ from the reference.

Run in a container that has the reference tree and the reference build
(oracle/_ref/ref_driver, from `make -C oracle`):

    python tests/golden/make_golden.py /root/reference

Outputs (committed; the GPU host has no reference tree):
  reference_tests.json  rho_0 vectors hard-coded in the reference's own tests
                        (src/hierarchy_integrator_test.cc), read as text
  ref_outputs.json      rho_0 printed with %.17g by the reference build for
                        the problems listed in CASES (builder + arguments)
  ref_order.json        node order of the reference's ConstructI for a set of
                        (terms, truncation) pairs
  ref_output_indep_n3_rk4.txt / .json
                        the output file the reference's `phi` writes for an
                        RK4 run (PrepareForOutput + dynamics rows + closing
                        lines), for the output-file layout
  ref_restart_indep_n3.txt / .json
                        a restart file written by the reference build
                        (RestartFile, RestartOutputTimeSecs; restart_helper.cc
                        :30-53) at the end of an RK4 run, with the run's
                        parameters and its rho_0 printed with %.17g

  ref_filter.json       adaptive hierarchy filtering (FilterTolerance): per
                        case, rho_0 printed with %.17g by the reference
                        build and, for hierarchies of at most 100 nodes, the
                        whole final state from the restart file the same run
                        wrote (PHI prints it with 6 significant digits)

    python tests/golden/make_golden.py /root/reference restart   # restart fixture only
    python tests/golden/make_golden.py /root/reference output    # output-file fixture only
  ref_timelocal.json    time-local truncation (TimeLocal=1): per case, rho_0
                        with %.17g, for small hierarchies the whole final
                        state from the restart file, and for RKF45 the sums
                        over k of the stored Q_{m,k} the restart file ends
                        with (RK4 never stores them: PHI writes zeros there)

    python tests/golden/make_golden.py /root/reference filter    # filtering fixture only
  ref_anneal.json       annealing Hamiltonians (TransverseHamiltonian /
                        LongitudinalHamiltonian and their fields): per case,
                        rho_0 with %.17g and, for small hierarchies, the whole
                        final state from the restart file (the reference build
                        runs them with its LAPACK shim's tridiagonal solve)

    python tests/golden/make_golden.py /root/reference timelocal # time-local fixture only
  ref_restart_timelocal_n3.txt / .json
                        a restart file the reference build wrote at t1 of an
                        RKF45 time-local run (nodes, then the stored Q_{m,k}),
                        and rho_0 (%.17g) of the reference restarted from it
                        (RestartInput) to t2.  PHI writes the step size after
                        its last-step clamp, 0, and a run restarted with it
                        never advances, so the step-size line is replaced by
                        the run's timestep before the restart

    python tests/golden/make_golden.py /root/reference anneal    # annealing fixture only
    python tests/golden/make_golden.py /root/reference restart_tl # time-local restart fixture only
  ref_trunc_anneal.json Hilbert-space truncation of annealing Hamiltonians,
                        rho_0 (F x F, %.17g) from the reference built in BLAS
                        mode (oracle/_ref_blas): seeded problems and the
                        problems of the reference's truncated annealing tests

    python tests/golden/make_golden.py /root/reference trunc_anneal
"""
from __future__ import annotations

import json
import os
import re
import tempfile
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
from phi_b200 import configs  # noqa: E402
import cases  # noqa: E402

# (case id, builder, builder kwargs, method, run kwargs)
CASES = []
for name in cases.REFERENCE_CASES:
    for method in ("rk4", "rkf45"):
        CASES.append((f"{name}/{method}", "reference_fixture_case", {"name": name}, method, {}))
for kind in ("independent", "diagonal", "full"):
    for method in ("rk4", "rkf45"):
        for seed, (n, K1, tr) in enumerate([(3, 2, 3), (4, 1, 4), (2, 3, 3)]):
            CASES.append((f"random_{kind}_{n}_{K1}_{tr}/{method}", "random_problem",
                          {"kind": kind, "n": n, "matsubara": K1, "truncation": tr, "seed": seed,
                           "complex_h": seed == 1},
                          method, {"timestep": 0.001, "t_end": 0.05}))
CASES.append(("random_independent_unnormalized/rk4", "random_problem",
              {"kind": "independent", "n": 3, "matsubara": 2, "truncation": 3, "seed": 5,
               "normalized": False}, "rk4", {"timestep": 0.001, "t_end": 0.05}))
CASES.append(("spin_boson_L10/rk4", "config:spin_boson", {}, "rk4",
              {"timestep": 0.001, "t_end": 2.0}))
CASES.append(("spin_boson_L10_short/rkf45", "config:spin_boson", {}, "rkf45",
              {"timestep": 0.001, "t_end": 0.2}))
CASES.append(("frenkel7_L3/rkf45", "config:frenkel7", {"depth": 3}, "rkf45",
              {"timestep": 0.001, "t_end": 0.05}))
CASES.append(("frenkel7_L3/rk4", "config:frenkel7", {"depth": 3}, "rk4",
              {"timestep": 0.001, "t_end": 0.05}))
CASES.append(("chain4_L4/rk4", "config:chain4", {"depth": 4}, "rk4",
              {"timestep": 0.001, "t_end": 0.05}))
CASES.append(("ring24_L2/rk4", "config:ring24", {"depth": 2}, "rk4",
              {"timestep": 0.001, "t_end": 0.01}))

ORDERS = [(1, 5), (2, 4), (3, 5), (5, 4), (7, 3), (6, 5), (12, 3), (14, 4), (24, 3)]


def build(builder: str, kw: dict):
    if builder.startswith("config:"):
        return getattr(configs, builder.split(":", 1)[1])(**kw)
    return getattr(cases, builder)(**kw)


def parse_reference_tests(ref_root: str) -> dict:
    text = open(os.path.join(ref_root, "src", "hierarchy_integrator_test.cc")).read()
    keys = {k for k, _ in cases.REFERENCE_CASES.values()}
    out = {}
    for key in sorted(keys):
        m = re.search(r"const Complex %s\[\] = \{(.*?)\};" % key, text, re.S)
        vals = []
        for c in re.findall(r"Complex\(([^)]*)\)", m.group(1)):
            parts = [float(x) for x in c.split(",")]
            vals.append([parts[0], parts[1] if len(parts) > 1 else 0.0])
        out[key] = vals  # storage (column-major) order, as the test lists them
    return out


RESTART_CASE = ("random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=3), 0.001, 0.01)


def make_restart_fixture():
    builder, kw, dt, t_end = RESTART_CASE
    p = build(builder, kw)
    with tempfile.TemporaryDirectory() as d:
        prm, out, rst, rho_f = (os.path.join(d, x) for x in ("in.prm", "out.txt", "restart.txt", "rho.txt"))
        with open(prm, "w") as f:
            f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_file=out)
                    + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
        subprocess.run([O.REF_DRIVER, "run", prm, "rk4", "1", rho_f], check=True, timeout=120,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        text = open(rst).read()
        rho = O.parse_rho_file(rho_f, p.num_states)
    with open(os.path.join(HERE, "ref_restart_indep_n3.txt"), "w") as f:
        f.write(text)
    with open(os.path.join(HERE, "ref_restart_indep_n3.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "builder": builder, "kwargs": kw,
                   "method": "rk4", "timestep": dt, "t_end": t_end,
                   "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}, f, indent=0)
    print("restart fixture written", flush=True)


OUTPUT_CASE = ("random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=3), 0.001, 0.01,
               0.002)


# (file stem, annealed() kwargs or None, TimeLocal, FilterTolerance)
OUTPUT_VARIANTS = [("ref_output_indep_n3_rk4", None, False, 0.0),
                   ("ref_output_anneal_n3_rk4", dict(seed=1), True, 1e-3)]


def make_output_fixture():
    builder, kw, dt, t_end, out_step = OUTPUT_CASE
    phi_bin = os.path.join(os.path.dirname(O.REF_DRIVER), "phi")
    for stem, akw, tl, ft in OUTPUT_VARIANTS:
        p = build(builder, kw)
        if akw is not None:
            p = cases.annealed(p, t_end, **akw)
        p.use_time_local_truncation = tl
        p.filter_tolerance = ft
        with tempfile.TemporaryDirectory() as d:
            prm, out = os.path.join(d, "in.prm"), os.path.join(d, "out.txt")
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_min_step=out_step, output_file=out)
                        .replace("verbose=-2", "verbose=0"))
            subprocess.run([phi_bin, prm, "rk4", "1"], check=True, timeout=120, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            text = open(out).read()
        with open(os.path.join(HERE, stem + ".txt"), "w") as f:
            f.write(text)
        meta = {"generator": "tests/golden/make_golden.py", "builder": builder, "kwargs": kw,
                "method": "rk4", "timestep": dt, "t_end": t_end, "output_min_step": out_step}
        if akw is not None or tl or ft:
            meta.update({"anneal": akw, "time_local": tl, "filter_tolerance": ft})
        with open(os.path.join(HERE, stem + ".json"), "w") as f:
            json.dump(meta, f, indent=0)
        print(f"output fixture {stem} written", flush=True)


# (case id, builder, builder kwargs, method, timestep, t_end, FilterTolerance)
FILTER_CASES = [
    ("rand_n3_k2_t4/rk4/1e-3", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=4, seed=2), "rk4", 0.001, 0.05, 1e-3),
    ("rand_n3_k2_t4/rkf45/1e-3", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=4, seed=2), "rkf45", 0.001, 0.05, 1e-3),
    ("rand_n4_k1_t5/rk4/1e-2", "random_problem",
     dict(kind="independent", n=4, matsubara=1, truncation=5, seed=1), "rk4", 0.001, 0.05, 1e-2),
    ("rand_n3_k2_t5/rkf45/1e-4", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=5, seed=2), "rkf45", 0.001, 0.1, 1e-4),
    ("frenkel7_L3/rk4/1e-3", "config:frenkel7", dict(depth=3), "rk4", 0.001, 0.05, 1e-3),
]


def parse_restart_state(text: str, n: int) -> list:
    """Every "(re,im)" of a PHI restart file after its time and dt lines, in
    file order (node-major, column-major within a node)."""
    body = text.split("\n", 2)[2]
    return [[float(a), float(b)] for a, b in re.findall(r"\(([^,()]+),([^,()]+)\)", body)]


def make_filter_fixture():
    outs = []
    for cid, builder, kw, method, dt, t_end, ft in FILTER_CASES:
        p = build(builder, kw)
        p.filter_tolerance = ft
        if method == "rkf45":
            p.fix_incompatible_combinations("rkf45")
        with tempfile.TemporaryDirectory() as d:
            prm, out, rst, rho_f = (os.path.join(d, x) for x in ("in.prm", "out.txt", "restart.txt", "rho.txt"))
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_file=out)
                        + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
            try:
                subprocess.run([O.REF_DRIVER, "run", prm, method, "1", rho_f], check=True, timeout=120,
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            except subprocess.TimeoutExpired:
                print(f"{cid}: TIMEOUT", flush=True)
                continue
            rho = O.parse_rho_file(rho_f, p.num_states)
            state = parse_restart_state(open(rst).read(), p.num_states)
        M = len(state) // (p.num_states * p.num_states)
        case = {"id": cid, "builder": builder, "kwargs": kw, "method": method, "timestep": dt, "t_end": t_end,
                "filter_tolerance": ft, "num_nodes": M,
                "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}
        if M <= 100:
            case["state_6_digits"] = state
        outs.append(case)
        print(f"{cid}: M={M}", flush=True)
    with open(os.path.join(HERE, "ref_filter.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": outs}, f, indent=0)


# (case id, builder, builder kwargs, method, timestep, t_end, FilterTolerance)
TIMELOCAL_CASES = [
    ("rand_n3_k2_t3/rk4", "random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2),
     "rk4", 0.001, 0.05, 0.0),
    ("rand_n3_k2_t3/rkf45", "random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2),
     "rkf45", 0.001, 0.05, 0.0),
    ("rand_n3_k3_t1/rk4", "random_problem", dict(kind="independent", n=3, matsubara=3, truncation=1, seed=3),
     "rk4", 0.001, 0.05, 0.0),
    ("rand_n3_k3_t1/rkf45", "random_problem", dict(kind="independent", n=3, matsubara=3, truncation=1, seed=3),
     "rkf45", 0.001, 0.05, 0.0),
    ("rand_n4_k1_t4/rk4", "random_problem", dict(kind="independent", n=4, matsubara=1, truncation=4, seed=1),
     "rk4", 0.001, 0.05, 0.0),
    ("rand_n3_k2_t4/rkf45/filter1e-3", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=4, seed=2), "rkf45", 0.001, 0.05, 1e-3),
    ("frenkel7_L2/rkf45", "config:frenkel7", dict(depth=2), "rkf45", 0.001, 0.05, 0.0),
    # correlated (diagonal) and full bath couplings: DiagonalBath / FullBath
    # DoTimelocal and the NoHierarchy updaters of a single tier
    ("diag_n3_b2_k2_t3/rk4", "random_problem", dict(kind="diagonal", n=3, matsubara=2, truncation=3, baths=2,
                                                     seed=4), "rk4", 0.001, 0.05, 0.0),
    ("diag_n3_b2_k2_t3/rkf45", "random_problem", dict(kind="diagonal", n=3, matsubara=2, truncation=3, baths=2,
                                                       seed=4), "rkf45", 0.001, 0.05, 0.0),
    ("full_n3_b2_k2_t3/rk4", "random_problem", dict(kind="full", n=3, matsubara=2, truncation=3, baths=2,
                                                     seed=5), "rk4", 0.001, 0.05, 0.0),
    ("full_n3_b2_k2_t3/rkf45", "random_problem", dict(kind="full", n=3, matsubara=2, truncation=3, baths=2,
                                                       seed=5), "rkf45", 0.001, 0.05, 0.0),
    ("diag_n2_b2_k2_t1/rk4", "random_problem", dict(kind="diagonal", n=2, matsubara=2, truncation=1, baths=2,
                                                     seed=6), "rk4", 0.001, 0.05, 0.0),
    ("full_n3_b2_k1_t1/rkf45", "random_problem", dict(kind="full", n=3, matsubara=1, truncation=1, baths=2,
                                                       seed=7), "rkf45", 0.001, 0.05, 0.0),
]


def make_timelocal_fixture():
    outs = []
    for cid, builder, kw, method, dt, t_end, ft in TIMELOCAL_CASES:
        p = build(builder, kw)
        p.use_time_local_truncation = True
        p.filter_tolerance = ft
        if method == "rkf45":
            p.fix_incompatible_combinations("rkf45")
        n = p.num_states
        with tempfile.TemporaryDirectory() as d:
            prm, out, rst, rho_f = (os.path.join(d, x) for x in ("in.prm", "out.txt", "restart.txt", "rho.txt"))
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_file=out)
                        + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
            try:
                subprocess.run([O.REF_DRIVER, "run", prm, method, "1", rho_f], check=True, timeout=120,
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            except subprocess.TimeoutExpired:
                print(f"{cid}: TIMEOUT", flush=True)
                continue
            rho = O.parse_rho_file(rho_f, n)
            numbers = parse_restart_state(open(rst).read(), n)
        M = O.node_count(p.num_bath_couplings * p.num_matsubara_terms, p.hierarchy_truncation_level)
        E = n * n
        state, qk = numbers[:M * E], numbers[M * E:]
        K1 = p.num_matsubara_terms
        assert len(qk) == p.num_bath_couplings * K1 * E, (cid, len(qk))
        case = {"id": cid, "builder": builder, "kwargs": kw, "method": method, "timestep": dt, "t_end": t_end,
                "filter_tolerance": ft, "num_nodes": M,
                "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}
        if M <= 100:
            case["state_6_digits"] = state
        if method == "rkf45":
            q = np.array([complex(a, b) for a, b in qk]).reshape(p.num_bath_couplings, K1, E).sum(axis=1)
            case["q_sums_6_digits"] = [[float(z.real), float(z.imag)] for z in q.reshape(-1)]
        outs.append(case)
        print(f"{cid}: M={M}", flush=True)
    with open(os.path.join(HERE, "ref_timelocal.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": outs}, f, indent=0)


# (case id, builder, builder kwargs, annealed() kwargs, method, timestep, t_end, TimeLocal)
ANNEAL_CASES = [
    ("indep_n3_k2_t3/rk4", "random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2),
     dict(seed=1), "rk4", 0.001, 0.05, False),
    ("indep_n3_k2_t3/rkf45", "random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2),
     dict(seed=1), "rkf45", 0.001, 0.05, False),
    ("indep_n3_k2_t3_complex/rk4", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2), dict(seed=2, complex_x=True), "rk4",
     0.001, 0.05, False),
    ("indep_n3_k2_t3_gate0.2/rk4", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2), dict(seed=3, min_field_change=0.2),
     "rk4", 0.001, 0.05, False),
    ("indep_n3_k2_t3_timelocal/rkf45", "random_problem",
     dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2), dict(seed=1), "rkf45", 0.001, 0.05, True),
    ("diag_n4_k2_t3/rk4", "random_problem", dict(kind="diagonal", n=4, matsubara=2, truncation=3, seed=3),
     dict(seed=1), "rk4", 0.001, 0.05, False),
    ("full_n3_k2_t3/rkf45", "random_problem", dict(kind="full", n=3, matsubara=2, truncation=3, seed=3),
     dict(seed=4), "rkf45", 0.001, 0.05, False),
    ("frenkel7_L2/rkf45", "config:frenkel7", dict(depth=2), dict(seed=1), "rkf45", 0.001, 0.05, False),
]


def make_anneal_fixture():
    outs = []
    for cid, builder, kw, akw, method, dt, t_end, tl in ANNEAL_CASES:
        p = cases.annealed(build(builder, kw), t_end, **akw)
        p.use_time_local_truncation = tl
        if method == "rkf45":
            p.fix_incompatible_combinations("rkf45")
        n = p.num_states
        with tempfile.TemporaryDirectory() as d:
            prm, out, rst, rho_f = (os.path.join(d, x) for x in ("in.prm", "out.txt", "restart.txt", "rho.txt"))
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_file=out)
                        + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
            try:
                subprocess.run([O.REF_DRIVER, "run", prm, method, "1", rho_f], check=True, timeout=120,
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            except subprocess.TimeoutExpired:
                print(f"{cid}: TIMEOUT", flush=True)
                continue
            rho = O.parse_rho_file(rho_f, n)
            numbers = parse_restart_state(open(rst).read(), n)
        M = O.node_count(p.num_bath_couplings * p.num_matsubara_terms, p.hierarchy_truncation_level)
        case = {"id": cid, "builder": builder, "kwargs": kw, "anneal": akw, "method": method, "timestep": dt,
                "t_end": t_end, "time_local": tl, "num_nodes": M,
                "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}
        if M <= 100:
            case["state_6_digits"] = numbers[:M * n * n]
        outs.append(case)
        print(f"{cid}: M={M}", flush=True)
    with open(os.path.join(HERE, "ref_anneal.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": outs}, f, indent=0)


RESTART_TL_CASE = ("random_problem", dict(kind="independent", n=3, matsubara=2, truncation=3, seed=2),
                   0.001, 0.02, 0.04)


def make_restart_tl_fixture():
    builder, kw, dt, t1, t2 = RESTART_TL_CASE
    p = build(builder, kw)
    p.use_time_local_truncation = True
    p.fix_incompatible_combinations("rkf45")
    n = p.num_states
    with tempfile.TemporaryDirectory() as d:
        prm1, prm2, out, rst, rho1, rho2 = (os.path.join(d, x) for x in
                                            ("a.prm", "b.prm", "o.txt", "restart.txt", "r1.txt", "r2.txt"))
        with open(prm1, "w") as f:
            f.write(O.param_file_text(p, timestep=dt, t_end=t1, output_file=out)
                    + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
        subprocess.run([O.REF_DRIVER, "run", prm1, "rkf45", "1", rho1], check=True, timeout=120,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        lines = open(rst).read().split("\n")
        lines[1] = repr(float(dt))  # PHI wrote the clamped step size (0)
        text = "\n".join(lines)
        with open(rst, "w") as f:
            f.write(text)
        with open(prm2, "w") as f:
            f.write(O.param_file_text(p, timestep=dt, t_end=t2, output_file=out) + f"RestartInput={rst}\n")
        subprocess.run([O.REF_DRIVER, "run", prm2, "rkf45", "1", rho2], check=True, timeout=120,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        rho = O.parse_rho_file(rho2, n)
    with open(os.path.join(HERE, "ref_restart_timelocal_n3.txt"), "w") as f:
        f.write(text)
    with open(os.path.join(HERE, "ref_restart_timelocal_n3.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "builder": builder, "kwargs": kw,
                   "method": "rkf45", "time_local": True, "timestep": dt, "t1": t1, "t2": t2,
                   "num_matrices": p.num_bath_couplings * p.num_matsubara_terms,
                   "edited": "step-size line set to the timestep (PHI writes the clamped 0)",
                   "rho0_t2_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}, f, indent=0)
    print("time-local restart fixture written", flush=True)


# Benchmarked configurations at their full size, run by the reference build
# with all host threads (its results do not depend on the thread count):
# (case id, configs builder, builder kwargs, method, timestep, t_end).
FULLSIZE_CASES = [
    ("frenkel7_L6/rkf45", "frenkel7", {}, "rkf45", 0.001, 1.0),
    ("frenkel7_L6/rk4", "frenkel7", {}, "rk4", 0.001, 0.3),
    ("ring24_L4/rkf45", "ring24", {}, "rkf45", 0.001, 0.5),
    # RK4 at 1 fs is unstable at this depth (tier-8 Matsubara damping of
    # ~4e3 ps^-1); the reference and the device both diverge there.
    ("chain4_L8/rk4", "chain4", {}, "rk4", 0.00025, 0.025),
]


def make_fullsize_fixture(only=None):
    """ref_fullsize.json: rho_0 (%.17g) and PHI's own step counts for the
    benchmarked configurations at full size (38,760 / 20,475 / 125,970
    nodes).  Each case runs the reference for minutes; the file is
    rewritten after every case so a partial run keeps what it finished."""
    path = os.path.join(HERE, "ref_fullsize.json")
    done = {}
    if os.path.exists(path):
        done = {c["id"]: c for c in json.load(open(path))["cases"]}
    threads = os.cpu_count() or 1
    for cid, builder, kw, method, dt, t_end in FULLSIZE_CASES:
        if only and cid not in only:
            continue
        p = getattr(configs, builder)(**kw)
        with tempfile.TemporaryDirectory() as d:
            prm, out, rho_f = (os.path.join(d, x) for x in ("in.prm", "out.txt", "rho.txt"))
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=dt, t_end=t_end, output_min_step=t_end,
                                          output_file=out).replace("verbose=-2", "verbose=0"))
            subprocess.run([O.REF_DRIVER, "run", prm, method, str(threads), rho_f], check=True,
                           timeout=3600, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            rho = O.parse_rho_file(rho_f, p.num_states)
            secs = float(open(rho_f).read().split("\n")[0].split()[1])
            steps = accepted = None
            for ln in open(out):
                if ln.startswith("#Total number of integration steps"):
                    steps = int(ln.split("=")[1])
                if ln.startswith("#Total number of accepted integration steps"):
                    accepted = int(ln.split("=")[1])
        done[cid] = {"id": cid, "builder": builder, "kwargs": kw, "seed": int(p.seed), "method": method,
                     "timestep": dt, "t_end": t_end, "rkf45_tolerance": float(p.rkf45_tolerance),
                     "rkf45_mindt": float(p.rkf45_minimum_timestep), "steps": steps,
                     "accepted_steps": accepted, "threads": threads, "launch_seconds": secs,
                     "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]}
        with open(path, "w") as f:
            json.dump({"generator": "tests/golden/make_golden.py fullsize",
                       "cases": [done[c[0]] for c in FULLSIZE_CASES if c[0] in done]}, f, indent=0)
        print(f"{cid}: {steps} steps ({accepted} accepted), {secs:.1f} s", flush=True)


# Hilbert-space truncation, run by the reference built in BLAS mode (its
# -DNOBLAS loops flip signs in the truncator): (case id, truncated_problem
# kwargs, method, timestep, t_end).
TRUNCATION_CASES = [
    ("trunc_f4_k3_b2_k2_t3/rk4", dict(full=4, k=3, baths=2, matsubara=2, truncation=3, seed=1), "rk4", 0.001, 0.05),
    ("trunc_f4_k3_b2_k2_t3/rkf45", dict(full=4, k=3, baths=2, matsubara=2, truncation=3, seed=1), "rkf45", 0.001,
     0.05),
    ("trunc_f5_k2_b3_k1_t3/rk4", dict(full=5, k=2, baths=3, matsubara=1, truncation=3, seed=2), "rk4", 0.001, 0.05),
    ("trunc_f3_k2_vacuum/rk4", dict(full=3, k=2, baths=1, matsubara=1, truncation=1, seed=3), "rk4", 0.001, 0.05),
    ("trunc_f4_k3_timelocal/rkf45", dict(full=4, k=3, baths=2, matsubara=2, truncation=3, seed=4, time_local=True),
     "rkf45", 0.001, 0.05),
]


def make_truncation_fixture():
    """ref_truncation.json: rho_0 (F x F, %.17g) of the BLAS-mode reference
    build for Hilbert-space truncated problems."""
    if not os.path.exists(O.REF_DRIVER_BLAS):
        raise SystemExit("build the BLAS-mode reference first: make -C oracle/refbuild blas REF_SRC=... BLAS_LIB=...")
    outs = []
    for cid, kw, method, dt, t_end in TRUNCATION_CASES:
        p = cases.truncated_problem(**kw)
        if method == "rkf45":
            p.fix_incompatible_combinations("rkf45")
        rho, secs = O.run_reference(p, method, 1, timeout=300, driver=O.REF_DRIVER_BLAS, timestep=dt, t_end=t_end)
        outs.append({"id": cid, "kwargs": kw, "method": method, "timestep": dt, "t_end": t_end,
                     "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]})
        print(f"{cid}: {secs:.3f}s", flush=True)
    with open(os.path.join(HERE, "ref_truncation.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py truncation (reference built in BLAS mode)",
                   "cases": outs}, f, indent=0)


# (case id, builder, kwargs, method, timestep, t_end): Hilbert-space truncation
# of annealing Hamiltonians.  "truncated_annealed" draws seeded problems;
# "reference_truncated_anneal" builds the problems of the reference's own
# truncated annealing tests.
TRUNC_ANNEAL_CASES = [
    ("ta_f4_k2_t3/rkf45", "truncated_annealed", dict(full=4, k=2, seed=1), "rkf45", 0.001, 0.05),
    ("ta_f4_k2_t3/rk4", "truncated_annealed", dict(full=4, k=2, seed=1), "rk4", 0.001, 0.05),
    ("ta_f5_k3_t2/rk4", "truncated_annealed", dict(full=5, k=3, seed=2, truncation=2), "rk4", 0.001, 0.05),
    ("ta_f4_k3_t1/rkf45", "truncated_annealed", dict(full=4, k=3, seed=4, truncation=1), "rkf45", 0.001, 0.05),
    ("ta_f4_k2_t3_gate0.2/rkf45", "truncated_annealed", dict(full=4, k=2, seed=5, min_field_change=0.2), "rkf45",
     0.001, 0.05),
    ("ta_f4_k2_t3_timelocal/rkf45", "truncated_annealed", dict(full=4, k=2, seed=3, time_local=True), "rkf45",
     0.001, 0.05),
    ("refcfg_vacuum/rk4", "reference_truncated_anneal", dict(test="vacuum"), "rk4", 0.001, 1.0),
    ("refcfg_vacuum/rkf45", "reference_truncated_anneal", dict(test="vacuum"), "rkf45", 0.001, 1.0),
    ("refcfg_medium_full_indep/rk4", "reference_truncated_anneal", dict(test="medium_full_indep"), "rk4", 0.001,
     1.0),
    ("refcfg_medium_full_indep/rkf45", "reference_truncated_anneal", dict(test="medium_full_indep"), "rkf45",
     0.001, 1.0),
    ("refcfg_weak_full_indep_tl/rkf45", "reference_truncated_anneal", dict(test="weak_full_indep_tl"), "rkf45",
     0.001, 10.0),
    ("refcfg_weak_full_tl/rkf45", "reference_truncated_anneal", dict(test="weak_full_tl"), "rkf45", 0.001, 10.0),
]


def trunc_anneal_problem(builder, kw, method):
    p = getattr(cases, builder)(**kw)
    if method == "rkf45":
        p.fix_incompatible_combinations("rkf45")
    return p


def make_trunc_anneal_fixture():
    """ref_trunc_anneal.json: rho_0 (F x F, %.17g) of the BLAS-mode reference
    build for Hilbert-space truncated annealing problems."""
    if not os.path.exists(O.REF_DRIVER_BLAS):
        raise SystemExit("build the BLAS-mode reference first: make -C oracle/refbuild blas REF_SRC=... BLAS_LIB=...")
    outs = []
    for cid, builder, kw, method, dt, t_end in TRUNC_ANNEAL_CASES:
        p = trunc_anneal_problem(builder, kw, method)
        rho, secs = O.run_reference(p, method, 1, timeout=600, driver=O.REF_DRIVER_BLAS, timestep=dt, t_end=t_end)
        outs.append({"id": cid, "builder": builder, "kwargs": kw, "method": method, "timestep": dt, "t_end": t_end,
                     "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]})
        print(f"{cid}: {secs:.3f}s", flush=True)
    with open(os.path.join(HERE, "ref_trunc_anneal.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py trunc_anneal (reference built in BLAS mode)",
                   "cases": outs}, f, indent=0)


def make_fullsize_decisions():
    """For each full-size RKF45 case of ref_fullsize.json: the oracle's error
    estimate of every attempted step and the accept decision it leads to
    (0 reject, 1 accept, 2 accept and grow the step).  The oracle must end
    on the reference's rho_0 bit for bit and take its step counts, so its
    decisions are the reference's (which the reference does not print)."""
    path = os.path.join(HERE, "ref_fullsize.json")
    data = json.load(open(path))
    O.set_threads(os.cpu_count() or 1)
    for c in data["cases"]:
        if c["method"] != "rkf45" or "decisions" in c:
            continue
        p = getattr(configs, c["builder"])(**c["kwargs"])
        p.fix_incompatible_combinations("rkf45")
        o = O.Oracle(p)
        state, st = o.rkf45(o.initial_state(), c["timestep"], c["t_end"], c["rkf45_tolerance"],
                            c["rkf45_mindt"], trace_capacity=c["steps"] + 1)
        v = np.array(c["rho0_colmajor"])
        ref = (v[:, 0] + 1j * v[:, 1]).reshape(p.num_states, p.num_states).T
        diff = float(np.abs(o.rho0(state) - ref).max())
        if diff != 0.0 or st["steps"] != c["steps"] or st["accepted"] != c["accepted_steps"]:
            raise SystemExit(f"{c['id']}: oracle differs from the reference ({diff}, {st})")
        tol = c["rkf45_tolerance"]
        errs = st["errors"]
        # The accept rule (hierarchy_integrator.cc:2355, :2400): the step-size
        # floor is never reached on these runs (checked: no attempt below 2 mindt).
        c["oracle_errors"] = [float(e) for e in errs]
        c["decisions"] = [0 if not e < tol else (2 if e < tol / 10 else 1) for e in errs]
        c["oracle_rho0_max_abs_diff"] = diff
        print(f"{c['id']}: {len(errs)} decisions, min |err - tol| / tol = "
              f"{min(abs(e - tol) / tol for e in errs):.3e}", flush=True)
        with open(path, "w") as f:
            json.dump(data, f, indent=0)
    O.set_threads(1)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PHI_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("usage: make_golden.py <reference source root> [fixture]  "
                         "(or set PHI_REFERENCE_ROOT)")
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle REF_SRC=<reference>/src")
    if len(sys.argv) > 2 and sys.argv[2] == "fullsize":
        make_fullsize_fixture(sys.argv[3:] or None)
        make_fullsize_decisions()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "truncation":
        make_truncation_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "trunc_anneal":
        make_trunc_anneal_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "fullsize_decisions":
        make_fullsize_decisions()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "restart":
        make_restart_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "output":
        make_output_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "filter":
        make_filter_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "timelocal":
        make_timelocal_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "anneal":
        make_anneal_fixture()
        return
    if len(sys.argv) > 2 and sys.argv[2] == "restart_tl":
        make_restart_tl_fixture()
        return
    make_restart_fixture()
    make_output_fixture()
    make_filter_fixture()
    make_timelocal_fixture()
    make_anneal_fixture()
    make_restart_tl_fixture()
    golden = parse_reference_tests(ref_root)
    with open(os.path.join(HERE, "reference_tests.json"), "w") as f:
        json.dump({"source": "src/hierarchy_integrator_test.cc:350-509", "vectors": golden}, f, indent=1)

    outs = []
    for cid, builder, kw, method, run in CASES:
        p = build(builder, kw)
        try:
            rho, secs = O.run_reference(p, method, 1, timeout=60, **run)
        except subprocess.TimeoutExpired:
            # The reference's RKF45 accept test races with its writer thread
            # (hierarchy_integrator.cc:2355 vs :2434-2437) and can deadlock.
            outs.append({"id": cid, "builder": builder, "kwargs": kw, "method": method,
                         "run": run, "unavailable": "reference run timed out (RKF45 thread race)"})
            print(f"{cid}: TIMEOUT", flush=True)
            continue
        outs.append({"id": cid, "builder": builder, "kwargs": kw, "method": method, "run": run,
                     "rho0_colmajor": [[float(z.real), float(z.imag)] for z in rho.T.reshape(-1)]})
        print(f"{cid}: {secs:.3f}s", flush=True)
    with open(os.path.join(HERE, "ref_outputs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": outs}, f, indent=0)

    orders = []
    for T, tr in ORDERS:
        p = cases.random_problem("independent", n=T, matsubara=1, truncation=tr, seed=0)
        mi = O.reference_order(p)
        orders.append({"terms": T, "truncation": tr, "multi_index": mi.tolist()})
        print(f"order T={T} trunc={tr}: {mi.shape[0]} nodes", flush=True)
    with open(os.path.join(HERE, "ref_order.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "orders": orders}, f)


if __name__ == "__main__":
    main()
