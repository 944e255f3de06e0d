"""The parameter-file boundary on the GPU: PhiParameters::ReadCommandLine ->
phi_gpu_create_from_file gives the same context as the descriptor path, and
the phi_b200 command-line driver (phi.cc:4-10's interface) writes PHI's
output file (hierarchy_integrator.cc:313-319 header, :2858-2880 rows,
:2905-2924 closing row; :3730-3761 for steady state)."""
import os
import re
import subprocess

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "phi_b200", "phi_b200")
_CPLX = re.compile(r"\(([^,()]+),([^,()]+)\)")


def _complexes(line):
    return np.array([complex(float(a), float(b)) for a, b in _CPLX.findall(line)])


def _write(tmp_path, text, name="params.txt"):
    f = tmp_path / name
    f.write_text(text)
    return str(f)


@pytest.mark.parametrize("make", [configs.spin_boson, lambda: configs.frenkel7(depth=3),
                                  lambda: cases.random_problem("diagonal", n=3, matsubara=2, truncation=3, seed=2),
                                  lambda: cases.random_problem("full", n=2, matsubara=2, truncation=3, seed=2)],
                         ids=["spin_boson", "frenkel7_L3", "diagonal_n3", "full_n2"])
def test_file_context_equals_descriptor_context(tmp_path, make):
    p = make()
    path = _write(tmp_path, O.param_file_text(p, timestep=0.001, t_end=0.05))
    with Hierarchy.from_file(path, "rk4") as hf, Hierarchy(p) as hd:
        assert (hf.num_nodes, hf.num_terms, hf.n) == (hd.num_nodes, hd.num_terms, hd.n)
        assert np.array_equal(hf.get_state(), hd.get_state())
        hf.rk4(0.001, 0.05)
        hd.rk4(0.001, 0.05)
        assert np.array_equal(hf.get_state(), hd.get_state())


def test_cli_rk4_output_file(tmp_path):
    p = configs.frenkel7(depth=3)
    out = tmp_path / "out.txt"
    path = _write(tmp_path, O.param_file_text(p, timestep=0.001, t_end=0.02, output_min_step=0.005,
                                              output_file=str(out)).replace("verbose=-2", "verbose=0"))
    r = subprocess.run([CLI, path, "rk4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = out.read_text().splitlines()
    assert any(l.startswith("#Total Number of matrices:") for l in lines)
    assert "#Integrator=rk4" in lines
    body = [l for l in lines if l and not l.startswith("#")]
    with Hierarchy(p) as h:
        _, times, rows = h.rk4(0.001, 0.02, 0.005, capacity=64)
        rho = h.rho0()
    # initial row, one row per output step, the closing row at 4 digits
    assert len(body) == 1 + len(times) + 1
    np.testing.assert_allclose(_complexes(body[0]), np.asarray(p.initial_density_matrix).T.reshape(-1), atol=1e-6)
    for line, t, row in zip(body[1:-1], times, rows):
        assert abs(float(line.split()[0]) - t) <= 1e-5 * max(1.0, t)
        np.testing.assert_allclose(_complexes(line), row.T.reshape(-1), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(_complexes(body[-1]), rho.T.reshape(-1), rtol=0, atol=1e-3)


def test_cli_steady_state_output_file(tmp_path):
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=4, seed=3)
    out = tmp_path / "ss.txt"
    text = O.param_file_text(p, output_file=str(out)) + "bicgstab_tolerance=1e-9\n"
    path = _write(tmp_path, text)
    r = subprocess.run([CLI, path, "bicgstab"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = out.read_text().splitlines()
    assert "#Calculating steady-state using BiCGSTAB(2)" in lines  # PhiParameters::Write (phi_parameters.cc:1108-1116)
    assert any(l.startswith("#Info: Converged to diff =") for l in lines)
    ref = O.Oracle(p)
    rho_ref = ref.rho0(ref.steady_state())
    final = [l for l in lines if l and not l.startswith("#")][-1]
    np.testing.assert_allclose(_complexes(final), rho_ref.T.reshape(-1), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("stem", ["ref_output_indep_n3_rk4", "ref_output_anneal_n3_rk4"],
                         ids=["static", "annealing_timelocal_filter"])
def test_cli_output_file_matches_reference_layout(tmp_path, stem):
    """Our CLI's output file against the one the reference's `phi` wrote for
    the same parameters (tests/golden/<stem>.txt; the second run anneals
    with time-local truncation and filtering on): the same '#' header lines
    (memory figures are each implementation's own), the same dynamics-row
    times and values to PHI's 6 significant digits, the same closing step
    count and the final row to its 4 digits."""
    import json as _json
    here = os.path.dirname(os.path.abspath(__file__))
    meta = _json.load(open(os.path.join(here, "golden", stem + ".json")))
    ref_lines = open(os.path.join(here, "golden", stem + ".txt")).read().splitlines()
    p = getattr(cases, meta["builder"])(**meta["kwargs"])
    if meta.get("anneal") is not None:
        p = cases.annealed(p, meta["t_end"], **meta["anneal"])
    p.use_time_local_truncation = bool(meta.get("time_local", False))
    p.filter_tolerance = float(meta.get("filter_tolerance", 0.0))
    out = tmp_path / "out.txt"
    path = _write(tmp_path, O.param_file_text(p, timestep=meta["timestep"], t_end=meta["t_end"],
                                              output_min_step=meta["output_min_step"], output_file=str(out))
                  .replace("verbose=-2", "verbose=0"))
    r = subprocess.run([CLI, path, "rk4", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ours = out.read_text().splitlines()

    def header(lines):
        h = []
        for l in lines:
            if not l.startswith("#"):
                break
            key = l.split(":")[0] if (" Mb." in l) else l
            h.append(key)
        return h
    assert header(ours) == header(ref_lines)

    def rows(lines):
        body = [l for l in lines if l and not l.startswith("#")]
        return body[:-1], body[-1]
    (ro, fo), (rr, fr) = rows(ours), rows(ref_lines)
    assert len(ro) == len(rr)
    for k, (a, b) in enumerate(zip(ro, rr)):
        assert a.split()[0] == b.split()[0]  # the time as PHI prints it
        # PHI's writer thread prints node 0 after the "rho updated" barrier
        # while the workers go on (hierarchy_integrator.cc:2856-2878); at the
        # first output row it also writes its timing comments, and the row
        # it prints (time 0.001) already holds the second step's state.  The
        # rows here hold the state of their time; rows 0 (rho(0)) and from
        # the second output on coincide.
        if k == 1:
            continue
        np.testing.assert_allclose(_complexes(a), _complexes(b), rtol=2e-5, atol=1e-9)
    np.testing.assert_allclose(_complexes(fo), _complexes(fr), rtol=1e-3, atol=1e-6)
    steps = [l for l in ours if l.startswith("#Total number of integration steps")]
    assert steps == [l for l in ref_lines if l.startswith("#Total number of integration steps")]
