"""Restart and state files on the GPU: a run split by a restart file equals
the uninterrupted run bit for bit; a restart file written by the reference
build continues on the device; the binary state file round-trips; the C++
facade reads RestartInput and writes RestartFile."""
import json
import os
import subprocess

import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_restart_indep_n3.txt")
META = json.load(open(os.path.join(HERE, "golden", "ref_restart_indep_n3.json")))
CLI = os.path.join(os.path.dirname(HERE), "phi_b200", "phi_b200")


def _rk4_steps(h, dt, steps):
    t0 = h.time
    h.rk4(dt, t0 + (steps - 0.5) * dt)


def test_split_run_equals_uninterrupted_run(tmp_path):
    p = configs.frenkel7(depth=3)
    with Hierarchy(p) as a:
        _rk4_steps(a, 0.001, 40)
        ref = a.get_state()
    with Hierarchy(p) as b:
        _rk4_steps(b, 0.001, 20)
        b.write_restart(tmp_path / "r.txt", 0.001)
    with Hierarchy(p) as c:
        dt = c.read_restart(tmp_path / "r.txt")
        assert dt == 0.001 and abs(c.time - 0.02) < 1e-15
        _rk4_steps(c, dt, 20)
        got = c.get_state()
    assert np.array_equal(got, ref)


def test_reference_restart_file_continues_on_device():
    p = getattr(cases, META["builder"])(**META["kwargs"])
    dt = META["timestep"]
    with Hierarchy(p) as h:
        assert h.read_restart(FIX) == pytest.approx(dt)
        _rk4_steps(h, dt, 10)
        got = h.rho0()
    with Hierarchy(p) as h:
        _rk4_steps(h, dt, 20)
        ref = h.rho0()
    assert np.abs(got - ref).max() <= 1e-5


def test_binary_state_file_round_trip(tmp_path):
    p = configs.chain4(depth=3)
    with Hierarchy(p) as a:
        _rk4_steps(a, 0.001, 7)
        a.save_state(tmp_path / "s.bin", 0.001)
        ref = a.get_state()
        t = a.time
    with Hierarchy(p) as b:
        assert b.load_state(tmp_path / "s.bin") == 0.001
        assert np.array_equal(b.get_state(), ref) and b.time == t
    with Hierarchy(configs.chain4(depth=2)) as c:  # another hierarchy size
        with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
            c.load_state(tmp_path / "s.bin")


def test_facade_writes_and_reads_restart_files(tmp_path):
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=3)
    rst = tmp_path / "restart.txt"
    prm = tmp_path / "a.prm"
    prm.write_text(O.param_file_text(p, timestep=0.001, t_end=0.01, output_file=str(tmp_path / "a.out"))
                   + f"RestartFile={rst}\nRestartOutputTimeSecs=1\n")
    r = subprocess.run([CLI, str(prm), "rk4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = p.num_states
    M = configs.hierarchy_nodes(6, 2)
    st, t, dt = capi.restart_read(rst, n, M)
    assert t == pytest.approx(0.01) and dt == 0.001
    with Hierarchy(p) as h:
        _rk4_steps(h, 0.001, 10)
        assert np.array_equal(h.get_state(), st)  # 17 digits: exact
    # continue from it through RestartInput
    prm2 = tmp_path / "b.prm"
    out2 = tmp_path / "b.out"
    prm2.write_text(O.param_file_text(p, timestep=0.001, t_end=0.02, output_file=str(out2))
                    + f"RestartInput={rst}\n")
    r = subprocess.run([CLI, str(prm2), "rk4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    with Hierarchy(p) as h:
        _rk4_steps(h, 0.001, 20)
        ref = h.rho0()
    last = [l for l in out2.read_text().splitlines() if l and not l.startswith("#")][-1]
    import re
    vals = np.array([complex(float(a), float(b)) for a, b in re.findall(r"\(([^,()]+),([^,()]+)\)", last)])
    np.testing.assert_allclose(vals, ref.T.reshape(-1), rtol=0, atol=1e-3)
