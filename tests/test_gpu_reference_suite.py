"""The reference's own test file (src/hierarchy_integrator_test.cc: 28
TEST_Fs with hard-coded rho_0 vectors, RK4 within 1e-6 and RKF45 within 1e-3)
compiled unchanged against this library's drop-in headers (include/phi/)
and run on the GPU through PhiParameters -> HierarchyIntegrator::Launch ->
density_matrix().  tests/refsuite/Makefile builds the binary from the
reference sources where they are present; it travels with the tree."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "refsuite", "_bin", "ref_hierarchy_integrator_test")


def _run_suite():
    if not os.path.exists(BIN):
        pytest.fail(f"{BIN} is missing: build it with make -C tests/refsuite REF_SRC=<reference>/src")
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    results, current = {}, None
    for ln in out.stdout.splitlines():
        if ln.startswith(("PASS ", "FAIL ")):
            current = ln.split()[1].split(".", 1)[1]
            results[current] = [ln.startswith("PASS")]
        elif ln.startswith("  ") and current:
            results[current].append(ln.strip())
    return results, out.stdout


def test_reference_suite_passes_on_the_drop_in():
    results, text = _run_suite()
    assert len(results) == 28, text[-2000:]
    failed = {k: v[1:] for k, v in results.items() if not v[0]}
    print(f"{28 - len(failed)} of 28 reference tests pass; failing: {sorted(failed)}")
    for k, msgs in failed.items():
        print(k, "\n  ".join(msgs[:2]))
    assert not failed, sorted(failed)
