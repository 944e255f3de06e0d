"""The C-ABI library loads and exports every symbol include/phi_b200.h declares
(CPU: no compute calls), and host-side validation errors need no GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import cases
from phi_b200 import capi
from phi_b200.heom import Hierarchy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:PHI_API\s+)?int\s+(phi_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_library_exports_declared_symbols():
    lib = capi.load()
    names = declared_symbols()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declared_symbols():
    bound = {name for name, _, _ in capi.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_invalid_descriptor_rejected_before_gpu():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=0)
    p.num_bath_couplings = 2  # independent baths must match the states
    p.gamma = p.gamma[:2]
    p.lambda_ = p.lambda_[:2]
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p)
    assert e.value.code == capi.PHI_E_INVALID


def test_non_hermitian_initial_state_rejected():
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=0)
    r = np.array(p.initial_density_matrix)
    r[0, 1] = 0.3
    p.initial_density_matrix = r
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p)
    assert e.value.code == capi.PHI_E_INVALID


def test_asymmetric_full_coupling_rejected():
    p = cases.random_problem("full", n=3, matsubara=1, truncation=2, seed=0)
    V = np.array(p.bath_coupling_op)
    V[0, 0, 1] += 1.0
    p.bath_coupling_op = V
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p)
    assert e.value.code == capi.PHI_E_INVALID


def test_zero_gamma_rejected_for_normalised_hierarchy():
    p = cases.random_problem("independent", n=2, matsubara=1, truncation=3, seed=0)
    p.gamma = np.array([0.0, 1.0])
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p)
    assert e.value.code == capi.PHI_E_INVALID


def test_null_arguments():
    lib = capi.load()
    out = ctypes.c_void_p()
    assert lib.phi_gpu_create(None, ctypes.byref(out)) == capi.PHI_E_INVALID
    assert lib.phi_gpu_destroy(None) == capi.PHI_OK
