"""Loaders for the committed golden fixtures (tests/golden/*.json)."""
from __future__ import annotations

import json
import os

import numpy as np

import cases
from phi_b200 import configs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def reference_test_vectors():
    """{key: N x N complex} from the reference's own tests."""
    data = _load("reference_tests.json")["vectors"]
    out = {}
    for k, vals in data.items():
        v = np.array([a + 1j * b for a, b in vals])
        n = int(round(len(v) ** 0.5))
        out[k] = v.reshape(n, n).T.copy()  # listed in storage (column-major) order
    return out


def build_case(builder: str, kwargs: dict):
    if builder.startswith("config:"):
        return getattr(configs, builder.split(":", 1)[1])(**kwargs)
    return getattr(cases, builder)(**kwargs)


def ref_outputs():
    """[(case dict, problem, rho_0 N x N complex or None)] printed by the reference."""
    out = []
    for c in _load("ref_outputs.json")["cases"]:
        p = build_case(c["builder"], c["kwargs"])
        rho = None
        if "rho0_colmajor" in c:
            v = np.array([a + 1j * b for a, b in c["rho0_colmajor"]])
            n = int(p.num_states)
            rho = v.reshape(n, n).T.copy()
        out.append((c, p, rho))
    return out


def ref_orders():
    return [(o["terms"], o["truncation"], np.array(o["multi_index"], np.int32))
            for o in _load("ref_order.json")["orders"]]
