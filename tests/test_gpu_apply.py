"""One Liouvillian apply (HierarchyUpdater::Get over every node,
hierarchy_updater.h:36-52) on the GPU against the CPU oracle, on random
Hermitian ADOs.  FP64: max-abs difference <= 1e-12 of the output scale."""
import numpy as np
import pytest

import cases
from oracle import oracle as O
from phi_b200 import configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12

PROBLEMS = [
    ("indep_n2_K1_L4", dict(kind="independent", n=2, matsubara=1, truncation=5)),
    ("indep_n3_K2_L3", dict(kind="independent", n=3, matsubara=2, truncation=4)),
    ("indep_n4_K3_L3", dict(kind="independent", n=4, matsubara=3, truncation=4, complex_h=True)),
    ("indep_n7_K2_L2", dict(kind="independent", n=7, matsubara=2, truncation=3)),
    ("indep_n12_K1_L2", dict(kind="independent", n=12, matsubara=1, truncation=3)),
    ("indep_n16_K1_L2", dict(kind="independent", n=16, matsubara=1, truncation=3)),
    ("indep_n24_K1_L2", dict(kind="independent", n=24, matsubara=1, truncation=3)),
    ("indep_unnormalized", dict(kind="independent", n=3, matsubara=2, truncation=4, normalized=False)),
    ("diag_n2_b1_L6", dict(kind="diagonal", n=2, matsubara=1, truncation=7, baths=1)),
    ("diag_n3_b2_K2", dict(kind="diagonal", n=3, matsubara=2, truncation=4, baths=2)),
    ("diag_n5_b3_K1", dict(kind="diagonal", n=5, matsubara=1, truncation=3, baths=3, complex_h=True)),
    ("full_n2_b2_K2", dict(kind="full", n=2, matsubara=2, truncation=4, baths=2)),
    ("full_n4_b3_K1", dict(kind="full", n=4, matsubara=1, truncation=3, baths=3)),
    ("full_n13_b2_K1", dict(kind="full", n=13, matsubara=1, truncation=3, baths=2)),
]


def _check(p, seed=1):
    o = O.Oracle(p)
    s = cases.random_hermitian_state(o.M, p.num_states, seed=seed)
    ref = o.apply(s)
    with Hierarchy(p) as h:
        got = h.apply(s)
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max()
    assert err <= FP64_RTOL * scale, (err, scale)
    # every output ADO Hermitian, exactly
    n = p.num_states
    d = got.view(np.complex128).reshape(-1, n, n)
    assert np.array_equal(d, np.conj(np.transpose(d, (0, 2, 1))))


@pytest.mark.parametrize("name,kw", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_apply_matches_oracle(name, kw):
    _check(cases.random_problem(seed=3, **kw))


@pytest.mark.parametrize("make", [configs.spin_boson, lambda: configs.frenkel7(depth=3),
                                  lambda: configs.chain4(depth=3), lambda: configs.ring24(depth=2)],
                         ids=["spin_boson", "frenkel7_L3", "chain4_L3", "ring24_L2"])
def test_apply_matches_oracle_on_workloads(make):
    _check(make())


def test_vacuum_apply_is_unitary_only():
    p = cases.reference_fixture_case("TestVacuum")
    _check(p)


def test_apply_is_linear():
    p = cases.random_problem("independent", n=4, matsubara=2, truncation=4, seed=9)
    with Hierarchy(p) as h:
        a = cases.random_hermitian_state(h.num_nodes, 4, seed=1)
        b = cases.random_hermitian_state(h.num_nodes, 4, seed=2)
        la, lb, lab = h.apply(a), h.apply(b), h.apply(2.0 * a - 0.5 * b)
    assert np.abs(lab - (2.0 * la - 0.5 * lb)).max() <= 1e-12 * np.abs(lab).max()
