"""Device hierarchy construction: bit-exact to the reference node order
(hierarchy.cc:45-155) and to the neighbour lists of LinkHierarchyNodes
(hierarchy_integrator.cc:1204-1338)."""
import numpy as np
import pytest

import cases
import golden_data
from oracle import oracle as O
from phi_b200 import configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", golden_data.ref_orders(), ids=lambda o: f"T{o[0]}_trunc{o[1]}")
def test_device_order_matches_reference_print(order):
    T, trunc, mi_ref = order
    p = cases.random_problem("independent", n=T, matsubara=1, truncation=trunc, seed=0)
    with Hierarchy(p) as h:
        mi, nx, pv = h.node_table()
    assert np.array_equal(mi, mi_ref)


SHAPES = [
    ("spin_boson_L10", lambda: configs.spin_boson()),
    ("frenkel7_L6", lambda: configs.frenkel7()),           # 38,760 nodes, T = 14
    ("chain4_L8", lambda: configs.chain4()),               # 125,970 nodes, T = 12
    ("ring24_L4", lambda: configs.ring24()),               # 20,475 nodes, T = 24
    ("indep_n3_K2_L5", lambda: cases.random_problem("independent", n=3, matsubara=3, truncation=6)),
    ("full_n2_K3_L3", lambda: cases.random_problem("full", n=2, matsubara=3, truncation=4, baths=3)),
    ("vacuum", lambda: cases.reference_fixture_case("TestVacuum")),
]


@pytest.mark.parametrize("name,make", SHAPES, ids=[s[0] for s in SHAPES])
def test_device_tables_match_oracle(name, make):
    p = make()
    o = O.Oracle(p)
    mi_o, nx_o, pv_o = o.tables()
    with Hierarchy(p) as h:
        assert h.num_nodes == o.M and h.num_terms == o.T
        mi, nx, pv = h.node_table()
    assert np.array_equal(mi, mi_o)
    assert np.array_equal(nx, nx_o)
    assert np.array_equal(pv, pv_o)


def test_node_budget_is_enforced():
    p = configs.frenkel7()
    from phi_b200 import capi
    with pytest.raises(capi.PhiError) as e:
        Hierarchy(p, max_nodes=1000)
    assert e.value.code == capi.PHI_E_BUDGET
