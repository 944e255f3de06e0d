"""The tile-kernel schedule: the autotuner at context creation (block size
variant x persistent CTAs per SM, timed on one Liouvillian apply) and the
manual override.  Every schedule gives the same results bit for bit: each
element's arithmetic does not depend on the tile it falls in."""
import numpy as np
import pytest

import cases
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu

ALT = {7: 320, 24: 256}


def _run(p, precision, threads, cps):
    with Hierarchy(p, precision=precision) as h:
        default = h.tile_schedule()["threads"]
        h.set_tile_schedule(threads or default, cps)
        st = h.rkf45(0.001, 0.01, 1e-6, 1e-6)
        return h.get_state(), st["steps"]


@pytest.mark.parametrize("make,n", [(lambda: configs.frenkel7(depth=3), 7), (lambda: configs.ring24(depth=2), 24)],
                         ids=["frenkel7_L3", "ring24_L2"])
@pytest.mark.parametrize("precision", [capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED], ids=["fp64", "mixed"])
def test_every_schedule_gives_the_same_bits(make, n, precision):
    p = make()
    p.fix_incompatible_combinations("rkf45")
    ref, steps = _run(p, precision, 0, 0)
    with Hierarchy(p, precision=precision) as h:
        sizes = {h.tile_schedule()["threads"]}
    other = (320 if 256 in sizes else 256)
    for threads, cps in [(other, 0), (0, 1), (other, 1)]:
        got, s2 = _run(p, precision, threads, cps)
        assert s2 == steps
        assert np.array_equal(got, ref), (threads, cps)


def test_autotuned_schedule_is_reported():
    p = configs.frenkel7()  # 38,760 nodes of 7x7: tuned at creation
    with Hierarchy(p, precision=capi.PHI_PREC_MIXED) as h:
        s = h.tile_schedule()
    assert s["threads"] in (256, 320)
    assert s["ctas_per_sm"] >= 0
    assert 0 < s["ms_per_apply"] <= s["ms_per_apply_default"]


def test_schedule_override_is_checked():
    p = configs.frenkel7(depth=3)
    with Hierarchy(p) as h:
        with pytest.raises(capi.PhiError) as e:
            h.set_tile_schedule(100, 0)
        assert e.value.code == capi.PHI_E_INVALID
    q = cases.random_problem("diagonal", n=3, matsubara=2, truncation=3, seed=1)
    with Hierarchy(q) as h:
        assert h.tile_schedule()["threads"] == 0  # generic kernel
        with pytest.raises(capi.PhiError):
            h.set_tile_schedule(256, 0)
