"""Batched uneven instances on the GPU: every RK4 stage of all instances in
one persistent launch (phi_gpu_batch_*).

* Each instance's state after the batch equals the state the same problem
  reaches alone in its own context, bit for bit (same tile arithmetic), in
  FP64 and in mixed precision, under every schedule.
* FP64 instances match the oracle's RK4 (Rk4Integrate,
  hierarchy_integrator.cc:2705-2826) within 1e-10.
* Mixed-precision rho_0 stays within 1e-6 of FP64.
"""
import numpy as np
import pytest

from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Batch, Hierarchy

pytestmark = pytest.mark.gpu

DT = 0.0005
STEPS = 40


def _small_batch(count=24, seed=11):
    # Uneven N, K and depth, budget 1 MiB per instance so the test is quick.
    return configs.batched(seed=seed, count=count, budget_bytes=2**20, depth_range=(2, 6))


def _alone(p, steps, precision=capi.PHI_PREC_FP64):
    with Hierarchy(p, precision=precision) as h:
        h.rk4(DT, (steps - 0.5) * DT)  # exactly `steps` steps of the reference loop
        return h.get_state(), h.time


@pytest.mark.parametrize("precision", [capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED], ids=["fp64", "mixed"])
def test_batch_equals_instances_alone(precision):
    probs = _small_batch()
    with Batch(probs, precision=precision) as b:
        st = b.rk4(DT, STEPS)
        got = [b[i].get_state() for i in range(b.count)]
        times = [b[i].time for i in range(b.count)]
    assert st["steps"] == STEPS and st["node_applies"] == 4 * STEPS * sum(p.nodes for p in probs)
    for i, p in enumerate(probs):
        ref, t = _alone(p, STEPS, precision)
        assert np.array_equal(got[i], ref), (i, p.name, np.abs(got[i] - ref).max())
        assert times[i] == t


def test_batch_matches_oracle():
    probs = _small_batch(count=8, seed=5)
    with Batch(probs) as b:
        b.rk4(DT, STEPS)
        got = [b[i].get_state() for i in range(b.count)]
    for i, p in enumerate(probs):
        o = O.Oracle(p)
        s, steps, _, _ = o.rk4(o.initial_state(), DT, (STEPS - 0.5) * DT)
        assert steps == STEPS
        assert np.abs(got[i] - s).max() <= 1e-10, (p.name, np.abs(got[i] - s).max())


def test_schedules_give_identical_results():
    probs = _small_batch(count=16, seed=21)
    results = []
    for cps, order in [(1, 0), (2, 1), (3, 0)]:
        with Batch(probs) as b:
            b.set_schedule(cps, order)
            b.rk4(DT, 20)  # > 16: graph replay plus direct tail steps
            results.append([b[i].get_state() for i in range(b.count)])
    for r in results[1:]:
        for a, c in zip(results[0], r):
            assert np.array_equal(a, c)


def test_autotune_keeps_state_and_picks_a_schedule():
    probs = _small_batch(count=16, seed=8)
    with Batch(probs) as b:
        before = [b[i].get_state() for i in range(b.count)]
        s = b.autotune()
        after = [b[i].get_state() for i in range(b.count)]
        assert s["ctas_per_sm"] >= 1 and s["order"] in (0, 1) and s["ms_per_stage"] > 0
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        b.rk4(DT, 4)


def test_mixed_rho0_within_1e6_of_fp64():
    probs = _small_batch(count=16, seed=13)
    with Batch(probs) as b:
        b.rk4(DT, 200)
        r64 = [b[i].rho0() for i in range(b.count)]
    with Batch(probs, precision=capi.PHI_PREC_MIXED) as b:
        b.rk4(DT, 200)
        r32 = [b[i].rho0() for i in range(b.count)]
    err = max(np.abs(a - c).max() for a, c in zip(r64, r32))
    assert err <= 1e-6, err


def test_batch_rejects_instances_without_tile_kernel():
    probs = _small_batch(count=3)
    probs.append(configs.spin_boson())  # DiagonalBath
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Batch(probs)


def test_batch_covers_every_tile_instantiation():
    """Instances of every tile-kernel N with K+1 = 1, 2 and 3 in one launch,
    each equal to its own context bit for bit."""
    import cases
    probs = []
    seed = 100
    for n in (2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 24):
        for k1 in (1, 2, 3):
            if n * k1 > 64:  # the library's limit on terms per hierarchy
                continue
            depth = 2 if n >= 10 or k1 == 3 else 3
            probs.append(cases.random_problem("independent", n=n, matsubara=k1, truncation=depth + 1,
                                              seed=seed))
            seed += 1
    with Batch(probs) as b:
        b.rk4(DT, 5)
        got = [b[i].get_state() for i in range(b.count)]
    for i, p in enumerate(probs):
        ref, _ = _alone(p, 5)
        assert np.array_equal(got[i], ref), (i, p.num_states, p.num_matsubara_terms)
