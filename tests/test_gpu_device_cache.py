"""Device memory of destroyed contexts is kept for the next context of the
same shape in the process (device_cache.cpp) and returned to the driver by
phi_gpu_release_cached_memory; a context built from reused blocks computes
the same result as one built from fresh ones."""
import numpy as np
import pytest

from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy

pytestmark = pytest.mark.gpu


def _run():
    p = configs.frenkel7(depth=3)
    p.fix_incompatible_combinations("rkf45")
    with Hierarchy(p, precision=capi.PHI_PREC_MIXED) as h:
        h.rkf45(0.001, 0.02, 1e-6, 1e-6)
        return h.get_state()


def test_cache_reuse_and_release():
    lib = capi.load()
    lib.phi_gpu_release_cached_memory()
    first = _run()                        # fresh blocks, cached at destroy
    cached = lib.phi_gpu_release_cached_memory()
    assert cached > 0
    assert lib.phi_gpu_release_cached_memory() == 0
    again = _run()                        # fresh blocks again
    reused = _run()                       # the blocks of `again`, with its stale contents
    assert np.array_equal(first, again)
    assert np.array_equal(again, reused)
