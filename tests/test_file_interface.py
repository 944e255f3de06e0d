"""Parameter-file errors are reported before any device work (CPU):
PhiParameters marks the input invalid and phi_gpu_create_from_file returns
PHI_E_INVALID with the reason in phi_gpu_last_error(NULL, ...)."""
import pytest

from oracle import oracle as O
from phi_b200 import capi, configs
from phi_b200.heom import Hierarchy


def _write(tmp_path, text):
    f = tmp_path / "params.txt"
    f.write_text(text)
    return str(f)


def test_malformed_file_is_rejected(tmp_path):
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy.from_file(_write(tmp_path, "NumStates=2\nHamiltonian:\n0 1\n1 0\n"), "rk4")


def test_unknown_method_is_rejected(tmp_path):
    text = O.param_file_text(configs.spin_boson())
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy.from_file(_write(tmp_path, text), "no_such_method")


def test_time_local_outside_identity_map_is_rejected(tmp_path):
    """TimeLocal with independent baths on another site map
    (DiagonalCouplingIndices): PHI adds c at (b, b) whatever site bath b
    couples to, so the library refuses the input instead of guessing."""
    import cases
    p = cases.random_problem("independent", n=3, matsubara=2, truncation=3, seed=1)
    text = O.param_file_text(p) + "TimeLocal=1\nDiagonalCouplingIndices:\n0,2,1\n"
    with pytest.raises(capi.PhiError, match="PHI_E_INVALID"):
        Hierarchy.from_file(_write(tmp_path, text), "rkf45")
