"""phi_b200 -- B200-native integrator for PHI's hierarchy equations of motion.

The product is the native library phi_b200/libphi_b200.so (C ABI in
include/phi_b200.h, C++ facade in include/phi/).  This package is the Python
binding of that library; it does no numerical work itself.
"""
from . import capi
from .heom import (HBAR, K_B, Hierarchy, PhiParameters, col_major, from_col_major,
                   matrices_to_state, state_to_matrices)

__all__ = ["capi", "Hierarchy", "PhiParameters", "HBAR", "K_B", "col_major",
           "from_col_major", "state_to_matrices", "matrices_to_state"]
