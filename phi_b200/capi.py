"""ctypes binding of the C ABI declared in include/phi_b200.h.

The shared library is built in-tree (phi_b200/libphi_b200.so).  There is no
fallback: if the library is missing or does not load, every entry point
raises, so nothing can silently run on the CPU.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libphi_b200.so")

PHI_OK = 0
PHI_E_INVALID = 1
PHI_E_OOM = 2
PHI_E_BUDGET = 3
PHI_E_STEP_COLLAPSE = 4
PHI_E_NO_CONVERGENCE = 5
PHI_E_TIMEOUT = 6
PHI_E_CUDA = 7
PHI_E_STATE = 8
PHI_E_NUMERIC = 9

STATUS_NAMES = {
    0: "PHI_OK", 1: "PHI_E_INVALID", 2: "PHI_E_OOM", 3: "PHI_E_BUDGET",
    4: "PHI_E_STEP_COLLAPSE", 5: "PHI_E_NO_CONVERGENCE", 6: "PHI_E_TIMEOUT",
    7: "PHI_E_CUDA", 8: "PHI_E_STATE", 9: "PHI_E_NUMERIC",
}

PHI_BATH_INDEPENDENT = 0
PHI_BATH_DIAGONAL = 1
PHI_BATH_FULL = 2

PHI_PREC_FP64 = 0
PHI_PREC_MIXED = 1
PHI_TOL_RELATIVE = 0
PHI_TOL_ABSOLUTE = 1
PHI_TOL_ABS_SQUARED = 2


class PhiProblemDesc(ctypes.Structure):
    """Mirror of phi_problem_desc."""
    _fields_ = [
        ("num_states", c_int32),
        ("num_baths", c_int32),
        ("num_matsubara_terms", c_int32),
        ("truncation_level", c_int32),
        ("bath_kind", c_int32),
        ("normalized", c_int32),
        ("hbar", c_double),
        ("boltzmann_constant", c_double),
        ("temperature", c_double),
        ("hamiltonian", POINTER(c_double)),
        ("gamma", POINTER(c_double)),
        ("lambda_", POINTER(c_double)),
        ("coupling", POINTER(c_double)),
        ("bath_sites", POINTER(c_int32)),
        ("initial_density_matrix", POINTER(c_double)),
        ("precision", c_int32),
        ("device", c_int32),
        ("max_nodes", c_int64),
        ("filter_tolerance", c_double),
        ("time_local", c_int32),
        ("annealing_h_x", POINTER(c_double)),
        ("annealing_h_z", POINTER(c_double)),
        ("transverse_field", POINTER(c_double)),
        ("transverse_field_size", c_int32),
        ("longitudinal_field", POINTER(c_double)),
        ("longitudinal_field_size", c_int32),
        ("integration_time", c_double),
        ("minimum_field_change", c_double),
        ("hilbert_space_size", c_int32),
    ]


class PhiRkf45Stats(ctypes.Structure):
    _fields_ = [
        ("steps", c_int64),
        ("accepted", c_int64),
        ("final_time", c_double),
        ("final_dt", c_double),
        ("max_error", c_double),
    ]


class PhiTileSchedule(ctypes.Structure):
    _fields_ = [
        ("threads", c_int32),
        ("ctas_per_sm", c_int32),
        ("ms_per_apply", c_double),
        ("ms_per_apply_default", c_double),
    ]


class PhiSolveStats(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("residual", c_double),
        ("seconds", c_double),
        ("deflated_tiers", c_int32),
        ("deflation_size", c_int32),
    ]


class PhiBatchSchedule(ctypes.Structure):
    _fields_ = [
        ("ctas_per_sm", c_int32),
        ("order", c_int32),
        ("ms_per_stage", c_double),
    ]


class PhiBatchStats(ctypes.Structure):
    _fields_ = [
        ("steps", c_int64),
        ("node_applies", c_int64),
        ("seconds", c_double),
        ("launches", c_int64),
    ]


# (name, restype, argtypes) for every entry point of include/phi_b200.h.
SIGNATURES = [
    ("phi_gpu_create", c_int, [POINTER(PhiProblemDesc), POINTER(c_void_p)]),
    ("phi_gpu_create_from_file", c_int, [c_char_p, c_char_p, c_int32, c_int32, POINTER(c_void_p)]),
    ("phi_gpu_destroy", c_int, [c_void_p]),
    ("phi_gpu_dims", c_int, [c_void_p, POINTER(c_int64), POINTER(c_int32), POINTER(c_int32)]),
    ("phi_gpu_get_rho0_full", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_hilbert_space_size", c_int, [c_void_p, POINTER(c_int32)]),
    ("phi_gpu_get_tile_schedule", c_int, [c_void_p, POINTER(PhiTileSchedule)]),
    ("phi_gpu_set_tile_schedule", c_int, [c_void_p, c_int32, c_int32]),
    ("phi_gpu_num_baths", c_int, [c_void_p, POINTER(c_int32)]),
    ("phi_gpu_get_node_table", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("phi_gpu_set_state", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_get_state", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_get_rho0", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_get_active", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_get_time_local", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_get_hamiltonian", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_release_cached_memory", c_int64, []),
    ("phi_gpu_apply", c_int, [c_void_p, c_void_p, c_void_p]),
    ("phi_gpu_apply_device", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("phi_gpu_rk4", c_int, [c_void_p, c_double, c_double, c_double, c_void_p, c_void_p, c_int64,
                            POINTER(c_int64), POINTER(c_int64)]),
    ("phi_gpu_rkf45", c_int, [c_void_p, c_double, c_double, c_double, c_double, c_int64,
                              POINTER(PhiRkf45Stats)]),
    ("phi_gpu_rkf45_advance", c_int, [c_void_p, c_double, c_double, c_double, c_double, c_int64,
                                      POINTER(PhiRkf45Stats)]),
    ("phi_gpu_stream", c_int, [c_void_p, POINTER(c_void_p)]),
    ("phi_gpu_steady_state", c_int, [c_void_p, c_int32, c_double, c_int32, c_int32, c_void_p,
                                      POINTER(PhiSolveStats)]),
    ("phi_gpu_set_steady_deflation", c_int, [c_void_p, c_int32]),
    ("phi_gpu_get_time", c_int, [c_void_p, POINTER(c_double)]),
    ("phi_gpu_set_time", c_int, [c_void_p, c_double]),
    ("phi_gpu_reset", c_int, [c_void_p, c_double]),
    ("phi_gpu_rk4_step_noalloc", c_int, [c_void_p, c_void_p, c_void_p, c_double, c_void_p]),
    ("phi_gpu_check_device_flag", c_int, [c_void_p, c_void_p]),
    ("phi_gpu_debug_set_wait_limit", c_int, [c_void_p, c_int64]),
    ("phi_gpu_debug_set_rkf45_replay", c_int, [c_void_p, c_void_p, c_int64, c_int64]),
    ("phi_gpu_debug_get_rkf45_errors", c_int, [c_void_p, c_void_p, c_int64, POINTER(c_int64)]),
    ("phi_gpu_last_error", c_int, [c_void_p, c_char_p, c_size_t]),
    ("phi_restart_read_file", c_int, [c_char_p, c_int32, c_int64, c_void_p, POINTER(c_double), POINTER(c_double)]),
    ("phi_restart_write_file", c_int, [c_char_p, c_int32, c_int64, c_void_p, c_double, c_double]),
    ("phi_restart_read_file_ex", c_int, [c_char_p, c_int32, c_int64, c_void_p, POINTER(c_double),
                                         POINTER(c_double), c_void_p, c_int64]),
    ("phi_restart_write_file_ex", c_int, [c_char_p, c_int32, c_int64, c_void_p, c_double, c_double, c_void_p,
                                          c_int64]),
    ("phi_restart_last_error", c_int, [c_char_p, c_size_t]),
    ("phi_gpu_write_restart", c_int, [c_void_p, c_char_p, c_double]),
    ("phi_gpu_read_restart", c_int, [c_void_p, c_char_p, POINTER(c_double)]),
    ("phi_gpu_save_state", c_int, [c_void_p, c_char_p, c_double]),
    ("phi_gpu_load_state", c_int, [c_void_p, c_char_p, POINTER(c_double)]),
    ("phi_gpu_batch_create", c_int, [POINTER(PhiProblemDesc), c_int32, POINTER(c_void_p)]),
    ("phi_gpu_batch_destroy", c_int, [c_void_p]),
    ("phi_gpu_batch_instance", c_int, [c_void_p, c_int32, POINTER(c_void_p)]),
    ("phi_gpu_batch_autotune", c_int, [c_void_p, POINTER(PhiBatchSchedule)]),
    ("phi_gpu_batch_set_schedule", c_int, [c_void_p, POINTER(PhiBatchSchedule)]),
    ("phi_gpu_batch_rk4", c_int, [c_void_p, c_double, c_int64, POINTER(PhiBatchStats)]),
    ("phi_gpu_batch_last_error", c_int, [c_void_p, c_char_p, c_size_t]),
    ("phi_nn_linear_forward", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                      c_int32, c_void_p]),
    ("phi_nn_linear_backward", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_int32, c_int32, c_int32, c_int32, c_void_p]),
    ("phi_nn_mse", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p]),
    ("phi_nn_adam", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, ctypes.c_float,
                            ctypes.c_float, ctypes.c_float, ctypes.c_float, c_int32, c_void_p]),
    ("phi_nn_to_bf16", c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    ("phi_gpu_steady_state_rho0", c_int, [c_void_p, c_int32, c_double, c_int32, c_int32, c_void_p,
                                           POINTER(PhiSolveStats)]),
]

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the in-tree library once; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"phi_b200 native library not found at {path}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C phi_b200/csrc`")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        if not hasattr(lib, name):
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class PhiError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def last_error(ctx=None) -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.phi_gpu_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


def check(code: int, ctx=None) -> None:
    if code != PHI_OK:
        raise PhiError(code, last_error(ctx))


def restart_last_error() -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.phi_restart_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def restart_read(path: str, num_states: int, num_nodes: int):
    """PHI restart file -> (state as 2*M*N*N doubles, time, step size)."""
    import numpy as np
    lib = load()
    st = np.zeros(2 * num_nodes * num_states * num_states)
    t, dt = c_double(), c_double()
    rc = lib.phi_restart_read_file(str(path).encode(), num_states, num_nodes, st.ctypes.data, ctypes.byref(t),
                                   ctypes.byref(dt))
    if rc != PHI_OK:
        raise PhiError(rc, restart_last_error())
    return st, t.value, dt.value


def restart_write(path: str, num_states: int, num_nodes: int, state, time: float, timestep: float):
    import numpy as np
    lib = load()
    st = np.ascontiguousarray(state, dtype=np.float64)
    assert st.size == 2 * num_nodes * num_states * num_states
    rc = lib.phi_restart_write_file(str(path).encode(), num_states, num_nodes, st.ctypes.data, float(time),
                                    float(timestep))
    if rc != PHI_OK:
        raise PhiError(rc, restart_last_error())


def batch_last_error(batch=None) -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.phi_gpu_batch_last_error(batch, buf, 1024)
    return buf.value.decode(errors="replace")


def check_batch(code: int, batch=None) -> None:
    if code != PHI_OK:
        raise PhiError(code, batch_last_error(batch))
