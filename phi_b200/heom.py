"""Python binding of the HEOM integrator (tests, benchmarks, notebooks).

`PhiParameters` mirrors the fields of PHI's `struct PhiParameters`
(phi_parameters.h:32-122) that the propagation and steady-state paths read,
with the same names and the same conventions:

* `num_matsubara_terms` is K + 1, `hierarchy_truncation_level` is L + 1;
* matrices are complex N x N numpy arrays (indexed [row, col]); they are
  passed to the library column-major, as PHI stores them;
* `bath_coupling_op` is (num_baths, N) for diagonal coupling
  (`CorrelatedCouplingTerms`) or (num_baths, N, N) for `FullBathTerms`.

`Hierarchy` owns one device context (one hierarchy instance on one GPU).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import capi

HBAR = 5.3088354   # cm^-1 ps   (phi_parameters.h:13-14)
K_B = 0.6950344    # cm^-1 / K  (phi_parameters.h:15-16)


@dataclass
class PhiParameters:
    num_states: int = 0
    time_indepenent_hamiltonian: Optional[np.ndarray] = None  # (sic), as in PHI
    num_bath_couplings: int = 0
    num_matsubara_terms: int = 1
    hierarchy_truncation_level: int = 1
    gamma: Optional[np.ndarray] = None
    lambda_: Optional[np.ndarray] = None
    bath_coupling_op: Optional[np.ndarray] = None
    is_diagonal_bath_coupling: bool = False
    is_full_bath_coupling: bool = False
    bath_sites: Optional[np.ndarray] = None
    initial_density_matrix: Optional[np.ndarray] = None
    temperature: float = 300.0
    hbar: float = HBAR
    boltzmann_constant: float = K_B
    is_rho_normalized: bool = True
    timestep: float = 0.001
    integration_time: float = 0.0
    output_minimum_timestep: float = 0.01
    rkf45_tolerance: float = 1e-6
    rkf45_minimum_timestep: float = 1e-6
    bicgstab_tolerance: float = 1e-6
    filter_tolerance: float = 0.0
    use_time_local_truncation: bool = False
    # Annealing Hamiltonian (time_indepenent_hamiltonian None):
    # H(t) = f_x(t/T) H_X + f_z(t/T) H_Z, f_x / f_z cubic splines through the
    # field samples on [0, 1], T = integration_time.
    transverse_hamiltonian: Optional[np.ndarray] = None    # H_X
    longitudinal_hamiltonian: Optional[np.ndarray] = None  # H_Z
    transverse_field: Optional[np.ndarray] = None
    longitudinal_field: Optional[np.ndarray] = None
    minimum_field_change: float = 0.01
    # Hilbert-space truncation: > num_states gives the Hamiltonian, the
    # initial density matrix and the full bath operators in this larger space
    # (PHI's HilbertSpaceSize); the hierarchy keeps the lowest num_states
    # eigenvectors of the Hamiltonian.  0 = no truncation.
    hilbert_space_size: int = 0

    @property
    def bath_kind(self) -> int:
        if self.is_full_bath_coupling:
            return capi.PHI_BATH_FULL
        if self.is_diagonal_bath_coupling:
            return capi.PHI_BATH_DIAGONAL
        return capi.PHI_BATH_INDEPENDENT

    @property
    def num_terms(self) -> int:
        return self.num_bath_couplings * self.num_matsubara_terms

    def fix_incompatible_combinations(self, method: str) -> None:
        """RKF45 and the steady-state solver force normalised ADOs
        (FixIncompatibleCombinations, phi_parameters.cc:817-829)."""
        if method in ("rkf45", "bicgstab", "steady"):
            self.is_rho_normalized = True


def col_major(m: np.ndarray) -> np.ndarray:
    """Complex N x N matrix -> interleaved column-major doubles."""
    m = np.asarray(m, dtype=np.complex128)
    return np.ascontiguousarray(m.T).view(np.float64).reshape(-1).copy()


def from_col_major(buf: np.ndarray, n: int) -> np.ndarray:
    """Interleaved column-major doubles -> complex N x N matrix."""
    return np.asarray(buf, dtype=np.float64).view(np.complex128).reshape(n, n).T.copy()


def state_to_matrices(state: np.ndarray, n: int) -> np.ndarray:
    """Node-major hierarchy state (2*M*N*N doubles) -> (M, N, N) complex."""
    s = np.asarray(state, dtype=np.float64).view(np.complex128).reshape(-1, n, n)
    return np.transpose(s, (0, 2, 1)).copy()


def matrices_to_state(mats: np.ndarray) -> np.ndarray:
    m = np.asarray(mats, dtype=np.complex128)
    return np.ascontiguousarray(np.transpose(m, (0, 2, 1))).view(np.float64).reshape(-1).copy()


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def problem_desc(p: PhiParameters, precision: int, device: int, max_nodes: int, keep_list: list):
    """phi_problem_desc of a PhiParameters; the arrays it points to are
    appended to keep_list (the caller keeps them alive)."""
    n = int(p.num_states)
    hs = int(p.hilbert_space_size or 0)
    if hs > n:
        n = hs  # matrices are given in the full space
    d = capi.PhiProblemDesc()
    d.hilbert_space_size = hs
    d.num_states = int(p.num_states)
    d.num_baths = int(p.num_bath_couplings)
    d.num_matsubara_terms = int(p.num_matsubara_terms)
    d.truncation_level = int(p.hierarchy_truncation_level)
    d.bath_kind = p.bath_kind
    d.normalized = 1 if p.is_rho_normalized else 0
    d.hbar = float(p.hbar)
    d.boltzmann_constant = float(p.boltzmann_constant)
    d.temperature = float(p.temperature)

    def keep(a, dtype=np.float64):
        a = np.ascontiguousarray(np.asarray(a, dtype=dtype).reshape(-1))
        keep_list.append(a)
        return a

    if p.transverse_hamiltonian is not None:
        # Annealing: H(t) = f_x(t/T) H_X + f_z(t/T) H_Z.
        d.annealing_h_x = _dptr(keep(col_major(p.transverse_hamiltonian)))
        d.annealing_h_z = _dptr(keep(col_major(p.longitudinal_hamiltonian)))
        fx, fz = keep(p.transverse_field), keep(p.longitudinal_field)
        d.transverse_field, d.transverse_field_size = _dptr(fx), fx.size
        d.longitudinal_field, d.longitudinal_field_size = _dptr(fz), fz.size
        d.integration_time = float(p.integration_time)
        d.minimum_field_change = float(p.minimum_field_change)
    else:
        d.hamiltonian = _dptr(keep(col_major(p.time_indepenent_hamiltonian)))
    d.initial_density_matrix = _dptr(keep(col_major(p.initial_density_matrix)))
    d.gamma = _dptr(keep(p.gamma))
    d.lambda_ = _dptr(keep(p.lambda_))
    if p.bath_coupling_op is not None and p.bath_kind != capi.PHI_BATH_INDEPENDENT:
        v = np.asarray(p.bath_coupling_op, dtype=np.float64)
        if p.bath_kind == capi.PHI_BATH_FULL:
            # (nb, N, N) [row, col] -> per-bath column-major
            v = np.ascontiguousarray(np.transpose(v.reshape(-1, n, n), (0, 2, 1)))
        d.coupling = _dptr(keep(v))
    if p.bath_sites is not None:
        s = keep(p.bath_sites, np.int32)
        d.bath_sites = s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    d.precision = precision
    d.device = device
    d.max_nodes = max_nodes
    d.filter_tolerance = float(p.filter_tolerance or 0.0)
    d.time_local = 1 if p.use_time_local_truncation else 0
    return d


class Hierarchy:
    """One hierarchy instance on one GPU (a phi_ctx)."""

    def __init__(self, p: PhiParameters, precision: int = capi.PHI_PREC_FP64,
                 device: int = 0, max_nodes: int = 0):
        self.lib = capi.load()
        self.n = int(p.num_states)
        self._keep = []
        d = problem_desc(p, precision, device, max_nodes, self._keep)
        ctx = ctypes.c_void_p()
        capi.check(self.lib.phi_gpu_create(ctypes.byref(d), ctypes.byref(ctx)))
        self.ctx = ctx
        self._read_dims()

    @classmethod
    def _borrowed(cls, lib, ctx) -> "Hierarchy":
        """View of a context owned elsewhere (a batch instance); close() does
        not destroy it."""
        self = cls.__new__(cls)
        self.lib = lib
        self._keep = []
        self.ctx = ctx
        self._owned = False
        self._read_dims()
        return self

    @classmethod
    def from_file(cls, path: str, method: str = "rk4", precision: int = capi.PHI_PREC_FP64,
                  device: int = 0) -> "Hierarchy":
        """Context from a PHI parameter file (PhiParameters::ReadCommandLine,
        phi_parameters.cc:93-146, then the library's scope checks)."""
        self = cls.__new__(cls)
        self.lib = capi.load()
        self._keep = []
        ctx = ctypes.c_void_p()
        capi.check(self.lib.phi_gpu_create_from_file(str(path).encode(), method.encode(), precision, device,
                                                     ctypes.byref(ctx)))
        self.ctx = ctx
        self._read_dims()
        return self

    def _read_dims(self):
        M = ctypes.c_int64()
        T = ctypes.c_int32()
        N = ctypes.c_int32()
        self._check(self.lib.phi_gpu_dims(self.ctx, ctypes.byref(M), ctypes.byref(T), ctypes.byref(N)))
        self.num_nodes = M.value
        self.num_terms = T.value
        self.n = N.value
        nb = ctypes.c_int32()
        self._check(self.lib.phi_gpu_num_baths(self.ctx, ctypes.byref(nb)))
        self.num_baths = nb.value

    def _check(self, code):
        capi.check(code, self.ctx)

    def close(self):
        if getattr(self, "ctx", None):
            if getattr(self, "_owned", True):
                self.lib.phi_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def state_len(self) -> int:
        return 2 * self.num_nodes * self.n * self.n

    def node_table(self):
        MT = self.num_nodes * self.num_terms
        mi = np.zeros(MT, np.int32)
        nx = np.zeros(MT, np.int32)
        pv = np.zeros(MT, np.int32)
        self._check(self.lib.phi_gpu_get_node_table(self.ctx, mi.ctypes.data, nx.ctypes.data, pv.ctypes.data))
        shape = (self.num_nodes, self.num_terms)
        return mi.reshape(shape), nx.reshape(shape), pv.reshape(shape)

    def get_state(self) -> np.ndarray:
        out = np.zeros(self.state_len, np.float64)
        self._check(self.lib.phi_gpu_get_state(self.ctx, out.ctypes.data))
        return out

    def set_state(self, state: np.ndarray) -> None:
        s = np.ascontiguousarray(state, dtype=np.float64)
        assert s.size == self.state_len
        self._check(self.lib.phi_gpu_set_state(self.ctx, s.ctypes.data))

    def active(self) -> np.ndarray:
        """Adaptive-filtering flags of the current state (M bools; all True
        when filtering is off)."""
        out = np.zeros(self.num_nodes, np.uint8)
        self._check(self.lib.phi_gpu_get_active(self.ctx, out.ctypes.data))
        return out.astype(bool)

    def time_local(self) -> np.ndarray:
        """Time-local truncation sums Q_m, (num_baths, N, N) complex in PHI's
        column-major storage (element [m, j, i] = Q_m[i, j]); zeros when
        off."""
        nb = self.num_baths
        out = np.zeros(2 * nb * self.n * self.n, np.float64)
        self._check(self.lib.phi_gpu_get_time_local(self.ctx, out.ctypes.data))
        return out.view(np.complex128).reshape(nb, self.n, self.n)

    def hamiltonian(self) -> np.ndarray:
        """The Hamiltonian the next stage starts from (N x N complex)."""
        out = np.zeros(2 * self.n * self.n, np.float64)
        self._check(self.lib.phi_gpu_get_hamiltonian(self.ctx, out.ctypes.data))
        return from_col_major(out, self.n)

    def rho0_full(self) -> np.ndarray:
        """rho_0 in the full Hilbert space (V rho_0 V^+ under Hilbert-space
        truncation; rho0() otherwise), F x F complex."""
        F = ctypes.c_int32()
        self._check(self.lib.phi_gpu_hilbert_space_size(self.ctx, ctypes.byref(F)))
        out = np.zeros(2 * F.value * F.value, np.float64)
        self._check(self.lib.phi_gpu_get_rho0_full(self.ctx, out.ctypes.data))
        return from_col_major(out, F.value)

    def rho0(self) -> np.ndarray:
        out = np.zeros(2 * self.n * self.n, np.float64)
        self._check(self.lib.phi_gpu_get_rho0(self.ctx, out.ctypes.data))
        return from_col_major(out, self.n)

    def apply(self, state: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=np.float64)
        assert s.size == self.state_len
        out = np.zeros_like(s)
        self._check(self.lib.phi_gpu_apply(self.ctx, s.ctypes.data, out.ctypes.data))
        return out

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        self._check(self.lib.phi_gpu_get_time(self.ctx, ctypes.byref(t)))
        return t.value

    @time.setter
    def time(self, v: float) -> None:
        self._check(self.lib.phi_gpu_set_time(self.ctx, float(v)))

    def rk4(self, dt: float, t_end: float, output_min_step: float = 0.0, capacity: int = 0):
        """Returns (steps, times, rho_0 rows as (k, N, N) complex)."""
        E2 = 2 * self.n * self.n
        traj = np.zeros(max(capacity, 1) * E2, np.float64)
        times = np.zeros(max(capacity, 1), np.float64)
        ns = ctypes.c_int64()
        no = ctypes.c_int64()
        self._check(self.lib.phi_gpu_rk4(
            self.ctx, float(dt), float(t_end), float(output_min_step),
            traj.ctypes.data if capacity else None, times.ctypes.data if capacity else None,
            int(capacity), ctypes.byref(ns), ctypes.byref(no)))
        k = min(no.value, capacity)
        rows = np.stack([from_col_major(traj[r * E2:(r + 1) * E2], self.n) for r in range(k)]) if k else \
            np.zeros((0, self.n, self.n), np.complex128)
        return ns.value, times[:k].copy(), rows

    def rkf45(self, dt0: float, t_end: float, tol: float, min_dt: float, max_steps: int = 0):
        st = capi.PhiRkf45Stats()
        self._check(self.lib.phi_gpu_rkf45(self.ctx, float(dt0), float(t_end), float(tol),
                                           float(min_dt), int(max_steps), ctypes.byref(st)))
        return {"steps": st.steps, "accepted": st.accepted, "final_time": st.final_time,
                "final_dt": st.final_dt, "max_error": st.max_error}

    def rkf45_advance(self, dt0: float, t_end: float, tol: float, min_dt: float, steps: int):
        """Exactly `steps` attempted steps (fewer at t_end); dt0 <= 0 continues."""
        st = capi.PhiRkf45Stats()
        self._check(self.lib.phi_gpu_rkf45_advance(self.ctx, float(dt0), float(t_end), float(tol),
                                                   float(min_dt), int(steps), ctypes.byref(st)))
        return {"steps": st.steps, "accepted": st.accepted, "final_time": st.final_time,
                "final_dt": st.final_dt, "max_error": st.max_error}

    def _restart_check(self, rc):
        if rc != capi.PHI_OK:
            raise capi.PhiError(rc, capi.restart_last_error() or capi.last_error(self.ctx))

    def write_restart(self, path: str, timestep: float) -> None:
        """PHI restart file of the state and time (17 significant digits)."""
        self._restart_check(self.lib.phi_gpu_write_restart(self.ctx, str(path).encode(), float(timestep)))

    def read_restart(self, path: str) -> float:
        """State and time from a PHI restart file; returns its step size."""
        dt = ctypes.c_double()
        self._restart_check(self.lib.phi_gpu_read_restart(self.ctx, str(path).encode(), ctypes.byref(dt)))
        return dt.value

    def save_state(self, path: str, timestep: float = 0.0) -> None:
        """Binary state file (exact)."""
        self._restart_check(self.lib.phi_gpu_save_state(self.ctx, str(path).encode(), float(timestep)))

    def load_state(self, path: str) -> float:
        dt = ctypes.c_double()
        self._restart_check(self.lib.phi_gpu_load_state(self.ctx, str(path).encode(), ctypes.byref(dt)))
        return dt.value

    def tile_schedule(self) -> dict:
        """The tiled kernel's schedule (block size, CTAs per SM cap; threads 0
        when the problem runs on the generic kernel) and the apply times the
        autotuner measured for it and for the default."""
        s = capi.PhiTileSchedule()
        self._check(self.lib.phi_gpu_get_tile_schedule(self.ctx, ctypes.byref(s)))
        return {"threads": s.threads, "ctas_per_sm": s.ctas_per_sm, "ms_per_apply": s.ms_per_apply,
                "ms_per_apply_default": s.ms_per_apply_default}

    def set_tile_schedule(self, threads: int, ctas_per_sm: int = 0) -> None:
        self._check(self.lib.phi_gpu_set_tile_schedule(self.ctx, int(threads), int(ctas_per_sm)))

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.phi_gpu_stream(self.ctx, ctypes.byref(s)))
        return s.value or 0

    def reset(self, time: float = 0.0) -> None:
        """Initial state (rho(0) in node 0) restored on the device, time set."""
        self._check(self.lib.phi_gpu_reset(self.ctx, float(time)))

    def steady_state(self, tol: float = 1e-10, ell: int = 2, max_steps: int = 0, guess=None,
                     tol_mode: int = capi.PHI_TOL_RELATIVE, check: bool = True, rho0_guess=None):
        """BiCGSTAB(ell) steady state (L rho = 0, tr rho_0 = 1); the context
        state becomes the solution.  tol_mode: PHI_TOL_RELATIVE
        (||r|| <= tol ||b||), PHI_TOL_ABSOLUTE (||r|| <= tol) or
        PHI_TOL_ABS_SQUARED (||r||^2 <= tol).  rho0_guess (N x N complex)
        starts from that rho_0 with every other node zero."""
        st = capi.PhiSolveStats()
        if rho0_guess is not None:
            g = col_major(rho0_guess)
            rc = self.lib.phi_gpu_steady_state_rho0(self.ctx, int(ell), float(tol), int(tol_mode),
                                                    int(max_steps), g.ctypes.data, ctypes.byref(st))
        else:
            g = None
            if guess is not None:
                g = np.ascontiguousarray(guess, dtype=np.float64)
                assert g.size == self.state_len
            rc = self.lib.phi_gpu_steady_state(self.ctx, int(ell), float(tol), int(tol_mode), int(max_steps),
                                               g.ctypes.data if g is not None else None, ctypes.byref(st))
        if check:
            self._check(rc)
        return {"steps": st.iterations, "converged": bool(st.converged), "residual": st.residual,
                "seconds": st.seconds, "status": rc, "deflated_tiers": st.deflated_tiers,
                "deflation_size": st.deflation_size}

    def set_steady_deflation(self, tiers: int) -> None:
        """Deflation of the steady-state solves by the ADOs of tiers
        0..tiers-1: -1 automatic (the default), 0 off (PHI's plain
        BiCGSTAB(ell)), 1 rho_0, 2 rho_0 and the first tier."""
        self._check(self.lib.phi_gpu_set_steady_deflation(self.ctx, int(tiers)))


class Batch:
    """Many independent hierarchies integrated together (a phi_batch): every
    RK4 stage of all instances is one persistent kernel launch."""

    def __init__(self, problems, precision: int = capi.PHI_PREC_FP64, device: int = 0):
        self.lib = capi.load()
        self._keep = []
        arr = (capi.PhiProblemDesc * len(problems))()
        for i, p in enumerate(problems):
            arr[i] = problem_desc(p, precision, device, 0, self._keep)
        b = ctypes.c_void_p()
        capi.check_batch(self.lib.phi_gpu_batch_create(arr, len(problems), ctypes.byref(b)))
        self.batch = b
        self.count = len(problems)
        self.instances = []
        for i in range(self.count):
            c = ctypes.c_void_p()
            self._check(self.lib.phi_gpu_batch_instance(self.batch, i, ctypes.byref(c)))
            self.instances.append(Hierarchy._borrowed(self.lib, c))

    def _check(self, code):
        capi.check_batch(code, self.batch)

    def close(self):
        if getattr(self, "batch", None):
            for h in self.instances:
                h.close()
            self.lib.phi_gpu_batch_destroy(self.batch)
            self.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __getitem__(self, i) -> Hierarchy:
        return self.instances[i]

    @property
    def total_nodes(self) -> int:
        return sum(h.num_nodes for h in self.instances)

    def autotune(self) -> dict:
        s = capi.PhiBatchSchedule()
        self._check(self.lib.phi_gpu_batch_autotune(self.batch, ctypes.byref(s)))
        return {"ctas_per_sm": s.ctas_per_sm, "order": s.order, "ms_per_stage": s.ms_per_stage}

    def set_schedule(self, ctas_per_sm: int, order: int):
        s = capi.PhiBatchSchedule(ctas_per_sm, order, 0.0)
        self._check(self.lib.phi_gpu_batch_set_schedule(self.batch, ctypes.byref(s)))

    def rk4(self, dt: float, steps: int) -> dict:
        st = capi.PhiBatchStats()
        self._check(self.lib.phi_gpu_batch_rk4(self.batch, float(dt), int(steps), ctypes.byref(st)))
        return {"steps": st.steps, "node_applies": st.node_applies, "seconds": st.seconds,
                "launches": st.launches}
