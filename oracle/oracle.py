"""Python access to the oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:

* the C restatement of the PHI path (heom_oracle.c -> _build/libheom_oracle.so);
* the reference PHI itself, built unchanged from its sources by
  refbuild/Makefile into _ref/ (ref_driver runs PhiParameters ->
  HierarchyIntegrator -> Launch -> density_matrix and prints %.17g).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libheom_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
# The reference built in BLAS mode (oracle/refbuild/Makefile `blas`): the
# configuration its Hilbert-space truncation is correct in.
REF_DRIVER_BLAS = os.path.join(HERE, "_ref_blas", "ref_driver")


class _Problem(ctypes.Structure):
    _fields_ = [
        ("num_states", c_int), ("num_baths", c_int), ("num_matsubara", c_int),
        ("truncation", c_int), ("bath_kind", c_int), ("normalized", c_int),
        ("hbar", c_double), ("kb", c_double), ("temperature", c_double),
        ("hamiltonian", POINTER(c_double)), ("gamma", POINTER(c_double)),
        ("lambda_", POINTER(c_double)), ("coupling", POINTER(c_double)),
        ("filter_tolerance", c_double),
        ("time_local", c_int),
        ("h_x", POINTER(c_double)), ("h_z", POINTER(c_double)),
        ("field_x", POINTER(c_double)), ("field_z", POINTER(c_double)),
        ("num_field_x", c_int), ("num_field_z", c_int),
        ("integration_time", c_double), ("min_field_change", c_double),
        ("hilbert_space_size", c_int),
    ]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE, "_build/libheom_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(LIB)
    lib.oracle_node_count.restype = c_int64
    lib.oracle_node_count.argtypes = [c_int, c_int]
    lib.oracle_build_hierarchy.restype = c_int64
    lib.oracle_build_hierarchy.argtypes = [c_int, c_int, c_void_p, c_int64]
    lib.oracle_create.restype = c_void_p
    lib.oracle_create.argtypes = [POINTER(_Problem)]
    lib.oracle_destroy.argtypes = [c_void_p]
    lib.oracle_num_nodes.restype = c_int64
    lib.oracle_num_nodes.argtypes = [c_void_p]
    lib.oracle_num_terms.restype = c_int
    lib.oracle_num_terms.argtypes = [c_void_p]
    lib.oracle_get_tables.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
    lib.oracle_get_constants.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.oracle_apply.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.oracle_initial_state.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.oracle_reset_filter.argtypes = [c_void_p]
    lib.oracle_reset_time_local.argtypes = [c_void_p]
    lib.oracle_reset_hamiltonian.argtypes = [c_void_p]
    lib.oracle_get_hamiltonian.argtypes = [c_void_p, c_void_p]
    lib.oracle_get_time_local.argtypes = [c_void_p, c_void_p]
    lib.oracle_get_active.argtypes = [c_void_p, c_void_p]
    lib.oracle_rk4.restype = c_int64
    lib.oracle_rk4.argtypes = [c_void_p, c_void_p, c_double, c_double, c_double, c_double,
                               c_void_p, c_void_p, c_int64, POINTER(c_int64)]
    lib.oracle_rkf45.restype = c_int64
    lib.oracle_rkf45.argtypes = [c_void_p, c_void_p, c_double, c_double, c_double, c_double,
                                 c_double, POINTER(c_int64), POINTER(c_double), POINTER(c_double)]
    lib.oracle_set_threads.restype = None
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.oracle_hilbert_space_size.restype = c_int
    lib.oracle_hilbert_space_size.argtypes = [c_void_p]
    lib.oracle_truncate.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.oracle_get_basis.argtypes = [c_void_p, c_void_p]
    lib.oracle_rkf45_trace.restype = c_int64
    lib.oracle_rkf45_trace.argtypes = [c_void_p, c_void_p, c_double, c_double, c_double, c_double,
                                       c_double, POINTER(c_int64), POINTER(c_double), POINTER(c_double),
                                       c_void_p, c_int64]
    _lib = lib
    return lib


def _colmajor(m):
    m = np.asarray(m, dtype=np.complex128)
    return np.ascontiguousarray(m.T).view(np.float64).reshape(-1).copy()


def _from_colmajor(buf, n):
    return np.asarray(buf).view(np.complex128).reshape(n, n).T.copy()


def bath_kind(p) -> int:
    if getattr(p, "is_full_bath_coupling", False):
        return 2
    if getattr(p, "is_diagonal_bath_coupling", False):
        return 1
    return 0


def node_count(T: int, truncation: int) -> int:
    return int(load().oracle_node_count(T, truncation))


def build_hierarchy(T: int, truncation: int) -> np.ndarray:
    """Hierarchy::ConstructI order: (M, T) multi-indices."""
    lib = load()
    M = node_count(T, truncation)
    mi = np.zeros(M * max(T, 1), np.int32)
    got = lib.oracle_build_hierarchy(T, truncation, mi.ctypes.data, M)
    assert got == M, (got, M)
    return mi.reshape(M, T)


class Oracle:
    """CPU restatement of one hierarchy instance (duck-typed PhiParameters)."""

    def __init__(self, p):
        self.lib = load()
        n = int(p.num_states)
        self.n = n
        self.num_baths = int(p.num_bath_couplings)
        self.p = p
        keep = []

        def arr(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
            keep.append(a)
            return a.ctypes.data_as(POINTER(c_double))

        pr = _Problem()
        pr.num_states = n
        # Hilbert-space truncation of an annealing Hamiltonian: operators are
        # F x F; the oracle keeps the basis (static truncation is restated in
        # the tests on the projected problem).
        hs = int(getattr(p, "hilbert_space_size", 0) or 0)
        annealing = getattr(p, "transverse_hamiltonian", None) is not None
        F = hs if (annealing and hs > n) else n
        self.F = F
        pr.num_baths = int(p.num_bath_couplings)
        pr.num_matsubara = int(p.num_matsubara_terms)
        pr.truncation = int(p.hierarchy_truncation_level)
        pr.bath_kind = bath_kind(p)
        pr.normalized = 1 if p.is_rho_normalized else 0
        pr.hbar = float(p.hbar)
        pr.kb = float(p.boltzmann_constant)
        pr.temperature = float(p.temperature)
        H0 = p.time_indepenent_hamiltonian
        pr.hamiltonian = arr(_colmajor(H0 if H0 is not None else np.zeros((n, n))))
        pr.gamma = arr(p.gamma)
        pr.lambda_ = arr(p.lambda_)
        if pr.bath_kind == 1:
            pr.coupling = arr(np.asarray(p.bath_coupling_op, np.float64))
        elif pr.bath_kind == 2:
            v = np.asarray(p.bath_coupling_op, np.float64).reshape(-1, F, F)
            pr.coupling = arr(np.transpose(v, (0, 2, 1)))
        # FixIncompatibleCombinations (phi_parameters.cc:847-851): filtering
        # only with independent baths.
        ft = float(getattr(p, "filter_tolerance", 0.0) or 0.0)
        pr.filter_tolerance = ft if pr.bath_kind == 0 else 0.0
        # Time-local truncation, restated for independent baths.
        pr.time_local = 1 if getattr(p, "use_time_local_truncation", False) else 0
        # Annealing Hamiltonian H(t) = f_x(t/T) H_X + f_z(t/T) H_Z.
        if getattr(p, "transverse_hamiltonian", None) is not None:
            pr.h_x = arr(_colmajor(np.asarray(p.transverse_hamiltonian, np.complex128)))
            pr.h_z = arr(_colmajor(np.asarray(p.longitudinal_hamiltonian, np.complex128)))
            fx = np.asarray(p.transverse_field, np.float64)
            fz = np.asarray(p.longitudinal_field, np.float64)
            pr.field_x, pr.field_z = arr(fx), arr(fz)
            pr.num_field_x, pr.num_field_z = fx.size, fz.size
            pr.integration_time = float(p.integration_time)
            pr.min_field_change = float(p.minimum_field_change)
            pr.hilbert_space_size = F
        self._keep = keep
        self.ctx = self.lib.oracle_create(ctypes.byref(pr))
        if not self.ctx:
            raise ValueError("oracle_create failed")
        self.M = int(self.lib.oracle_num_nodes(self.ctx))
        self.T = int(self.lib.oracle_num_terms(self.ctx))
        self.rho_init = _colmajor(p.initial_density_matrix)
        if F > n:
            out = np.zeros(2 * n * n)
            self.lib.oracle_truncate(self.ctx, self.rho_init.ctypes.data, out.ctypes.data)
            self.rho_init = out

    def __del__(self):
        if getattr(self, "ctx", None):
            self.lib.oracle_destroy(self.ctx)
            self.ctx = None

    @property
    def state_len(self):
        return 2 * self.M * self.n * self.n

    def tables(self):
        MT = self.M * self.T
        mi, nx, pv = (np.zeros(MT, np.int32) for _ in range(3))
        self.lib.oracle_get_tables(self.ctx, mi.ctypes.data, nx.ctypes.data, pv.ctypes.data)
        s = (self.M, self.T)
        return mi.reshape(s), nx.reshape(s), pv.reshape(s)

    def constants(self):
        corr = np.zeros(2 * self.T, np.float64)
        mats = np.zeros(int(self.p.num_bath_couplings), np.float64)
        self.lib.oracle_get_constants(self.ctx, corr.ctypes.data, mats.ctypes.data)
        return corr.view(np.complex128), mats

    def initial_state(self):
        s = np.zeros(self.state_len, np.float64)
        self.lib.oracle_initial_state(self.ctx, self.rho_init.ctypes.data, s.ctypes.data)
        return s

    def apply(self, state):
        s = np.ascontiguousarray(state, np.float64)
        out = np.zeros_like(s)
        self.lib.oracle_apply(self.ctx, s.ctypes.data, out.ctypes.data)
        return out

    def reset_filter(self):
        """Marks every node active (HierarchyNode::is_active)."""
        self.lib.oracle_reset_filter(self.ctx)

    def active(self):
        """Adaptive-filtering flags of the last integrated state (M bools)."""
        out = np.zeros(self.M, np.uint8)
        self.lib.oracle_get_active(self.ctx, out.ctypes.data)
        return out.astype(bool)

    def reset_run_state(self):
        """Filter flags, time-local matrices and the annealing Hamiltonian
        as a fresh PHI run has them."""
        self.reset_filter()
        self.reset_time_local()
        self.lib.oracle_reset_hamiltonian(self.ctx)

    def hamiltonian(self):
        """The current Hamiltonian (N x N complex)."""
        out = np.zeros(2 * self.n * self.n)
        self.lib.oracle_get_hamiltonian(self.ctx, out.ctypes.data)
        return _from_colmajor(out, self.n)

    def reset_time_local(self):
        """Zeroes the time-local truncation matrices (a fresh PHI run)."""
        self.lib.oracle_reset_time_local(self.ctx)

    def time_local(self):
        """Time-local truncation sums Q_m, (num_baths, N, N) complex in PHI's
        column-major storage (element [m, j, i] = Q_m[i, j])."""
        nb = self.num_baths
        out = np.zeros(2 * nb * self.n * self.n)
        self.lib.oracle_get_time_local(self.ctx, out.ctypes.data)
        return out.view(np.complex128).reshape(nb, self.n, self.n)

    def rk4(self, state, dt, t_end, output_min_step=0.0, capacity=0, start_time=0.0, continue_run=False):
        """RK4 from `state`.  The filter flags and the time-local matrices
        start as a fresh PHI run has them unless continue_run keeps those the
        previous call left."""
        if not continue_run:
            self.reset_run_state()
        s = np.ascontiguousarray(state, np.float64).copy()
        E2 = 2 * self.n * self.n
        traj = np.zeros(max(capacity, 1) * E2)
        times = np.zeros(max(capacity, 1))
        nout = c_int64()
        steps = self.lib.oracle_rk4(self.ctx, s.ctypes.data, dt, start_time, t_end, output_min_step,
                                    traj.ctypes.data if capacity else None,
                                    times.ctypes.data if capacity else None, capacity,
                                    ctypes.byref(nout))
        k = min(nout.value, capacity)
        rows = [_from_colmajor(traj[r * E2:(r + 1) * E2], self.n) for r in range(k)]
        return s, int(steps), times[:k].copy(), np.array(rows)

    def rkf45(self, state, dt0, t_end, tol, min_dt, start_time=0.0, continue_run=False, trace_capacity=0):
        """RKF45 from `state`; run state (flags, time-local matrices) as
        for rk4.  With trace_capacity > 0 the result also holds `errors`, the
        error estimate of every attempted step."""
        if not continue_run:
            self.reset_run_state()
        s = np.ascontiguousarray(state, np.float64).copy()
        acc = c_int64()
        tf = c_double()
        dtf = c_double()
        trace = np.zeros(trace_capacity, np.float64)
        steps = self.lib.oracle_rkf45_trace(self.ctx, s.ctypes.data, dt0, start_time, t_end, tol, min_dt,
                                            ctypes.byref(acc), ctypes.byref(tf), ctypes.byref(dtf),
                                            trace.ctypes.data if trace_capacity else None, trace_capacity)
        st = {"steps": int(steps), "accepted": acc.value, "final_time": tf.value, "final_dt": dtf.value}
        if trace_capacity:
            st["errors"] = trace[:min(int(steps), trace_capacity)].copy()
        return s, st

    def rho0(self, state):
        return _from_colmajor(np.asarray(state)[:2 * self.n * self.n], self.n)

    def basis(self):
        """Current truncation basis V (F x N real) of a truncated annealing
        run; the identity without truncation."""
        if self.F == self.n:
            return np.eye(self.n)
        v = np.zeros(self.F * self.n)
        self.lib.oracle_get_basis(self.ctx, v.ctypes.data)
        return v.reshape(self.n, self.F).T

    def rho0_full(self, state):
        """rho_0 in the full Hilbert space, V rho_0 V^T (UnTruncate,
        hilbert_space_truncator.cc:76-88), after the last run."""
        V = self.basis()
        return V @ self.rho0(state) @ V.T

    # -- steady state --------------------------------------------------------
    # Coordinates of a Hermitian ADO X (N*N reals, in the column-major element
    # order of the state): (i,i) -> Re X_ii, (i<j) -> Re X_ij, (i>j) -> Im X_ji.

    def _to_coords(self, state):
        n = self.n
        z = np.asarray(state).view(np.complex128).reshape(self.M, n, n)  # z[m, j, i] = X_ij
        x = np.transpose(z, (0, 2, 1))                                      # x[m, i, j] = X_ij
        iu = np.triu_indices(n, 1)
        c = np.empty((self.M, n, n))
        c[:, np.arange(n), np.arange(n)] = x[:, np.arange(n), np.arange(n)].real
        c[:, iu[0], iu[1]] = x[:, iu[0], iu[1]].real
        c[:, iu[1], iu[0]] = x[:, iu[0], iu[1]].imag
        return np.transpose(c, (0, 2, 1)).reshape(-1)                       # column-major like the state

    def _from_coords(self, coords):
        n = self.n
        c = np.transpose(np.asarray(coords).reshape(self.M, n, n), (0, 2, 1))  # c[m, i, j]
        iu = np.triu_indices(n, 1)
        x = np.zeros((self.M, n, n), np.complex128)
        x[:, np.arange(n), np.arange(n)] = c[:, np.arange(n), np.arange(n)]
        upper = c[:, iu[0], iu[1]] + 1j * c[:, iu[1], iu[0]]
        x[:, iu[0], iu[1]] = upper
        x[:, iu[1], iu[0]] = np.conj(upper)
        return np.ascontiguousarray(np.transpose(x, (0, 2, 1))).view(np.float64).reshape(-1)

    def liouvillian_matrix(self):
        """Real matrix of the Liouvillian on Hermitian hierarchies, in the
        coordinates above (one oracle apply per basis element)."""
        D = self.M * self.n * self.n
        A = np.empty((D, D))
        e = np.zeros(D)
        for k in range(D):
            e[k] = 1.0
            A[:, k] = self._to_coords(self.apply(self._from_coords(e)))
            e[k] = 0.0
        return A

    def steady_state(self, A=None):
        """Steady state L rho = 0 by a dense solve of the system that
        PrepForSteadyState / BicgstabSteadyState set up
        (hierarchy_integrator.cc:1471-1613 and :3495-3513): rho_0[0,0] fixed to
        1 and eliminated, minus its column of L as the right-hand side, the
        equation of output element (0,0) of node 0 dropped (the zeroed top
        row), and the solution divided by tr rho_0.  Small hierarchies only."""
        if A is None:
            A = self.liouvillian_matrix()
        u = np.zeros(A.shape[0])
        u[0] = 1.0
        u[1:] = np.linalg.solve(A[1:, 1:], -A[1:, 0])
        x = self._from_coords(u)
        return x / np.trace(self.rho0(x)).real


# ---------------------------------------------------------------------------
# The reference itself (oracle/_ref/ref_driver), driven through PHI parameter
# files.

def _fmt(x: float) -> str:
    return repr(float(x))


def _row(vals) -> str:
    vals = np.asarray(vals)
    if np.iscomplexobj(vals) and np.any(vals.imag != 0):
        return ",".join(f"({_fmt(v.real)},{_fmt(v.imag)})" for v in vals)
    return ",".join(_fmt(np.real(v)) for v in vals)


def param_file_text(p, timestep=None, t_end=None, output_min_step=None, rkf45_tol=None,
                    rkf45_mindt=None, output_file="/dev/null") -> str:
    """PHI parameter file (keys and layout of PhiParameters::ReadInputFile,
    phi_parameters.cc:152-784) for a duck-typed PhiParameters."""
    n = int(p.num_states)
    lines = [f"OutputFile={output_file}", "verbose=-2",
             f"hbar={_fmt(p.hbar)}", f"kB={_fmt(p.boltzmann_constant)}",
             f"NumStates={n}"]
    hs = int(getattr(p, "hilbert_space_size", 0) or 0)
    if hs > n:
        # Hilbert-space truncation: matrices in the full space (phi_parameters.cc:219-238)
        lines.append(f"HilbertSpaceSize={hs}")
        n = hs
    if getattr(p, "transverse_hamiltonian", None) is not None:
        # Annealing Hamiltonian (phi_parameters.cc:363-441).
        for key, M, fkey, f in (("TransverseHamiltonian", p.transverse_hamiltonian, "TransverseField",
                                 p.transverse_field),
                                ("LongitudinalHamiltonian", p.longitudinal_hamiltonian, "LongitudinalField",
                                 p.longitudinal_field)):
            M = np.asarray(M, np.complex128)
            lines.append(key + ":")
            lines += [_row(M[r]) for r in range(n)]
            lines.append(f"{fkey}=" + ",".join(_fmt(x) for x in np.asarray(f, np.float64)))
        lines.append(f"MinimumFieldChange={_fmt(p.minimum_field_change)}")
    else:
        lines.append("Hamiltonian:")
        H = np.asarray(p.time_indepenent_hamiltonian, np.complex128)
        lines += [_row(H[r]) for r in range(n)]
    lines.append(f"NumCouplingTerms={int(p.num_bath_couplings)}")
    kind = bath_kind(p)
    if kind == 1:
        lines.append("CorrelatedCouplingTerms:")
        V = np.asarray(p.bath_coupling_op, np.float64).reshape(-1, n)
        lines += [_row(V[b]) for b in range(V.shape[0])]
    elif kind == 2:
        lines.append("FullBathTerms:")
        V = np.asarray(p.bath_coupling_op, np.float64).reshape(-1, n, n)
        lines += [_row(V[b].T.reshape(-1)) for b in range(V.shape[0])]
    lines += ["Gamma:", _row(p.gamma), "Lambda:", _row(p.lambda_),
              f"Temperature={_fmt(p.temperature)}",
              f"MatsubaraTerms={int(p.num_matsubara_terms) - 1}",
              f"HierarchyTruncation={int(p.hierarchy_truncation_level)}",
              f"rho_normalized={1 if p.is_rho_normalized else 0}",
              "InitialDensityMatrix:"]
    R = np.asarray(p.initial_density_matrix, np.complex128)
    lines += [_row(R[r]) for r in range(n)]
    lines.append(f"Timestep={_fmt(timestep if timestep is not None else p.timestep)}")
    t_end = t_end if t_end is not None else p.integration_time
    if not t_end > 0:  # the reader rejects Time <= 0 (parameter_input.cc:18-24)
        t_end = 1e-3
    lines.append(f"Time={_fmt(t_end)}")
    lines.append(f"OutputMinimumTimestep={_fmt(output_min_step if output_min_step is not None else p.output_minimum_timestep)}")
    lines.append(f"RKF45tolerance={_fmt(rkf45_tol if rkf45_tol is not None else p.rkf45_tolerance)}")
    lines.append(f"RKF45mindt={_fmt(rkf45_mindt if rkf45_mindt is not None else p.rkf45_minimum_timestep)}")
    ft = float(getattr(p, "filter_tolerance", 0.0) or 0.0)
    if ft > 0:
        lines.append(f"FilterTolerance={_fmt(ft)}")
    if getattr(p, "use_time_local_truncation", False):
        lines.append("TimeLocal=1")
    return "\n".join(lines) + "\n"


def set_threads(n: int) -> None:
    """Threads of the oracle's independent-bath Liouvillian (default 1)."""
    load().oracle_set_threads(int(n))


def ref_available() -> bool:
    return os.path.exists(REF_DRIVER)


def run_reference(p, method: str, threads: int = 1, timeout: float = 600.0, driver: str = None, **kw):
    """Runs the reference integrator; returns (rho_0 as N x N complex, seconds)
    (F x F, F = hilbert_space_size, under Hilbert-space truncation)."""
    n = max(int(p.num_states), int(getattr(p, "hilbert_space_size", 0) or 0))
    with tempfile.TemporaryDirectory() as d:
        prm = os.path.join(d, "in.prm")
        out = os.path.join(d, "rho.txt")
        with open(prm, "w") as f:
            f.write(param_file_text(p, **kw))
        subprocess.run([driver or REF_DRIVER, "run", prm, method, str(threads), out], check=True,
                       timeout=timeout, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        secs = float(open(out).read().split("\n")[0].split()[1])
        return parse_rho_file(out, n), secs


def parse_rho_file(path: str, n: int) -> np.ndarray:
    """rho_0 as ref_driver prints it (a timing line, a header, then N*N
    `re im` lines in column-major order)."""
    with open(path) as f:
        lines = f.read().split("\n")
    vals = np.array([[float(x) for x in ln.split()] for ln in lines[2:2 + n * n]])
    rho_cm = vals[:, 0] + 1j * vals[:, 1]
    return rho_cm.reshape(n, n).T.copy()


def reference_order(p, timeout: float = 600.0) -> np.ndarray:
    """Node order of the reference's ConstructI: (M, T) multi-indices."""
    with tempfile.TemporaryDirectory() as d:
        prm = os.path.join(d, "in.prm")
        out = os.path.join(d, "order.txt")
        with open(prm, "w") as f:
            f.write(param_file_text(p))
        subprocess.run([REF_DRIVER, "order", prm, out], check=True, timeout=timeout,
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        rows = [ln.split() for ln in open(out).read().strip().split("\n")]
    return np.array([[int(x) for x in r] for r in rows], dtype=np.int32)
