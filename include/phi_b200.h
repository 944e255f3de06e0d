/*
 * phi_b200.h -- C ABI of the B200-native HEOM integrator.
 *
 * This library is a drop-in for the time-propagation (RK4, RKF45) and
 * steady-state (BiCGSTAB) paths of the PHI parallel hierarchy integrator.
 * Every entry point takes plain pointers and sizes and returns an int status
 * (PHI_OK = 0); the C++ facade in include/phi/ (PhiParameters,
 * HierarchyIntegrator) is written on top of it.  Each declaration names the
 * reference interface it replaces (paths relative to the PHI source tree).
 *
 * Conventions shared with PHI:
 *  - complex numbers are interleaved (re, im) doubles;
 *  - every N x N matrix (Hamiltonian, rho(0), rho_0, each auxiliary density
 *    operator) is column-major: element (r, c) at index r + c*N
 *    (parameter_input.cc:244-339 fills H[r + c*N] from file row r);
 *  - the full hierarchy state is node-major in PHI's node-id order
 *    (hierarchy.cc:45-155): node i occupies elements [i*N*N, (i+1)*N*N).
 *  - units are the caller's: PHI's defaults are hbar = 5.3088354 cm^-1 ps,
 *    k_B = 0.6950344 cm^-1/K (phi_parameters.h:13-16).
 *
 * Threading: a context is single-owner; calls on one context must not
 * overlap.  Distinct contexts are independent.
 */
#ifndef PHI_B200_H_
#define PHI_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PHI_API __attribute__((visibility("default")))
#else
#define PHI_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define PHI_OK 0
#define PHI_E_INVALID 1        /* invalid or unsupported parameters */
#define PHI_E_OOM 2            /* device or host allocation failed */
#define PHI_E_BUDGET 3         /* hierarchy larger than the node budget */
#define PHI_E_STEP_COLLAPSE 4  /* RKF45 step limit reached */
#define PHI_E_NO_CONVERGENCE 5 /* iterative solve hit its iteration limit */
#define PHI_E_TIMEOUT 6        /* a bounded device wait gave up */
#define PHI_E_CUDA 7           /* CUDA runtime error */
#define PHI_E_STATE 8          /* call made in the wrong state */
#define PHI_E_NUMERIC 9        /* non-finite values appeared */

/* Bath models: HierarchyUpdater subclasses (hierarchy_updater.h:24-436). */
#define PHI_BATH_INDEPENDENT 0 /* IndependentBath: bath j couples to |s_j><s_j| */
#define PHI_BATH_DIAGONAL 1    /* DiagonalBath: CorrelatedCouplingTerms */
#define PHI_BATH_FULL 2        /* FullBath: FullBathTerms */

/* Arithmetic of the Liouvillian applies. */
#define PHI_PREC_FP64 0  /* complex128 everywhere */
#define PHI_PREC_MIXED 1 /* FP32 stage arithmetic, FP64 state / norms / control */

/* Problem description: the PhiParameters fields the path reads
 * (phi_parameters.h:32-122).  Arrays are borrowed for the duration of the
 * create call only. */
typedef struct {
  int32_t num_states;          /* num_states (N) */
  int32_t num_baths;           /* num_bath_couplings */
  int32_t num_matsubara_terms; /* num_matsubara_terms: K + 1, as PHI stores it */
  int32_t truncation_level;    /* hierarchy_truncation_level: tiers incl. tier 0 */
  int32_t bath_kind;           /* PHI_BATH_* */
  int32_t normalized;          /* is_rho_normalized */
  double hbar;                 /* hbar */
  double boltzmann_constant;   /* boltzmann_constant */
  double temperature;          /* temperature */
  const double *hamiltonian;   /* time_indepenent_hamiltonian: 2*N*N */
  const double *gamma;         /* gamma: num_baths */
  const double *lambda;        /* lambda: num_baths */
  const double *coupling;      /* bath_coupling_op: diagonal num_baths*N,
                                  full num_baths*N*N (real); NULL otherwise */
  const int32_t *bath_sites;   /* independent baths: site of each bath, NULL
                                  for PHI's identity map (bath j on |j><j|) */
  const double *initial_density_matrix; /* initial_density_matrix: 2*N*N */
  int32_t precision;           /* PHI_PREC_* */
  int32_t device;              /* CUDA device ordinal */
  int64_t max_nodes;           /* node budget; 0 = limited by memory only */
  double filter_tolerance;     /* filter_tolerance (FilterTolerance): > 0 turns on
                                  adaptive hierarchy filtering for independent
                                  baths -- after every RK4 step and every
                                  accepted RKF45 step a node whose largest
                                  |element| is below the tolerance stops
                                  feeding its neighbours, and feeds them again
                                  once it exceeds it (the DoNext / DoPrevious
                                  overrides of IndependentBathAdaptiveTruncation,
                                  hierarchy_updater.cc:256-303; flag updates
                                  hierarchy_integrator.cc:2827-2850, :2359-2384).
                                  Ignored for diagonal and full baths, as
                                  FixIncompatibleCombinations drops it
                                  (phi_parameters.cc:847-851).  0 = off. */
  int32_t time_local;          /* use_time_local_truncation (TimeLocal): 1 turns
                                  on time-local truncation -- the deepest tier
                                  takes -sum_m [V_m, Q_m rho - rho Q_m^+] in
                                  place of its next terms, with the Q_m
                                  advanced along the integrator's stage times
                                  (UpdateTimeLocalTruncation,
                                  hierarchy_integrator.cc:1675-1733;
                                  hierarchy.cc:229-341).  Independent baths on
                                  PHI's identity site map only.  0 = off. */
  /* Annealing Hamiltonian (PHI's time_indepenent_hamiltonian == NULL case,
   * UpdateTimeDependentHamiltonian, hierarchy_integrator.cc:1618-1673, no
   * Hilbert-space truncation): when annealing_h_x is non-NULL, hamiltonian
   * is ignored and before every RK4 / RKF45 stage at time t
   *   H = f_x(t / T) H_X + f_z(t / T) H_Z,
   * f_x / f_z PHI's cubic splines (cubic_spline.cc) through the samples on
   * [0, 1], applied only when either field moved by minimum_field_change
   * relative to the last applied value.  H is zero until the first stage. */
  const double *annealing_h_x;       /* H_X (TransverseHamiltonian): 2*N*N */
  const double *annealing_h_z;       /* H_Z (LongitudinalHamiltonian): 2*N*N */
  const double *transverse_field;    /* TransverseField samples */
  int32_t transverse_field_size;     /* >= 2 */
  const double *longitudinal_field;  /* LongitudinalField samples */
  int32_t longitudinal_field_size;   /* >= 2 */
  double integration_time;           /* T (Time); > 0 */
  double minimum_field_change;       /* MinimumFieldChange (PHI's default 0.01) */
  /* Hilbert-space truncation (hilbert_space_size, is_truncated_system;
   * HilbertSpaceTruncator, hilbert_space_truncator.cc:34-134): when
   * hilbert_space_size F > num_states k, hamiltonian, initial_density_matrix
   * and the full bath operators in coupling are given in the F-dimensional
   * space and the hierarchy runs in the basis of the lowest k eigenvectors of
   * the Hamiltonian (V^+ A V); phi_gpu_get_rho0_full returns V rho_0 V^+.
   * Static, real symmetric Hamiltonians; full bath couplings (or a single
   * tier without time-local truncation).  0 = no truncation. */
  int32_t hilbert_space_size;
} phi_problem_desc;

typedef struct phi_ctx phi_ctx;

/* RKF45 run statistics (Rkf45Integrate's "#Total number of integration
 * steps" / "accepted integration steps", hierarchy_integrator.cc:2545-2550). */
typedef struct {
  int64_t steps;       /* attempted steps */
  int64_t accepted;    /* accepted steps */
  double final_time;   /* time reached */
  double final_dt;     /* step size after the last step */
  double max_error;    /* largest accepted step error estimate */
} phi_rkf45_stats;

/* Steady-state solve statistics. */
typedef struct {
  int32_t iterations;    /* BiCGSTAB iterations */
  int32_t converged;     /* 1 if the residual tolerance was met */
  double residual;       /* final ||r||_2 / ||b||_2 */
  double seconds;        /* device time of the solve */
  int32_t deflated_tiers; /* tiers of the deflation space (0: plain BiCGSTAB(ell)) */
  int32_t deflation_size; /* its dimension */
} phi_solve_stats;

/* Builds the hierarchy on the device, uploads constants and sets the initial
 * state.  Replaces HierarchyIntegrator(PhiParameters*) plus the setup half of
 * Launch(): Initialize, ConstructI, LinkHierarchyNodes, InitializePrefactors,
 * InitializeDensityMatrix (hierarchy_integrator.cc:49-62, :376-594,
 * :1038-1158, :1204-1466; hierarchy.cc:45-155). */
PHI_API int phi_gpu_create(const phi_problem_desc *desc, phi_ctx **out);

/* Same, from a PHI parameter file (PhiParameters::ReadInputFile and
 * FixIncompatibleCombinations, phi_parameters.cc:152-888).  method is one of
 * "rk4", "rkf45", "bicgstab" (decides the forced normalisation exactly as
 * FixIncompatibleCombinations does). */
PHI_API int phi_gpu_create_from_file(const char *path, const char *method, int32_t precision,
                             int32_t device, phi_ctx **out);

/* Releases every device and host resource of the context. */
PHI_API int phi_gpu_destroy(phi_ctx *ctx);

/* Hierarchy size: M nodes, T = num_baths * (K+1) terms, N states. */
PHI_API int phi_gpu_dims(const phi_ctx *ctx, int64_t *num_nodes, int32_t *num_terms,
                 int32_t *num_states);
/* Number of bath coupling terms (PHI's num_bath_couplings); T / num_baths
 * is K+1. */
PHI_API int phi_gpu_num_baths(const phi_ctx *ctx, int32_t *num_baths);

/* Node table built on the device, copied to host buffers of M*T int32 each
 * (any may be NULL): multi_index[i*T + t] = n_t of node i; next[i*T + t] =
 * id of node i + e_t or -1; prev[i*T + t] = id of node i - e_t or -1.
 * Replaces the multi_index_map_ of ConstructI (hierarchy.cc:45-155) and the
 * neighbour lists of LinkHierarchyNodes (hierarchy_integrator.cc:1204-1338). */
PHI_API int phi_gpu_get_node_table(const phi_ctx *ctx, int32_t *multi_index, int32_t *next,
                           int32_t *prev);

/* Whole-hierarchy state, host buffers of 2*M*N*N doubles. */
PHI_API int phi_gpu_set_state(phi_ctx *ctx, const double *state);
PHI_API int phi_gpu_get_state(const phi_ctx *ctx, double *state);

/* Adaptive filtering flags of the current state, host buffer of M bytes:
 * 1 = active (HierarchyNode::is_active).  All 1 after create, set_state,
 * reset and restart reads, and always when filtering is off. */
PHI_API int phi_gpu_get_active(const phi_ctx *ctx, uint8_t *flags);

/* Time-local truncation sums Q_m of the current state, host buffer of
 * 2*num_baths*N*N doubles: one complex column-major N x N matrix per bath
 * (num_baths = N for independent baths, which time-local truncation needs on
 * PHI's identity site map); all zero when it is off.  Zero after create,
 * set_state and reset. */
PHI_API int phi_gpu_get_time_local(const phi_ctx *ctx, double *q);

/* The Hamiltonian the next stage starts from, host buffer of 2*N*N doubles
 * (complex column-major): the static one, or an annealing Hamiltonian as
 * last updated (zero before the first stage, and after set_state / reset). */
PHI_API int phi_gpu_get_hamiltonian(const phi_ctx *ctx, double *h);

/* rho_0 (node 0), host buffer of 2*N*N doubles.  Replaces density_matrix()
 * (hierarchy_integrator.cc:177-191), which returns the same storage order. */
PHI_API int phi_gpu_get_rho0(const phi_ctx *ctx, double *rho0);

/* One Liouvillian apply over every node: out = L(in), host buffers of
 * 2*M*N*N doubles.  Replaces a sweep of HierarchyUpdater::Get
 * (hierarchy_updater.h:36-52) over all nodes.  Input ADOs must be Hermitian
 * (PHI's formulation keeps every ADO Hermitian). */
PHI_API int phi_gpu_apply(phi_ctx *ctx, const double *in, double *out);

/* Device-pointer variant: in/out are device buffers of M*N*N complex in the
 * context's precision; stream is a cudaStream_t (NULL = legacy default). */
PHI_API int phi_gpu_apply_device(phi_ctx *ctx, const void *d_in, void *d_out, void *stream);

/* Fixed-step RK4 from the current state (Rk4Integrate,
 * hierarchy_integrator.cc:2578-2939).  Steps while time < t_end with time
 * advanced by repeated addition of dt, as the reference does.  After step i
 * (0-based) with i % ceil(output_min_step/dt) == 0, rho_0 is written to
 * traj[k*2*N*N] and its time to times[k] for k < capacity (either may be
 * NULL).  Returns the number of steps and of output rows. */
PHI_API int phi_gpu_rk4(phi_ctx *ctx, double dt, double t_end, double output_min_step,
                double *traj, double *times, int64_t capacity, int64_t *num_steps,
                int64_t *num_out);

/* Adaptive RKF45 from the current state (Rkf45Integrate,
 * hierarchy_integrator.cc:1797-2573): max-abs error over every ADO element,
 * accept if error < tol or dt/2 < min_dt, grow x1.1 when error < tol/10,
 * shrink x0.5 on reject, last step clamped to t_end.  max_steps bounds the
 * attempted steps (0 = 10^7); hitting it returns PHI_E_STEP_COLLAPSE. */
PHI_API int phi_gpu_rkf45(phi_ctx *ctx, double dt0, double t_end, double tol, double min_dt,
                  int64_t max_steps, phi_rkf45_stats *stats);

/* Advances the adaptive integrator by exactly `steps` attempted RKF45 steps
 * (fewer if t_end is reached first), with the same step control as
 * phi_gpu_rkf45.  dt0 > 0 starts a new run; dt0 <= 0 continues the step size
 * and tableau scaling of the previous call.  Reaching the step count is not
 * an error. */
PHI_API int phi_gpu_rkf45_advance(phi_ctx *ctx, double dt0, double t_end, double tol,
                                  double min_dt, int64_t steps, phi_rkf45_stats *stats);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after the library's. */
PHI_API int phi_gpu_stream(const phi_ctx *ctx, void **stream);

/* Stopping rules of phi_gpu_steady_state. */
enum {
  PHI_TOL_RELATIVE = 0,    /* ||r||_2 <= tol * ||b||_2 */
  PHI_TOL_ABSOLUTE = 1,    /* ||r||_2 <= tol: BicgstabLSteadyState's diff
                              (hierarchy_integrator.cc:3400-3421) */
  PHI_TOL_ABS_SQUARED = 2  /* ||r||_2^2 <= tol: BicgstabSteadyState's diff
                              (hierarchy_integrator.cc:3566-3594) on one thread */
};

/* Steady state of the hierarchy, L rho = 0 with tr rho_0 = 1, by
 * BiCGSTAB(ell) on the device (replaces PrepForSteadyState followed by
 * BicgstabLSteadyState / BicgstabSteadyState, hierarchy_integrator.cc:
 * 1471-1613, :3112-3441, :3495-3783): rho_0[0,0] is eliminated, the
 * right-hand side is minus the column of L that multiplies it, the equation
 * of element (0,0) of node 0 is dropped and the solution is divided by
 * tr rho_0.  ell in 1..8 (1 = BiCGSTAB; the reference's default is 2).
 * Stops by tol_mode, or after max_steps BiCG steps (ell per outer iteration,
 * the reference's `step`; 0 = 9999).  guess (host, 2*M*N*N doubles, may be
 * NULL) is the initial hierarchy, scaled so that rho_0[0,0] = 1; NULL starts
 * from rho_0 = I/N, other nodes 0 (the reference's guess without eigen
 * data).  stats->iterations = BiCG steps taken; stats->residual = the
 * quantity tol_mode compares with tol.  On return the context's state holds
 * the last iterate, also when the solve stopped without converging
 * (PHI_E_NO_CONVERGENCE).  FP64 in every precision. */
PHI_API int phi_gpu_steady_state(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode, int32_t max_steps,
                                 const double *guess, phi_solve_stats *stats);

/* Deflation of the steady-state solves of this context by the low tiers of
 * the hierarchy: BiCGSTAB(ell) runs on P A y = P b with
 * P = I - A Z (Z^T A Z)^-1 Z^T, Z the real coordinates of the ADOs of tiers
 * 0..tiers-1 (rho_0's element (0,0) excluded), and the solution is
 * y + Z (Z^T A Z)^-1 Z^T (b - A y): the same system, the same residual and
 * stopping test, fewer iterations where slow population transfer sets the
 * iteration count (PHI's own solver is undeflated: tiers = 0).  tiers = -1
 * (the default): for ell <= 2, 2 where that space has at most 256
 * coordinates, else 1 where rho_0's has, else 0; for ell > 2, 0; a solve
 * deflated this way that breaks down is run again undeflated (its
 * statistics count both runs).  tiers = 1 or 2 is refused (PHI_E_INVALID)
 * where the space exceeds 256 coordinates.  A solve whose Galerkin matrix
 * Z^T A Z is singular runs undeflated (stats->deflated_tiers = 0). */
PHI_API int phi_gpu_set_steady_deflation(phi_ctx *ctx, int32_t tiers);

/* Schedule of the tiled stage kernel (IndependentBath on PHI's identity site
 * map, K + 1 <= 3, N in {2..8, 10, 12, 16, 24}).  phi_gpu_create times one
 * Liouvillian apply for each block size (the shape's default and one
 * alternative) and each cap on persistent CTAs per SM, for problems of at
 * least 2^20 complex elements, and keeps the fastest (once per device,
 * shape and size class in the process).  Results do not depend on the
 * schedule, only the time.  threads = 0: the problem runs on the generic
 * kernel.  ctas_per_sm = 0: as many as fit. */
typedef struct {
  int32_t threads;
  int32_t ctas_per_sm;
  double ms_per_apply;         /* the chosen schedule (0 if not tuned) */
  double ms_per_apply_default; /* the default schedule (0 if not tuned) */
} phi_tile_schedule;
PHI_API int phi_gpu_get_tile_schedule(const phi_ctx *ctx, phi_tile_schedule *out);
/* Sets the schedule: threads one of the two block sizes of the shape,
 * ctas_per_sm >= 0.  PHI_E_INVALID otherwise or off the tiled kernel. */
PHI_API int phi_gpu_set_tile_schedule(phi_ctx *ctx, int32_t threads, int32_t ctas_per_sm);

/* rho_0 in the full Hilbert space, V rho_0 V^+ (UnTruncate,
 * hilbert_space_truncator.cc:82-95; hierarchy_integrator.cc:177-191): host
 * buffer of 2*F*F doubles, F = hilbert_space_size (the same as
 * phi_gpu_get_rho0 without truncation). */
PHI_API int phi_gpu_get_rho0_full(const phi_ctx *ctx, double *rho0);
/* F, the Hilbert-space size of the problem (num_states without truncation). */
PHI_API int phi_gpu_hilbert_space_size(const phi_ctx *ctx, int32_t *size);

/* Time carried by the context (advanced by the integrators). */
PHI_API int phi_gpu_get_time(const phi_ctx *ctx, double *time);
/* Restores the initial hierarchy state (rho(0) in node 0, zeros elsewhere,
 * InitializeDensityMatrix, hierarchy_integrator.cc:1070-1096) on the device,
 * sets the time to `time` and forgets the RKF45 step size; no host transfer
 * of the state. */
PHI_API int phi_gpu_reset(phi_ctx *ctx, double time);
PHI_API int phi_gpu_set_time(phi_ctx *ctx, double time);

/* One RK4 step that allocates no memory, for callers that cannot call
 * cudaMalloc when they step (code under stream capture, hosts that own all
 * device memory through their own allocator, latency-bound loops).  No
 * counterpart in the reference.  d_in and d_out are distinct caller-owned
 * device buffers of M*N*N complex128 (node-major); d_out receives the state
 * one step of size dt after d_in, d_in is not modified; the work runs on
 * `stream` (a cudaStream_t) and the call returns without synchronising.  The
 * two stage-input buffers live in a built-in 16 MiB device array, so the
 * state may be at most 8 MiB (PHI_E_INVALID above that); all calls share
 * that array, so calls that overlap on the GPU race.  The first call on a
 * device looks up the array's address; make it before any stream capture
 * (after cudaDeviceReset on that device, reload the library).  Like one
 * phi_gpu_rk4 step, each call advances the context's time-local truncation
 * matrices by dt and makes the step's new filter flags current; the
 * context's time and its own state are unchanged.  d_out is therefore one
 * step after d_in when d_in continues the trajectory those matrices and
 * flags belong to (phi_gpu_set_state resets both).  The call does not
 * synchronise: a bounded device wait that gave up inside it is reported by
 * phi_gpu_check_device_flag or by the next synchronising call. */
PHI_API int phi_gpu_rk4_step_noalloc(phi_ctx *ctx, const void *d_in, void *d_out, double dt,
                                     void *stream);

/* Waits for the work queued on `stream` (the context's own stream when NULL)
 * and reports whether a bounded device wait of the context's kernels gave up
 * since the last check (PHI_E_TIMEOUT; the flag is then cleared).  For
 * callers of the non-synchronising entry points (phi_gpu_apply_device,
 * phi_gpu_rk4_step_noalloc).  No counterpart in the reference. */
PHI_API int phi_gpu_check_device_flag(phi_ctx *ctx, void *stream);

/* Test hook for the timeout path: the poll limit of the tiled stage kernels'
 * first wait on a tile's bulk copies (0 restores the built-in limit, a
 * negative value gives up at once).  A kernel that gives up sets the
 * context's device flag, waits with the built-in limit for its own copies
 * and returns; the next checking call reports PHI_E_TIMEOUT and the context
 * stays usable.  No counterpart in the reference. */
PHI_API int phi_gpu_debug_set_wait_limit(phi_ctx *ctx, int64_t polls);

/* Test hooks for RKF45 parity.  An accept decision compares a computed
 * error estimate with the tolerance, so two FP64 evaluations that differ by
 * rounding can decide a borderline attempt differently and then follow
 * different step sequences.  set_rkf45_replay makes the next phi_gpu_rkf45
 * runs take the given decisions for their first `count` attempts (0 reject,
 * 1 accept, 2 accept and grow the step by the grow factor; the last-step
 * clamp still applies) and record the error estimate of their first
 * `trace_capacity` attempts; count = trace_capacity = 0 switches both off.
 * get_rkf45_errors copies the recorded estimates of the last run.  No
 * counterpart in the reference (its accept test is Rkf45Integrate's,
 * hierarchy_integrator.cc:2355). */
PHI_API int phi_gpu_debug_set_rkf45_replay(phi_ctx *ctx, const int8_t *decisions, int64_t count,
                                           int64_t trace_capacity);
PHI_API int phi_gpu_debug_get_rkf45_errors(phi_ctx *ctx, double *out, int64_t capacity, int64_t *count);

/* Device memory of destroyed contexts is kept (up to 8 GiB) for the next
 * allocation of the same size in this process; this returns it to the
 * driver and gives the bytes released. */
PHI_API int64_t phi_gpu_release_cached_memory(void);

/* Copies the text of the last error on this context (or of the calling
 * thread's last failed create when ctx is NULL) into buf. */
PHI_API int phi_gpu_last_error(const phi_ctx *ctx, char *buf, size_t len);

/* ---- Restart files --------------------------------------------------------
 * PHI's restart layout (RestartHelper::WriteRestartFile / ReadRestartFile,
 * restart_helper.cc:30-84): the time, the step size, then one line per node
 * with its N*N elements in storage order as "(re,im)", and for a time-local
 * run one more line per (bath m, term k) with the stored Q_{m,k}.  Written
 * with 17 significant digits (PHI writes 6); read in either form.  The host
 * functions work on host buffers (2*M*N*N doubles of state, 2*N*N doubles
 * per extra matrix) and need no GPU.  phi_restart_read_file /
 * phi_restart_write_file handle files without extra matrices (a file with
 * more values is rejected); the _ex forms read / write exactly
 * num_matrices of them after the nodes. */
PHI_API int phi_restart_read_file(const char *path, int32_t num_states, int64_t num_nodes, double *state,
                                  double *time, double *timestep);
PHI_API int phi_restart_write_file(const char *path, int32_t num_states, int64_t num_nodes, const double *state,
                                   double time, double timestep);
PHI_API int phi_restart_read_file_ex(const char *path, int32_t num_states, int64_t num_nodes, double *state,
                                     double *time, double *timestep, double *matrices, int64_t num_matrices);
PHI_API int phi_restart_write_file_ex(const char *path, int32_t num_states, int64_t num_nodes,
                                      const double *state, double time, double timestep,
                                      const double *matrices, int64_t num_matrices);
/* Copies the text of the last failed restart call of the calling thread into buf. */
PHI_API int phi_restart_last_error(char *buf, size_t len);
/* The context's state and time to / from a restart file (RestartInput and
 * RestartFile of PHI's parameter file).  A time-local context writes its
 * stored Q_{m,k} after the nodes (zero after RK4, which never stores them,
 * as in PHI) and reads them back as PHI's Initialize does
 * (hierarchy_integrator.cc:1046-1068: Q_m = sum_k Q_{m,k}, then restored). */
PHI_API int phi_gpu_write_restart(phi_ctx *ctx, const char *path, double timestep);
PHI_API int phi_gpu_read_restart(phi_ctx *ctx, const char *path, double *timestep);
/* Binary fast path: "PHIB200S", uint32 version, uint32 N, int64 M, double
 * time, double step size, the 2*M*N*N doubles of the state; version 2 adds
 * an int64 count of time-local matrices and their 2*N*N doubles each
 * (written by time-local contexts; version 1 files load as count 0). */
PHI_API int phi_gpu_save_state(phi_ctx *ctx, const char *path, double timestep);
PHI_API int phi_gpu_load_state(phi_ctx *ctx, const char *path, double *timestep);

/* ---- Batched instances ------------------------------------------------
 * Many independent hierarchies of uneven N, K and depth integrated together
 * (the reference runs one problem per process; this replaces a loop of
 * HierarchyIntegrator::Launch over RK4 runs of many parameter sets,
 * hierarchy_integrator.cc:113-175, :2593-2943).  Every RK4 stage of ALL
 * instances runs as ONE persistent kernel launch over their concatenated
 * tile lists; the step loop replays from a CUDA graph.  Each instance needs
 * IndependentBath on PHI's identity site map, K + 1 <= 3 and N in
 * {2..8, 10, 12, 16, 24}; all share one precision (desc.precision of the
 * first) and one device.  Each instance's arithmetic is the one it gets
 * alone in a phi_ctx. */
typedef struct phi_batch phi_batch;

typedef struct {
  int32_t ctas_per_sm; /* persistent CTAs per SM (grid = ctas_per_sm * SMs) */
  int32_t order;       /* 0: instances in the given order; 1: largest tiles first */
  double ms_per_stage; /* measured by phi_gpu_batch_autotune (0 if not tuned) */
} phi_batch_schedule;

typedef struct {
  int64_t steps;        /* RK4 steps taken by every instance */
  int64_t node_applies; /* 4 * steps * sum of instance node counts */
  double seconds;       /* device time of the steps (CUDA events) */
  int64_t launches;     /* kernel launches issued for the steps */
} phi_batch_stats;

PHI_API int phi_gpu_batch_create(const phi_problem_desc *descs, int32_t count, phi_batch **out);
PHI_API int phi_gpu_batch_destroy(phi_batch *batch);
/* The context of instance `index` (owned by the batch): use it for dims,
 * node tables, get/set state, rho_0 and time; do not integrate it while the
 * batch is in use. */
PHI_API int phi_gpu_batch_instance(phi_batch *batch, int32_t index, phi_ctx **ctx);
/* Times the schedule candidates (CTAs per SM x work order) on one
 * Liouvillian apply of every instance (state unchanged) and keeps the
 * fastest for later RK4 calls; `chosen` may be NULL. */
PHI_API int phi_gpu_batch_autotune(phi_batch *batch, phi_batch_schedule *chosen);
PHI_API int phi_gpu_batch_set_schedule(phi_batch *batch, const phi_batch_schedule *schedule);
/* `steps` RK4 steps of size dt on every instance (Rk4Integrate's stages,
 * hierarchy_integrator.cc:2705-2826); each instance's time advances by
 * repeated addition of dt, as in the reference's loop. */
PHI_API int phi_gpu_batch_rk4(phi_batch *batch, double dt, int64_t steps, phi_batch_stats *stats);
/* Last error of the batch (or of the last failed batch create when NULL). */
PHI_API int phi_gpu_batch_last_error(const phi_batch *batch, char *buf, size_t len);

/* ---- Learned initial guess for the steady state ------------------------
 * Kernels of the small multilayer perceptron that maps a problem's
 * parameters to its steady-state rho_0 (the initial guess of
 * phi_gpu_steady_state_rho0).  All pointers are device pointers; `stream` is
 * a cudaStream_t (NULL = default stream).  Layer: Y = act(X W^T + b),
 * X: B x in FP32 row-major, W: out x in BF16 row-major, b: FP32; act 1 =
 * tanh, 0 = identity; FP32 accumulation. */
PHI_API int phi_nn_linear_forward(const float *X, const void *W_bf16, const float *b, float *Y, int32_t B,
                                  int32_t in, int32_t out, int32_t act, void *stream);
/* Backward of one layer given dY (overwritten with dZ = dY * act'(Y)):
 * dW = dZ^T X, db = column sums of dZ, dX = dZ W (skipped when dX is NULL). */
PHI_API int phi_nn_linear_backward(float *dY, const float *Y, const float *X, const void *W_bf16, float *dX,
                                   float *dW, float *db, int32_t B, int32_t in, int32_t out, int32_t act,
                                   void *stream);
/* loss = sum (P - T)^2 / B over n = B * width values; dP = 2 (P - T) / B. */
PHI_API int phi_nn_mse(const float *P, const float *T, float *dP, float *loss, int64_t n, int32_t B,
                       void *stream);
/* One Adam step (step >= 1, bias-corrected) on FP32 master weights w; when
 * w_bf16 is not NULL it receives the rounded weights. */
PHI_API int phi_nn_adam(float *w, void *w_bf16, const float *g, float *m, float *v, int64_t n, float lr,
                        float beta1, float beta2, float eps, int32_t step, void *stream);
PHI_API int phi_nn_to_bf16(const float *a, void *b, int64_t n, void *stream);

/* phi_gpu_steady_state from the initial hierarchy rho_0 = rho0_guess (host,
 * 2*N*N doubles, column-major), every other node zero. */
PHI_API int phi_gpu_steady_state_rho0(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode,
                                      int32_t max_steps, const double *rho0_guess, phi_solve_stats *stats);

#ifdef __cplusplus
}
#endif
#endif /* PHI_B200_H_ */
