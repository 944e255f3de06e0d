/*
 * heom_oracle.h -- CPU restatement of the PHI hierarchy-equations-of-motion
 * path (hierarchy construction, per-node Liouvillian, RK4, RKF45).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it; the
 * product library never links or calls it.  Every function cites the
 * reference file:line it restates (paths relative to the PHI source tree).
 *
 * Pinning: the restatement is checked against (1) the hard-coded rho_0
 * vectors of the reference's own tests (src/hierarchy_integrator_test.cc
 * :350-509) and (2) rho_0 printed with %.17g by the reference itself, built
 * unchanged from its sources (oracle/refbuild), on small seeded problems.
 *
 * Storage convention (same as PHI): every auxiliary density operator (ADO) is
 * an N x N complex128 matrix in column-major order, element (r, c) at
 * r + c*N, stored as interleaved (re, im) doubles; nodes follow one another
 * in node-id order.
 */
#ifndef PHI_ORACLE_HEOM_ORACLE_H_
#define PHI_ORACLE_HEOM_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum oracle_bath_kind {
  ORACLE_BATH_INDEPENDENT = 0, /* IndependentBath: bath m couples to |m><m| */
  ORACLE_BATH_DIAGONAL = 1,    /* DiagonalBath: diagonal V_m, unnormalised */
  ORACLE_BATH_FULL = 2         /* FullBath: real symmetric V_m */
};

typedef struct {
  int num_states;        /* N */
  int num_baths;         /* PhiParameters::num_bath_couplings */
  int num_matsubara;     /* PhiParameters::num_matsubara_terms (= K + 1) */
  int truncation;        /* PhiParameters::hierarchy_truncation_level (= L + 1) */
  int bath_kind;         /* enum oracle_bath_kind */
  int normalized;        /* PhiParameters::is_rho_normalized */
  double hbar, kb, temperature;
  const double *hamiltonian;  /* 2*N*N, complex column-major */
  const double *gamma;        /* num_baths */
  const double *lambda;       /* num_baths */
  const double *coupling;     /* diagonal: num_baths*N; full: num_baths*N*N */
  double filter_tolerance;    /* > 0: adaptive hierarchy filtering (IndependentBath) */
  int time_local;             /* PhiParameters::use_time_local_truncation (IndependentBath) */
  /* Annealing Hamiltonian (time_indepenent_hamiltonian NULL in PHI):
   * H(t) = f_x(t/T) H_X + f_z(t/T) H_Z.  hamiltonian is ignored when h_x is
   * set.  2*N*N complex column-major each; fields sampled on [0, 1]. */
  const double *h_x, *h_z;
  const double *field_x, *field_z;
  int num_field_x, num_field_z;   /* >= 2 each */
  double integration_time;        /* T (PhiParameters::integration_time) */
  double min_field_change;        /* PhiParameters::minimum_field_change */
  /* Hilbert-space truncation of an annealing Hamiltonian
   * (PhiParameters::hilbert_space_size F > num_states = k): h_x, h_z and full
   * coupling operators are F x F, real; the hierarchy runs in the lowest k
   * eigenvectors of H(t), re-diagonalised at every Hamiltonian update.
   * 0 or num_states: no truncation. */
  int hilbert_space_size;
} oracle_problem;

typedef struct oracle_ctx oracle_ctx;

/* Number of multi-indices of T non-negative entries with sum < truncation. */
int64_t oracle_node_count(int num_terms, int truncation);

/* Hierarchy::ConstructI (hierarchy.cc:45-155): writes the multi-index of
 * every node, node-id order, num_terms ints per node.  Returns M or -1. */
int64_t oracle_build_hierarchy(int num_terms, int truncation, int32_t *multi_index,
                               int64_t capacity);

oracle_ctx *oracle_create(const oracle_problem *p);
void oracle_destroy(oracle_ctx *c);
int64_t oracle_num_nodes(const oracle_ctx *c);
int oracle_num_terms(const oracle_ctx *c);
/* Copies of the construction results (M*T each). */
void oracle_get_tables(const oracle_ctx *c, int32_t *multi_index, int32_t *next,
                       int32_t *prev);
/* c_{j,k} (2*T doubles) and the Matsubara correction Delta_j (num_baths). */
void oracle_get_constants(const oracle_ctx *c, double *corr, double *matsubara);

/* One HierarchyUpdater::Get sweep over every node (hierarchy_updater.h:36-52);
 * with filtering, over the current active flags. */
void oracle_apply(const oracle_ctx *c, const double *rho, double *drho);

/* Adaptive filtering flags (HierarchyNode::is_active): every node active at
 * creation and after oracle_reset_filter; oracle_rk4 / oracle_rkf45 update
 * them after every step (accepted step) and keep them for the next call.
 * oracle_get_active copies M bytes. */
void oracle_reset_filter(oracle_ctx *c);

/* Time-local truncation state (the Q_{m,k} matrices of every bath and Matsubara
 * term, their sums Q_m and the stored copies RKF45 restores on a rejected
 * step): zero at creation and after oracle_reset_time_local; oracle_rk4 /
 * oracle_rkf45 advance it and keep it for the next call.  oracle_get_time_local
 * copies the sums Q_m (2 * num_baths * N * N doubles). */
void oracle_reset_time_local(oracle_ctx *c);

/* Annealing Hamiltonian state (the current H, the last applied field values,
 * the spline search positions): H zero, fields unset after creation and
 * oracle_reset_hamiltonian; oracle_rk4 / oracle_rkf45 update H before every
 * stage (hierarchy_integrator.cc:1988-2252, :2688-2792) and keep the state
 * for the next call.  oracle_get_hamiltonian copies H (2*N*N doubles). */
void oracle_reset_hamiltonian(oracle_ctx *c);
void oracle_get_hamiltonian(const oracle_ctx *c, double *h);
void oracle_get_time_local(const oracle_ctx *c, double *q);
void oracle_get_active(const oracle_ctx *c, unsigned char *flags);

/* Truncated annealing contexts: Truncate (hilbert_space_truncator.cc:34-58)
 * of a full F x F operator into the initial basis (the lowest k eigenvectors
 * of H(0)), written as 2*k*k doubles; and the current basis V (F x k real,
 * column-major), which the Hamiltonian updates rotate.  rho_0 in the full
 * space is V rho_0 V^T (UnTruncate, :76-88).  oracle_reset_hamiltonian puts
 * the basis and the bath operators back to their initial values. */
int oracle_hilbert_space_size(const oracle_ctx *c);
void oracle_truncate(const oracle_ctx *c, const double *full, double *out);
void oracle_get_basis(const oracle_ctx *c, double *basis);

/* Initial hierarchy state: rho(0) scaled into node 0, zeros elsewhere
 * (hierarchy_integrator.cc:1070-1096). */
void oracle_initial_state(const oracle_ctx *c, const double *rho0, double *state);

/* Rk4Integrate (hierarchy_integrator.cc:2578-2939).  Integrates state in place
 * from start_time while time < end_time.  If traj is non-NULL, rho_0 is
 * appended after every step i with i % output_factor == 0 (times in
 * traj_times); returns the number of steps taken. */
int64_t oracle_rk4(const oracle_ctx *c, double *state, double dt, double start_time,
                   double end_time, double output_min_step, double *traj,
                   double *traj_times, int64_t traj_capacity, int64_t *num_out);

/* Rkf45Integrate (hierarchy_integrator.cc:1797-2573), with the accept test
 * taken on the step size the step was attempted with.  Returns total steps;
 * accepted steps and the final time go to the out-params. */
int64_t oracle_rkf45(const oracle_ctx *c, double *state, double dt0, double start_time,
                     double end_time, double tolerance, double min_dt,
                     int64_t *accepted, double *final_time, double *final_dt);
/* Threads of the Liouvillian's node loop for independent baths (default 1;
 * results do not depend on it). */
void oracle_set_threads(int n);

/* oracle_rkf45 that also records the max-abs error estimate of every
 * attempted step (the value PHI's accept test compares, :2355) in
 * err_trace[0 .. trace_cap-1]. */
int64_t oracle_rkf45_trace(const oracle_ctx *c, double *state, double dt0, double start_time,
                           double end_time, double tolerance, double min_dt, int64_t *accepted,
                           double *final_time, double *final_dt, double *err_trace, int64_t trace_cap);

#ifdef __cplusplus
}
#endif
#endif  /* PHI_ORACLE_HEOM_ORACLE_H_ */
