/*
 * heom_oracle.c -- CPU restatement of the PHI HEOM path.  TEST
 * INFRASTRUCTURE ONLY (see heom_oracle.h): the checker for the CUDA kernels,
 * never part of the product library.
 *
 * The arithmetic follows the reference's -DNOBLAS code path operation by
 * operation (its Gemm loop, blas_wrapper.cc:11-34, stands in for every
 * zhemm), so results agree with the reference build to rounding.  Citations
 * are relative to the PHI source tree (src/...).
 */
#include "heom_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* hierarchy_node.h:7 */
static const double kPi = 3.14159265358979323846264338327950288419716939937510;

struct oracle_ctx {
  int N, nb, K1, T, trunc, kind, normalized;
  double hbar, kb, temp;
  int64_t M;
  int32_t *mi;     /* M*T multi-indices */
  int32_t *next;   /* M*T: id of n + e_t, -1 when absent */
  int32_t *prev;   /* M*T: id of n - e_t, -1 when absent */
  int32_t *tier;   /* M: sum of the multi-index */
  cplx *H, *Hadj;  /* N*N */
  cplx *corr;      /* T: correlation-function constants c_t */
  double *abs_corr;
  cplx *matsubara; /* nb: Matsubara/residual correction Delta_j */
  double *gamma;   /* nb */
  cplx *bath;      /* diagonal: nb*N; full: nb*N*N */
  cplx *same, *nextop, *prevop; /* diagonal / full bath operator tables */
  double filter_tol;       /* > 0: adaptive filtering (IndependentBath only) */
  unsigned char *active;   /* M: HierarchyNode::is_active, all 1 at the start */
  /* Time-local truncation (IndependentBath): per bath m and term k the
   * matrix Q_{m,k} (time_local_truncation_terms_th_), the sum Q_m and its
   * adjoint (time_local_matrices_ / _adjoint_), and the stored copies
   * (time_local_truncation_store_th_, time_local_matrices_store_). */
  int tl;
  cplx *tlqk, *tlqk_st;    /* nb*K1*N*N */
  cplx *tlq, *tlq_st, *tlqa;  /* nb*N*N */
  /* Annealing Hamiltonian: H and Hadj above follow the fields. */
  int anneal;
  cplx *hx, *hz;
  struct spline { int n, last; double *x, *a, *b, *c, *d; } sx, sz;
  double old_fx, old_fz;          /* old_*_field_value_th_ */
  double integration_time, min_field_change;
  /* Hilbert-space truncation of the annealing Hamiltonian: F > N, hx / hz
   * are F x F, V the current basis (F x N, real, column-major), V0 and
   * bath0 the initial basis and truncated bath operators. */
  int F;
  double *V, *V0;
  cplx *bath0;
};

/* ------------------------------------------------------------------------ */
/* Multi-index hash set (stands in for the std::map of hierarchy.h:34-35).   */

typedef struct {
  int64_t *slot; /* node id or -1 */
  int64_t mask;
  const int32_t *keys; /* node-major multi-indices */
  int T;
} index_set;

static uint64_t hash_index(const int32_t *v, int T) {
  uint64_t h = 1469598103934665603ULL;
  for (int i = 0; i < T; ++i) {
    h ^= (uint64_t)(uint32_t)v[i] + 0x9e3779b97f4a7c15ULL;
    h *= 1099511628211ULL;
    h ^= h >> 29;
  }
  return h;
}

static int set_init(index_set *s, int64_t capacity, const int32_t *keys, int T) {
  int64_t size = 16;
  while (size < 2 * capacity + 16) size <<= 1;
  s->slot = (int64_t *)malloc(sizeof(int64_t) * size);
  if (!s->slot) return -1;
  for (int64_t i = 0; i < size; ++i) s->slot[i] = -1;
  s->mask = size - 1;
  s->keys = keys;
  s->T = T;
  return 0;
}

/* Returns the id stored for v, or -1. */
static int64_t set_find(const index_set *s, const int32_t *v) {
  int64_t h = (int64_t)(hash_index(v, s->T) & (uint64_t)s->mask);
  for (;;) {
    int64_t id = s->slot[h];
    if (id < 0) return -1;
    if (memcmp(s->keys + id * s->T, v, sizeof(int32_t) * s->T) == 0) return id;
    h = (h + 1) & s->mask;
  }
}

static void set_insert(index_set *s, int64_t id) {
  const int32_t *v = s->keys + id * s->T;
  int64_t h = (int64_t)(hash_index(v, s->T) & (uint64_t)s->mask);
  while (s->slot[h] >= 0) h = (h + 1) & s->mask;
  s->slot[h] = id;
}

/* ------------------------------------------------------------------------ */

int64_t oracle_node_count(int num_terms, int truncation) {
  /* C(T + L, L) with L = truncation - 1 (phi_parameters.cc:1138-1147). */
  if (num_terms < 0 || truncation < 1) return -1;
  int64_t L = truncation - 1;
  long double acc = 1.0L;
  int64_t c = 1;
  for (int64_t i = 1; i <= L; ++i) {
    acc = acc * (num_terms + i) / i;
    if (acc > 9.0e18L) return -1;
    c = (int64_t)(acc + 0.5L);
  }
  return c;
}

int64_t oracle_build_hierarchy(int T, int truncation, int32_t *mi, int64_t capacity) {
  /* Hierarchy::ConstructI, hierarchy.cc:45-155. */
  int64_t M = oracle_node_count(T, truncation);
  if (M < 0 || M > capacity) return -1;
  index_set set;
  if (set_init(&set, M, mi, T) != 0) return -1;
  memset(mi, 0, sizeof(int32_t) * (size_t)T);  /* tier 0: id 0 (:66-70) */
  set_insert(&set, 0);
  int64_t count = 1;
  int64_t level_size = 1;
  if (truncation >= 2) {
    /* tier 1: id t+1 = e_t (:77-96). */
    for (int t = 0; t < T; ++t) {
      int32_t *v = mi + (int64_t)(t + 1) * T;
      memset(v, 0, sizeof(int32_t) * (size_t)T);
      v[t] = 1;
      set_insert(&set, t + 1);
    }
    count += T;
    level_size = T;
  }
  int32_t *cand = (int32_t *)malloc(sizeof(int32_t) * (size_t)(T + 1));
  for (int level = 2; level < truncation; ++level) {
    /* (:99-143) for each position k, for each node n of the previous tier,
     * candidate = node + e_{(n+k) mod T}; appended when not yet present. */
    const int64_t prev_first = count - level_size;
    int64_t added = 0;
    for (int k = 0; k < T; ++k) {
      for (int64_t n = 0; n < level_size; ++n) {
        memcpy(cand, mi + (prev_first + n) * T, sizeof(int32_t) * (size_t)T);
        cand[(n + k) % T] += 1;
        if (set_find(&set, cand) < 0) {
          if (count + added >= M) { free(cand); free(set.slot); return -1; }
          memcpy(mi + (count + added) * T, cand, sizeof(int32_t) * (size_t)T);
          set_insert(&set, count + added);
          ++added;
        }
      }
    }
    count += added;
    level_size = added;
  }
  free(cand);
  free(set.slot);
  return count == M ? M : -1;
}

/* ------------------------------------------------------------------------ */

static cplx cx(double re, double im) { return CMPLX(re, im); }

/* CubicSpline (cubic_spline.cc:4-120) over n samples on x_i = i / (n - 1).
 * PHI's construction as written: b_0 = 3 (y_1 - y_0), b_{n-1} =
 * 3 (y_{n-1} - y_{n-2}), b_i = 3 (y_{i+1} - y_i) otherwise, solved against
 * the tridiagonal (2, 4, ..., 4, 2 | 1) by L D L^T (dpttrf / dpttrs), then
 * c_i = 3 (a_{i+1} - a_i) - 2 b_i - b_{i+1}, d_i = 2 (a_i - a_{i+1}) + b_i +
 * b_{i+1}. */
static void spline_init(struct spline *s, const double *y, int n) {
  s->n = n;
  s->last = 0;
  s->x = (double *)malloc(sizeof(double) * (size_t)n);
  s->a = (double *)malloc(sizeof(double) * (size_t)n);
  s->b = (double *)malloc(sizeof(double) * (size_t)n);
  s->c = (double *)malloc(sizeof(double) * (size_t)n);
  s->d = (double *)malloc(sizeof(double) * (size_t)n);
  const double ds = 1. / (n - 1);
  for (int i = 0; i < n; ++i) s->x[i] = i * ds;
  for (int i = 0; i < n; ++i) s->a[i] = y[i];
  s->b[0] = 3. * (y[1] - y[0]);
  s->b[n - 1] = 3. * (y[n - 1] - y[n - 2]);
  for (int i = 1; i < n - 1; ++i) s->b[i] = 3. * (y[i + 1] - y[i]);
  double *dg = (double *)malloc(sizeof(double) * (size_t)n);
  double *e = (double *)malloc(sizeof(double) * (size_t)n);
  dg[0] = dg[n - 1] = 2.;
  for (int i = 1; i < n - 1; ++i) dg[i] = 4.;
  for (int i = 0; i < n - 1; ++i) e[i] = 1.;
  for (int i = 0; i < n - 1; ++i) {  /* factorisation */
    const double ei = e[i];
    e[i] = ei / dg[i];
    dg[i + 1] = dg[i + 1] - e[i] * ei;
  }
  double *x = s->b;                   /* forward, diagonal, backward */
  for (int i = 1; i < n; ++i) x[i] = x[i] - x[i - 1] * e[i - 1];
  x[n - 1] = x[n - 1] / dg[n - 1];
  for (int i = n - 2; i >= 0; --i) x[i] = x[i] / dg[i] - x[i + 1] * e[i];
  free(dg);
  free(e);
  for (int i = 0; i < n - 1; ++i) {
    s->c[i] = 3. * (s->a[i + 1] - s->a[i]) - 2. * s->b[i] - s->b[i + 1];
    s->d[i] = 2. * (s->a[i] - s->a[i + 1]) + s->b[i] + s->b[i + 1];
  }
}

/* CubicSpline::Locate / Get (cubic_spline.cc:33-81): the interval search
 * starts from the last interval found. */
static double spline_get(struct spline *s, double x) {
  if (x > s->x[s->n - 1]) return s->a[s->n - 1];
  if (x < s->x[0]) return s->a[0];
  int i;
  if (x > s->x[s->last] && x < s->x[s->last + 1]) {
    i = s->last;
  } else {
    i = s->last;
    while (x > s->x[i + 1]) ++i;
    while (x < s->x[i]) --i;
    s->last = i;
  }
  const double t = (x - s->x[i]) / (s->x[i + 1] - s->x[i]);
  return s->a[i] + s->b[i] * t + s->c[i] * t * t + s->d[i] * t * t * t;
}

void oracle_get_hamiltonian(const oracle_ctx *c, double *h) {
  memcpy(h, c->H, sizeof(cplx) * (size_t)(c->N * c->N));
}

static void fill_full_bath_tables(oracle_ctx *c);
static void truncate_op(int F, int k, const double *V, const cplx *A, cplx *to);

void oracle_reset_hamiltonian(oracle_ctx *c) {
  if (!c->anneal) return;
  const int E = c->N * c->N;
  for (int k = 0; k < E; ++k) c->H[k] = c->Hadj[k] = 0;
  c->old_fx = c->old_fz = DBL_MAX;   /* numeric_limits<Float>::max() (:518-523) */
  c->sx.last = c->sz.last = 0;
  if (c->F > c->N) {
    memcpy(c->V, c->V0, sizeof(double) * (size_t)c->F * c->N);
    if (c->bath0) {
      memcpy(c->bath, c->bath0, sizeof(cplx) * (size_t)(c->nb * E));
      fill_full_bath_tables(c);
    }
  }
}

int oracle_hilbert_space_size(const oracle_ctx *c) { return c->F > c->N ? c->F : c->N; }

void oracle_truncate(const oracle_ctx *c, const double *full, double *out) {
  const int F = c->F;
  cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)F * F);
  for (int k = 0; k < F * F; ++k) a[k] = cx(full[2 * k], full[2 * k + 1]);
  truncate_op(F, c->N, c->V0, a, (cplx *)out);
  free(a);
}

void oracle_get_basis(const oracle_ctx *c, double *basis) {
  memcpy(basis, c->V, sizeof(double) * (size_t)c->F * c->N);
}

/* ------------------------------------------------------------------------ */
/* Hilbert-space truncation of an annealing Hamiltonian.                     */

/* Eigenvalues (ascending) and orthonormal eigenvectors of a real symmetric
 * n x n matrix by the cyclic Jacobi method (Jacobi 1846; rotations as in
 * Rutishauser's formulation): a (column-major) is overwritten, w gets the
 * eigenvalues, v (n x n) the eigenvectors in the same order.  Stands in for
 * LAPACK's zheevr (lapack_wrapper.h:71-96); the kept subspace does not depend
 * on the method when eigenvalues k and k+1 are apart. */
static void jacobi_sym(int n, double *a, double *w, double *v) {
  for (int i = 0; i < n * n; ++i) v[i] = 0;
  for (int i = 0; i < n; ++i) v[i + i * n] = 1;
  double scale = 0;
  for (int i = 0; i < n * n; ++i) scale = fmax(scale, fabs(a[i]));
  for (int sweep = 0; sweep < 100 && scale > 0; ++sweep) {
    double off = 0;
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < q; ++p) off += a[p + q * n] * a[p + q * n];
    if (sqrt(off) <= 1e-16 * scale) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p + q * n];
        if (fabs(apq) <= 1e-300) continue;
        const double th = (a[q + q * n] - a[p + p * n]) / (2 * apq);
        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
        const double cs = 1 / sqrt(t * t + 1), sn = t * cs;
        for (int r = 0; r < n; ++r) {
          const double x = a[r + p * n], y = a[r + q * n];
          a[r + p * n] = cs * x - sn * y;
          a[r + q * n] = sn * x + cs * y;
        }
        for (int r = 0; r < n; ++r) {
          const double x = a[p + r * n], y = a[q + r * n];
          a[p + r * n] = cs * x - sn * y;
          a[q + r * n] = sn * x + cs * y;
        }
        a[p + q * n] = a[q + p * n] = 0;
        for (int r = 0; r < n; ++r) {
          const double x = v[r + p * n], y = v[r + q * n];
          v[r + p * n] = cs * x - sn * y;
          v[r + q * n] = sn * x + cs * y;
        }
      }
  }
  /* Selection sort of the eigenpairs by eigenvalue (stable for ties). */
  for (int i = 0; i < n; ++i) w[i] = a[i + i * n];
  for (int i = 0; i < n; ++i) {
    int best = i;
    for (int j = i + 1; j < n; ++j)
      if (w[j] < w[best]) best = j;
    if (best != i) {
      const double tw = w[i];
      w[i] = w[best];
      w[best] = tw;
      for (int r = 0; r < n; ++r) {
        const double tv = v[r + i * n];
        v[r + i * n] = v[r + best * n];
        v[r + best * n] = tv;
      }
    }
  }
}

/* The lowest k eigenvectors of the real part of the F x F matrix h (F x k,
 * column-major, into out).  With a previous basis, each kept vector takes
 * the sign that makes its overlap with the previous vector of the same index
 * non-negative (LAPACK's signs are arbitrary; any choice gives the same
 * truncated dynamics, and this one keeps the rotation near the identity). */
static void lowest_eigenvectors(int F, int k, const cplx *h, const double *prev, double *out) {
  double *a = (double *)malloc(sizeof(double) * (size_t)F * F);
  double *w = (double *)malloc(sizeof(double) * (size_t)F);
  double *v = (double *)malloc(sizeof(double) * (size_t)F * F);
  for (int i = 0; i < F * F; ++i) a[i] = creal(h[i]);
  jacobi_sym(F, a, w, v);
  for (int j = 0; j < k; ++j) {
    double d = 0;
    if (prev)
      for (int r = 0; r < F; ++r) d += prev[r + j * F] * v[r + j * F];
    const double sg = d < 0 ? -1.0 : 1.0;
    for (int r = 0; r < F; ++r) out[r + j * F] = sg * v[r + j * F];
  }
  free(a); free(w); free(v);
}

/* HilbertSpaceTruncator::Truncate (hilbert_space_truncator.cc:34-58) with a
 * real basis: to(j, i) = v_j^T A v_i for j <= i, to(i, j) its conjugate. */
static void truncate_op(int F, int k, const double *V, const cplx *A, cplx *to) {
  cplx *work = (cplx *)malloc(sizeof(cplx) * (size_t)F);
  for (int i = 0; i < k; ++i) {
    for (int r = 0; r < F; ++r) {
      cplx acc = 0;
      for (int l = 0; l < F; ++l) acc += A[r + l * F] * V[l + i * F];
      work[r] = acc;
    }
    for (int j = 0; j <= i; ++j) {
      cplx acc = 0;
      for (int r = 0; r < F; ++r) acc += V[r + j * F] * work[r];
      to[j + i * k] = acc;
      to[i + j * k] = conj(acc);
    }
  }
  free(work);
}

/* HilbertSpaceTruncator::Rotate (:63-74) in BLAS mode: zhemm reads A as
 * Hermitian from its upper triangle (diagonal real), so A <- R herm(A) R^+,
 * R(j, i) = <old_i | new_j> (:104-112). */
static void rotate_op(int k, const double *R, cplx *A, cplx *work) {
  for (int j = 0; j < k; ++j)    /* work = herm(A) R^T */
    for (int i = 0; i < k; ++i) {
      cplx acc = 0;
      for (int b = 0; b < k; ++b) {
        const cplx ab = i < b ? A[i + b * k] : (i > b ? conj(A[b + i * k]) : creal(A[i + i * k]));
        acc += ab * R[j + b * k];
      }
      work[i + j * k] = acc;
    }
  for (int j = 0; j < k; ++j)    /* A = R work */
    for (int i = 0; i < k; ++i) {
      cplx acc = 0;
      for (int a = 0; a < k; ++a) acc += R[i + a * k] * work[a + j * k];
      A[i + j * k] = acc;
    }
}

/* Hierarchy::FillFullBathOperators (hierarchy.cc:203-216). */
static void fill_full_bath_tables(oracle_ctx *c) {
  const int E = c->N * c->N;
  for (int m = 0; m < c->nb; ++m)
    for (int k = 0; k < E; ++k) {
      c->same[m * E + k] = csqrt(c->matsubara[m]) * c->bath[m * E + k];
      c->nextop[m * E + k] = cx(0, -1) * c->bath[m * E + k];
      c->prevop[m * E + k] = -c->bath[m * E + k];
    }
}

/* UpdateTimeDependentHamiltonian (hierarchy_integrator.cc:1618-1673):
 * H = f_x H_X + f_z H_Z at alpha = t / T, applied only when either field
 * moved by at least the minimum relative change.  With Hilbert-space
 * truncation the full H is re-diagonalised (UpdateWith, :101-113), H is
 * truncated into the new basis, the bath operators are rotated when the
 * hierarchy has more than one tier or time-local truncation (:1661-1668),
 * and the caller's live ADO arrays (live[0..nlive), M*N*N each) are rotated
 * (:1990-1995 and the other stage times) -- the time-local matrices are not. */
static void anneal_update(const oracle_ctx *cc, double time, cplx *const *live, int nlive) {
  oracle_ctx *c = (oracle_ctx *)cc;
  if (!c->anneal) return;
  const double alpha = time / c->integration_time;
  const cplx fx = spline_get(&c->sx, alpha), fz = spline_get(&c->sz, alpha);
  const double chx = fabs(creal(fx) / c->old_fx - 1.);
  const double chz = fabs(creal(fz) / c->old_fz - 1.);
  if (chx < c->min_field_change && chz < c->min_field_change) return;
  c->old_fx = creal(fx);
  c->old_fz = creal(fz);
  const int N = c->N;
  if (c->F > N) {
    const int F = c->F, E = N * N;
    cplx *hf = (cplx *)malloc(sizeof(cplx) * (size_t)F * F);
    for (int k = 0; k < F * F; ++k) hf[k] = fx * c->hx[k] + fz * c->hz[k];
    double *vn = (double *)malloc(sizeof(double) * (size_t)F * N);
    lowest_eigenvectors(F, N, hf, c->V, vn);
    double *R = (double *)malloc(sizeof(double) * (size_t)E);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double d = 0;
        for (int r = 0; r < F; ++r) d += c->V[r + i * F] * vn[r + j * F];
        R[j + i * N] = d;
      }
    memcpy(c->V, vn, sizeof(double) * (size_t)F * N);
    truncate_op(F, N, c->V, hf, c->H);
    cplx *work = (cplx *)malloc(sizeof(cplx) * (size_t)E);
    if (c->kind == ORACLE_BATH_FULL && (c->trunc > 1 || c->tl)) {
      for (int m = 0; m < c->nb; ++m) rotate_op(N, R, c->bath + (size_t)m * E, work);
      fill_full_bath_tables(c);
    }
    for (int v = 0; v < nlive; ++v)
      for (int64_t m = 0; m < c->M; ++m) rotate_op(N, R, live[v] + m * E, work);
    free(hf); free(vn); free(R); free(work);
  } else {
    for (int k = 0; k < N * N; ++k) c->H[k] = fx * c->hx[k] + fz * c->hz[k];
  }
  for (int r = 0; r < N; ++r)
    for (int col = 0; col < N; ++col) c->Hadj[r + col * N] = conj(c->H[col + r * N]);
}

oracle_ctx *oracle_create(const oracle_problem *p) {
  oracle_ctx *c = (oracle_ctx *)calloc(1, sizeof(oracle_ctx));
  if (!c) return NULL;
  const int N = p->num_states;
  c->N = N;
  c->nb = p->num_baths;
  c->K1 = p->num_matsubara;
  c->T = p->num_baths * p->num_matsubara;
  c->trunc = p->truncation;
  c->kind = p->bath_kind;
  c->normalized = p->normalized;
  c->hbar = p->hbar;
  c->kb = p->kb;
  c->temp = p->temperature;
  const int T = c->T;
  c->M = oracle_node_count(T, c->trunc);
  c->filter_tol = p->filter_tolerance;
  c->tl = p->time_local;
  c->active = (unsigned char *)malloc((size_t)(c->M > 0 ? c->M : 1));
  if (c->active) memset(c->active, 1, (size_t)(c->M > 0 ? c->M : 1));
  if (c->M <= 0) { free(c); return NULL; }
  c->mi = (int32_t *)malloc(sizeof(int32_t) * (size_t)(c->M * T + 1));
  c->next = (int32_t *)malloc(sizeof(int32_t) * (size_t)(c->M * T + 1));
  c->prev = (int32_t *)malloc(sizeof(int32_t) * (size_t)(c->M * T + 1));
  c->tier = (int32_t *)malloc(sizeof(int32_t) * (size_t)c->M);
  if (c->tl) {  /* zeroed, as SetElementsToZero does (hierarchy_integrator.cc:954-980) */
    const size_t E = (size_t)c->N * c->N, nq = (size_t)c->nb * E;
    c->tlqk = (cplx *)calloc(nq * (size_t)c->K1, sizeof(cplx));
    c->tlqk_st = (cplx *)calloc(nq * (size_t)c->K1, sizeof(cplx));
    c->tlq = (cplx *)calloc(nq, sizeof(cplx));
    c->tlq_st = (cplx *)calloc(nq, sizeof(cplx));
    c->tlqa = (cplx *)calloc(nq, sizeof(cplx));
  }
  if (oracle_build_hierarchy(T, c->trunc, c->mi, c->M) != c->M) {
    oracle_destroy(c);
    return NULL;
  }
  /* LinkHierarchyNodes (hierarchy_integrator.cc:1255-1330): prev for every t
   * with n_t > 0; next for every t while tier < truncation - 1. */
  index_set set;
  set_init(&set, c->M, c->mi, T);
  for (int64_t i = 0; i < c->M; ++i) set_insert(&set, i);
  int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(T + 1));
  for (int64_t i = 0; i < c->M; ++i) {
    const int32_t *v = c->mi + i * T;
    int tier = 0;
    for (int t = 0; t < T; ++t) tier += v[t];
    c->tier[i] = tier;
    for (int t = 0; t < T; ++t) {
      c->prev[i * T + t] = -1;
      c->next[i * T + t] = -1;
      if (v[t] > 0) {
        memcpy(tmp, v, sizeof(int32_t) * (size_t)T);
        tmp[t] -= 1;
        c->prev[i * T + t] = (int32_t)set_find(&set, tmp);
      }
      if (tier < c->trunc - 1) {
        memcpy(tmp, v, sizeof(int32_t) * (size_t)T);
        tmp[t] += 1;
        c->next[i * T + t] = (int32_t)set_find(&set, tmp);
      }
    }
  }
  free(tmp);
  free(set.slot);

  c->H = (cplx *)malloc(sizeof(cplx) * (size_t)(N * N));
  c->Hadj = (cplx *)malloc(sizeof(cplx) * (size_t)(N * N));
  double *trunc_coupling = NULL;
  if (p->h_x) {
    /* Annealing: the Hamiltonian stays zero until the first update
     * (hierarchy_integrator.cc:891-944 copies no static H). */
    c->anneal = 1;
    const int F = p->hilbert_space_size > N ? p->hilbert_space_size : N;
    c->F = F;
    c->hx = (cplx *)malloc(sizeof(cplx) * (size_t)(F * F));
    c->hz = (cplx *)malloc(sizeof(cplx) * (size_t)(F * F));
    for (int k = 0; k < F * F; ++k) {
      c->hx[k] = cx(p->h_x[2 * k], p->h_x[2 * k + 1]);
      c->hz[k] = cx(p->h_z[2 * k], p->h_z[2 * k + 1]);
    }
    spline_init(&c->sx, p->field_x, p->num_field_x);
    spline_init(&c->sz, p->field_z, p->num_field_z);
    c->integration_time = p->integration_time;
    c->min_field_change = p->min_field_change;
    if (F > N) {
      /* The truncator is first updated with H at alpha = 0 (:934-946); the
       * initial density matrix and full bath operators are truncated into
       * that basis (:1073-1075, :1179-1186). */
      const cplx f0x = spline_get(&c->sx, 0.0), f0z = spline_get(&c->sz, 0.0);
      cplx *h0 = (cplx *)malloc(sizeof(cplx) * (size_t)F * F);
      for (int k = 0; k < F * F; ++k) h0[k] = f0x * c->hx[k] + f0z * c->hz[k];
      c->V = (double *)malloc(sizeof(double) * (size_t)F * N);
      c->V0 = (double *)malloc(sizeof(double) * (size_t)F * N);
      lowest_eigenvectors(F, N, h0, NULL, c->V0);
      free(h0);
      if (p->bath_kind == ORACLE_BATH_FULL && p->coupling) {
        const size_t E = (size_t)N * N;
        trunc_coupling = (double *)malloc(sizeof(double) * (size_t)p->num_baths * E);
        cplx *full = (cplx *)malloc(sizeof(cplx) * (size_t)F * F);
        cplx *tk = (cplx *)malloc(sizeof(cplx) * E);
        for (int m = 0; m < p->num_baths; ++m) {
          for (int k = 0; k < F * F; ++k) full[k] = cx(p->coupling[(size_t)m * F * F + k], 0);
          truncate_op(F, N, c->V0, full, tk);
          for (size_t k = 0; k < E; ++k) trunc_coupling[m * E + k] = creal(tk[k]);
        }
        free(full); free(tk);
      }
    }
  } else {
    for (int k = 0; k < N * N; ++k) c->H[k] = cx(p->hamiltonian[2 * k], p->hamiltonian[2 * k + 1]);
    for (int r = 0; r < N; ++r)  /* ConjugateTranspose (complex_matrix.cc) */
      for (int col = 0; col < N; ++col) c->Hadj[r + col * N] = conj(c->H[col + r * N]);
  }

  /* Correlation-function constants, hierarchy_integrator.cc:427-473. */
  const double hbar = p->hbar;
  const double thermal = p->kb * p->temperature;
  const double nu = 2 * kPi * thermal / hbar;
  c->gamma = (double *)malloc(sizeof(double) * (size_t)(c->nb + 1));
  for (int b = 0; b < c->nb; ++b) c->gamma[b] = p->gamma[b];
  c->corr = (cplx *)calloc((size_t)T + 1, sizeof(cplx));
  c->abs_corr = (double *)calloc((size_t)T + 1, sizeof(double));
  for (int b = 0; b < c->nb; ++b) {
    const double g = p->gamma[b], l = p->lambda[b];
    if (g > 0) {
      const double a = g * l / hbar;
      const double ct = 1 / tan(g * hbar / (2 * thermal));
      c->corr[b * c->K1] = cx(a * ct, -a);
    }
    c->abs_corr[b * c->K1] = cabs(c->corr[b * c->K1]);
    for (int k = 1; k < c->K1; ++k) {
      if (g > 0) {
        c->corr[b * c->K1 + k] = cx(4 * l * g * thermal / hbar / hbar * (nu * k) /
                                        (pow(nu * k, 2) - pow(g, 2)), 0.0);
      }
      c->abs_corr[b * c->K1 + k] = cabs(c->corr[b * c->K1 + k]);
    }
  }
  /* Matsubara/residual correction, InitializePrefactors (:1375-1389). */
  c->matsubara = (cplx *)calloc((size_t)c->nb + 1, sizeof(cplx));
  for (int b = 0; b < c->nb; ++b) {
    const double g = p->gamma[b], l = p->lambda[b];
    if (g > 0) {
      double d = 2 * l * thermal / hbar / hbar / g - l / hbar / tan(hbar * g / (2 * thermal));
      for (int k = 1; k < c->K1; ++k)
        d -= 4 * l * thermal / hbar / hbar * g / (pow(nu * k, 2) - pow(g, 2));
      c->matsubara[b] = cx(d, 0.0);
    }
  }

  const int E = N * N;
  if (c->kind == ORACLE_BATH_DIAGONAL) {
    /* InitializeBathCouplingOperators (:1188-1198) and
     * Hierarchy::FillDiagonalBathOperators (hierarchy.cc:157-201). */
    c->bath = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * N));
    for (int k = 0; k < c->nb * N; ++k) c->bath[k] = cx(p->coupling[k], 0);
    c->same = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    c->nextop = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    c->prevop = (cplx *)malloc(sizeof(cplx) * (size_t)(T * E));
    for (int m = 0; m < c->nb; ++m) {
      const cplx *V = c->bath + m * N;
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
          const cplx d = V[j] - V[i];
          c->nextop[m * E + i * N + j] = cx(0, -1) * d;
          c->same[m * E + i * N + j] = c->matsubara[m] * (d * d);
        }
      for (int k = 0; k < c->K1; ++k)
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j) {
            const cplx cc = c->corr[m * c->K1 + k];
            c->prevop[m * c->K1 * E + k * E + i * N + j] =
                cx(0, -1) * (V[j] * cc - V[i] * conj(cc));
          }
    }
  } else if (c->kind == ORACLE_BATH_FULL) {
    /* Hierarchy::FillFullBathOperators (hierarchy.cc:203-216). */
    const double *cp = trunc_coupling ? trunc_coupling : p->coupling;
    c->bath = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    for (int k = 0; k < c->nb * E; ++k) c->bath[k] = cx(cp[k], 0);
    c->same = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    c->nextop = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    c->prevop = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
    fill_full_bath_tables(c);
    if (c->F > N) {
      c->bath0 = (cplx *)malloc(sizeof(cplx) * (size_t)(c->nb * E));
      memcpy(c->bath0, c->bath, sizeof(cplx) * (size_t)(c->nb * E));
    }
  }
  free(trunc_coupling);
  if (c->anneal) oracle_reset_hamiltonian(c);
  return c;
}

void oracle_destroy(oracle_ctx *c) {
  if (!c) return;
  free(c->mi); free(c->next); free(c->prev); free(c->tier);
  free(c->H); free(c->Hadj); free(c->corr); free(c->abs_corr); free(c->matsubara); free(c->gamma);
  free(c->bath); free(c->same); free(c->nextop); free(c->prevop); free(c->active);
  free(c->tlqk); free(c->tlqk_st); free(c->tlq); free(c->tlq_st); free(c->tlqa);
  free(c->hx); free(c->hz); free(c->V); free(c->V0); free(c->bath0);
  free(c->sx.x); free(c->sx.a); free(c->sx.b); free(c->sx.c); free(c->sx.d);
  free(c->sz.x); free(c->sz.a); free(c->sz.b); free(c->sz.c); free(c->sz.d);
  free(c);
}

int64_t oracle_num_nodes(const oracle_ctx *c) { return c->M; }
int oracle_num_terms(const oracle_ctx *c) { return c->T; }

void oracle_get_tables(const oracle_ctx *c, int32_t *mi, int32_t *next, int32_t *prev) {
  const size_t n = (size_t)(c->M * c->T);
  if (mi) memcpy(mi, c->mi, n * sizeof(int32_t));
  if (next) memcpy(next, c->next, n * sizeof(int32_t));
  if (prev) memcpy(prev, c->prev, n * sizeof(int32_t));
}

void oracle_get_constants(const oracle_ctx *c, double *corr, double *matsubara) {
  for (int t = 0; t < c->T; ++t) {
    corr[2 * t] = creal(c->corr[t]);
    corr[2 * t + 1] = cimag(c->corr[t]);
  }
  for (int b = 0; b < c->nb; ++b) matsubara[b] = creal(c->matsubara[b]);
}

/* ------------------------------------------------------------------------ */
/* blas::Gemm in -DNOBLAS form (blas_wrapper.cc:11-34): C = beta*C + alpha*A*B,
 * column-major square matrices; every blas::Hemm reduces to it (:36-56). */
static void gemm(int N, cplx alpha, const cplx *A, const cplx *B, cplx beta, cplx *C) {
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      C[i + j * N] *= beta;
      for (int n = 0; n < N; ++n) C[i + j * N] += alpha * (A[i + n * N] * B[j * N + n]);
    }
}
/* Hemm(CblasRight, alpha, A, B) -> alpha * B * A;  Hemm(CblasLeft) -> alpha * A * B. */
static void hemm_right(int N, cplx alpha, const cplx *A, const cplx *B, cplx beta, cplx *C) {
  gemm(N, alpha, B, A, beta, C);
}
static void hemm_left(int N, cplx alpha, const cplx *A, const cplx *B, cplx beta, cplx *C) {
  gemm(N, alpha, A, B, beta, C);
}

/* Per-node prefactors, InitializePrefactors (hierarchy_integrator.cc:1343-1466). */
typedef struct {
  cplx dephasing;
  int num_next, num_prev;
  int next_term[64], prev_term[64];
  int32_t next_id[64], prev_id[64];
  cplx next_pf[64], prev_row[64], prev_col[64];
} node_prefactors;

static void node_setup(const oracle_ctx *c, int64_t i, node_prefactors *np) {
  const int T = c->T;
  const int32_t *v = c->mi + i * T;
  const double nu = 2 * kPi * c->kb * c->temp / c->hbar;
  /* Dephasing: sum_t n_t nu_t; k = 0 terms decay with gamma of their bath,
   * k >= 1 Matsubara terms with nu * k (:1365-1371). */
  np->dephasing = 0;
  for (int m = 0; m < T; ++m) {
    const int drude = (m % c->K1) == 0;
    const int k = drude ? m / c->K1 : m % c->K1;
    const double nu_ak = drude ? c->gamma[k] : nu * k;
    np->dephasing += cx(v[m] * nu_ak, 0);
  }
  np->num_next = 0;
  np->num_prev = 0;
  for (int t = 0; t < T; ++t) {
    if (c->prev[i * T + t] >= 0) {
      const int j = np->num_prev++;
      np->prev_term[j] = t;
      np->prev_id[j] = c->prev[i * T + t];
      /* i n c and -i n c^*, scaled by 1/sqrt(n |c|) when normalised (:1420-1440). */
      np->prev_row[j] = cx(0, v[t]) * c->corr[t];
      np->prev_col[j] = cx(0, -v[t]) * conj(c->corr[t]);
      if (c->normalized) {
        const cplx s = 1.0 / cx(sqrt(v[t] * c->abs_corr[t]), 0);
        np->prev_row[j] *= s;
        np->prev_col[j] *= s;
      }
    }
  }
  for (int t = 0; t < T; ++t) {
    if (c->next[i * T + t] >= 0) {
      const int j = np->num_next++;
      np->next_term[j] = t;
      np->next_id[j] = c->next[i * T + t];
      /* i, times sqrt((n_t + 1) |c_t|) when normalised (:1398-1411). */
      np->next_pf[j] = cx(0, 1);
      if (c->normalized) np->next_pf[j] *= cx(sqrt((v[t] + 1) * c->abs_corr[t]), 0);
    }
  }
}

/* Coupling-operator index of term t: bath_indices[t / (K+1)], the identity map
 * (LinkHierarchyNodes, hierarchy_integrator.cc:1291-1293, :1320-1322). */
static int term_bath(const oracle_ctx *c, int t) { return t / c->K1; }

static void apply_node(const oracle_ctx *c, int64_t i, const cplx *rho, cplx *out,
                       cplx *temp) {
  const int N = c->N, E = N * N;
  const cplx *r = rho + i * E;
  cplx *d = out + i * E;
  const cplx lp = cx(0, -1.0 / c->hbar), nlp = cx(0, 1.0 / c->hbar);
  /* Adaptive filtering (FilterTolerance, IndependentBath): PHI calls the
   * updater through HierarchyUpdater::Get, which is not virtual
   * (hierarchy_updater.h:36-52), so IndependentBathAdaptiveTruncation::Get
   * (:227-240) never runs; only its virtual DoNext / DoPrevious overrides do
   * (hierarchy_updater.cc:256-303).  So every node keeps its own terms and
   * an inactive node contributes nothing to its neighbours. */
  const int filtered = c->filter_tol > 0 && c->kind == ORACLE_BATH_INDEPENDENT && c->trunc > 1;
  /* DoUnitary (hierarchy_updater.h:64-70): d = -i/hbar H rho + i/hbar rho H^+. */
  for (int k = 0; k < E; ++k) d[k] = 0;
  hemm_right(N, lp, r, c->H, 0, d);
  hemm_left(N, nlp, r, c->Hadj, 1, d);
  /* Vacuum updater: unitary part only (:206-219).  With time-local
   * truncation a single tier runs NoHierarchyIndependentBath through the
   * base Get instead (hierarchy_integrator.cc:1741-1758). */
  if (c->trunc == 1 && !c->tl) return;

  node_prefactors np;
  node_setup(c, i, &np);
  /* DoDephasing (:71-75). */
  for (int k = 0; k < E; ++k) d[k] -= np.dephasing * r[k];

  if (c->kind == ORACLE_BATH_INDEPENDENT) {
    /* IndependentBath::DoMatsubara (hierarchy_updater.cc:129-144). */
    for (int m = 0; m < N; ++m) {
      for (int n = 0; n < N; ++n)
        d[m * N + n] -= r[m * N + n] * (c->matsubara[n] + c->matsubara[m]);
      const int dd = (N + 1) * m;
      d[dd] += 2.0 * c->matsubara[m] * r[dd];
    }
    if (filtered) {  /* inactive neighbours contribute nothing */
      int nn = 0, pp = 0;
      for (int j = 0; j < np.num_next; ++j)
        if (c->active[np.next_id[j]]) {
          np.next_term[nn] = np.next_term[j];
          np.next_id[nn] = np.next_id[j];
          np.next_pf[nn] = np.next_pf[j];
          ++nn;
        }
      for (int j = 0; j < np.num_prev; ++j)
        if (c->active[np.prev_id[j]]) {
          np.prev_term[pp] = np.prev_term[j];
          np.prev_id[pp] = np.prev_id[j];
          np.prev_row[pp] = np.prev_row[j];
          np.prev_col[pp] = np.prev_col[j];
          ++pp;
        }
      np.num_next = nn;
      np.num_prev = pp;
    }
    /* HierarchyUpdater::Get (hierarchy_updater.h:43-49): a node of the
     * deepest tier (is_timelocal_truncated, hierarchy_integrator.cc:1324-1333)
     * takes DoTimelocal instead of DoNext.  IndependentBath::DoTimelocal
     * (hierarchy_updater.cc:171-190): temp = Q_m rho - rho Q_m^+, then
     * column m += temp[:, m] and row m -= temp[m, :]. */
    if (c->tl && c->tier[i] == c->trunc - 1) {
      for (int m = 0; m < N; ++m) {
        hemm_right(N, 1, r, c->tlq + (size_t)m * E, 0, temp);
        hemm_left(N, -1, r, c->tlqa + (size_t)m * E, 1, temp);
        for (int n = 0; n < N; ++n) d[m * N + n] += temp[m * N + n];
        for (int n = 0; n < N; ++n) d[m + n * N] -= temp[m + n * N];
      }
      np.num_next = 0;
    }
    /* IndependentBath::DoNext (:216-233): column m += p rho+[:, m];
     * row m -= p rho+[m, :]. */
    for (int j = 0; j < np.num_next; ++j) {
      const int m = term_bath(c, np.next_term[j]);
      const cplx *rn = rho + (int64_t)np.next_id[j] * E;
      for (int n = 0; n < N; ++n) d[N * m + n] += np.next_pf[j] * rn[N * m + n];
    }
    for (int n = 0; n < N; ++n)
      for (int j = 0; j < np.num_next; ++j) {
        const int m = term_bath(c, np.next_term[j]);
        const cplx *rn = rho + (int64_t)np.next_id[j] * E;
        d[N * n + m] -= np.next_pf[j] * rn[N * n + m];
      }
    /* IndependentBath::DoPrevious (:235-254). */
    for (int j = 0; j < np.num_prev; ++j) {
      const int m = term_bath(c, np.prev_term[j]);
      const cplx *rp = rho + (int64_t)np.prev_id[j] * E;
      for (int n = 0; n < N; ++n) d[N * m + n] -= np.prev_col[j] * rp[N * m + n];
    }
    for (int n = 0; n < N; ++n)
      for (int j = 0; j < np.num_prev; ++j) {
        const int m = term_bath(c, np.prev_term[j]);
        const cplx *rp = rho + (int64_t)np.prev_id[j] * E;
        d[N * n + m] -= np.prev_row[j] * rp[N * n + m];
      }
  } else if (c->kind == ORACLE_BATH_DIAGONAL) {
    /* DiagonalBath::DoMatsubara / DoNext / DoPrevious (:84-127); this updater
     * uses the bare (unnormalised) operators whatever is_rho_normalized says. */
    for (int m = 0; m < c->nb; ++m)
      for (int n = 0; n < E; ++n) d[n] -= c->same[m * E + n] * r[n];
    /* DiagonalBath::DoTimelocal (:93-104) on the deepest tier, whose next
     * list is empty: temp = -i (Q_m rho - rho Q_m^+), d += (-i)(V_j - V_i) temp. */
    if (c->tl && c->tier[i] == c->trunc - 1) {
      for (int m = 0; m < c->nb; ++m) {
        hemm_right(N, cx(0, -1), r, c->tlq + (size_t)m * E, 0, temp);
        hemm_left(N, cx(0, 1), r, c->tlqa + (size_t)m * E, 1, temp);
        for (int n = 0; n < E; ++n) d[n] += c->nextop[m * E + n] * temp[n];
      }
    }
    for (int j = 0; j < np.num_next; ++j) {
      const cplx *op = c->nextop + term_bath(c, np.next_term[j]) * E;
      const cplx *rn = rho + (int64_t)np.next_id[j] * E;
      for (int n = 0; n < E; ++n) d[n] += op[n] * rn[n];
    }
    const int32_t *v = c->mi + i * c->T;
    for (int j = 0; j < np.num_prev; ++j) {
      const int t = np.prev_term[j];
      const cplx *op = c->prevop + t * E;
      const cplx *rp = rho + (int64_t)np.prev_id[j] * E;
      const cplx pf = cx(v[t], 0);
      for (int n = 0; n < E; ++n) d[n] += pf * op[n] * rp[n];
    }
  } else {
    /* FullBath::DoMatsubara / DoNext / DoPrevious (:10-82). */
    for (int m = 0; m < c->nb; ++m) {
      const cplx *S = c->same + m * E;
      hemm_right(N, 1, r, S, 0, temp);
      hemm_left(N, -1, r, S, 1, temp);
      hemm_left(N, -1, S, temp, 1, d);
      hemm_right(N, 1, S, temp, 1, d);
    }
    /* FullBath::DoTimelocal (:28-44) on the deepest tier:
     * temp = -i (Q_m rho - rho Q_m^+), d += (-i V_m) temp - temp (-i V_m). */
    if (c->tl && c->tier[i] == c->trunc - 1) {
      for (int m = 0; m < c->nb; ++m) {
        const cplx *B = c->nextop + m * E;
        hemm_right(N, cx(0, -1), r, c->tlq + (size_t)m * E, 0, temp);
        hemm_left(N, cx(0, 1), r, c->tlqa + (size_t)m * E, 1, temp);
        hemm_right(N, 1, temp, B, 1, d);
        hemm_left(N, -1, temp, B, 1, d);
      }
    }
    for (int j = 0; j < np.num_next; ++j) {
      const cplx *B = c->nextop + term_bath(c, np.next_term[j]) * E;
      const cplx *rn = rho + (int64_t)np.next_id[j] * E;
      hemm_right(N, cx(0, -1) * np.next_pf[j], rn, B, 1, d);
      hemm_left(N, cx(0, 1) * np.next_pf[j], rn, B, 1, d);
    }
    for (int j = 0; j < np.num_prev; ++j) {
      const cplx *B = c->prevop + term_bath(c, np.prev_term[j]) * E;
      const cplx *rp = rho + (int64_t)np.prev_id[j] * E;
      hemm_right(N, np.prev_row[j], rp, B, 1, d);
      hemm_left(N, np.prev_col[j], rp, B, 1, d);
    }
  }
}

/* Threads of the node loop (1 unless oracle_set_threads raised it).  Only
 * independent-bath hierarchies are split: each node's derivative depends on
 * read-only inputs alone, so the result does not depend on the split (PHI's
 * own results are thread-count independent, too).  The diagonal and full
 * updaters keep one thread: FullBath carries its work matrix from node to
 * node, as PHI's per-thread scratch does. */
static int g_threads = 1;

void oracle_set_threads(int n) { g_threads = n > 0 ? n : 1; }

typedef struct {
  const oracle_ctx *c;
  const cplx *rho;
  cplx *out;
  int64_t begin, end;
} apply_range;

static void *apply_range_run(void *arg) {
  apply_range *r = (apply_range *)arg;
  cplx *t = (cplx *)calloc((size_t)(r->c->N * r->c->N), sizeof(cplx));
  for (int64_t i = r->begin; i < r->end; ++i) apply_node(r->c, i, r->rho, r->out, t);
  free(t);
  return NULL;
}

static void apply_all(const oracle_ctx *c, const cplx *rho, cplx *out, cplx *temp) {
  /* FullBath's work matrix starts zeroed, as new Complex[] does (:100-102). */
  for (int k = 0; k < c->N * c->N; ++k) temp[k] = 0;
  if (g_threads > 1 && c->kind == ORACLE_BATH_INDEPENDENT && c->M >= 4 * g_threads) {
    pthread_t th[64];
    apply_range rg[64];
    const int nt = g_threads < 64 ? g_threads : 64;
    for (int t = 0; t < nt; ++t) {
      rg[t].c = c;
      rg[t].rho = rho;
      rg[t].out = out;
      rg[t].begin = c->M * t / nt;
      rg[t].end = c->M * (t + 1) / nt;
    }
    int started = 0;
    for (int t = 1; t < nt; ++t, ++started)
      if (pthread_create(&th[t], NULL, apply_range_run, &rg[t]) != 0) break;
    apply_range_run(&rg[0]);
    for (int t = 1; t <= started; ++t) pthread_join(th[t], NULL);
    for (int t = started + 1; t < nt; ++t) apply_range_run(&rg[t]);  /* threads that did not start */
    return;
  }
  for (int64_t i = 0; i < c->M; ++i) apply_node(c, i, rho, out, temp);
}

void oracle_apply(const oracle_ctx *c, const double *rho_d, double *drho_d) {
  cplx *temp = (cplx *)malloc(sizeof(cplx) * (size_t)(c->N * c->N));
  apply_all(c, (const cplx *)rho_d, (cplx *)drho_d, temp);
  free(temp);
}

void oracle_initial_state(const oracle_ctx *c, const double *rho0, double *state) {
  /* InitializeDensityMatrix (hierarchy_integrator.cc:1070-1096): node 0 gets
   * rho(0) / prod_t sqrt(|c_t|^{n_t} n_t!), which is 1 at tier 0. */
  const int64_t total = c->M * c->N * c->N;
  memset(state, 0, sizeof(double) * 2 * (size_t)total);
  memcpy(state, rho0, sizeof(double) * 2 * (size_t)(c->N * c->N));
}

/* ------------------------------------------------------------------------ */

/* ConjugateTranspose (complex_matrix.cc:35-44). */
static void conj_transpose(int N, const cplx *A, cplx *Ah) {
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) Ah[i * N + j] = conj(A[j * N + i]);
}

/* UpdateTimeLocalTruncation (hierarchy_integrator.cc:1675-1693) for a step
 * of h: FillPropagator (hierarchy.cc:229-237), U = I - i H h (the Hamiltonian
 * as stored, without 1/hbar), then UpdateTimeLocalTruncationMatrices
 * (hierarchy.cc:264-341) for every bath m and term k,
 *   Q_{m,k} <- d_k U^+ (Q_{m,k} + h c_{m,k} |m><m|) U,
 * d_0 = exp(-gamma_m h), d_k = exp(-nu k h), and Q_m = sum_k Q_{m,k}
 * (SumMatrices, complex_matrix.cc:49-57).  Steps below 1e-9 are skipped. */
static void tl_update(const oracle_ctx *c, double h) {
  if (!c->tl || h < 1e-9) return;
  const int N = c->N, E = N * N, K1 = c->K1;
  cplx *U = (cplx *)malloc(sizeof(cplx) * (size_t)E);
  cplx *Ua = (cplx *)malloc(sizeof(cplx) * (size_t)E);
  cplx *tmp = (cplx *)calloc((size_t)E, sizeof(cplx));
  for (int i = 0; i < E; ++i) U[i] = cx(0, -1) * c->H[i] * h + ((i % (N + 1)) == 0 ? cx(1, 0) : cx(0, 0));
  conj_transpose(N, U, Ua);
  const double thermal = c->kb * c->temp;
  const double nu = 2 * kPi * thermal / c->hbar;
  for (int m = 0; m < c->nb; ++m) {
    for (int k = 0; k < K1; ++k) {
      cplx *Q = c->tlqk + ((size_t)m * K1 + k) * E;
      const cplx cf = h * c->corr[m * K1 + k];
      const cplx damp = k == 0 ? cx(exp(-c->gamma[m] * h), 0) : cx(exp(-nu * k * h), 0);
      /* AddIndependentBathOperator at (m, m); AddDiagonalBathOperator on the
       * diagonal; AddFullBathOperator (Axpy) on every element
       * (hierarchy.cc:218-233, :289-300). */
      if (c->kind == ORACLE_BATH_DIAGONAL) {
        for (int d = 0; d < N; ++d) Q[d * N + d] += cf * c->bath[(size_t)m * N + d];
      } else if (c->kind == ORACLE_BATH_FULL) {
        for (int e = 0; e < E; ++e) Q[e] = cf * c->bath[(size_t)m * E + e] + Q[e];
      } else {
        Q[m * N + m] += cf;
      }
      gemm(N, damp, Ua, Q, 0, tmp);
      gemm(N, 1, tmp, U, 0, Q);
    }
    cplx *S = c->tlq + (size_t)m * E;
    memcpy(S, c->tlqk + (size_t)m * K1 * E, sizeof(cplx) * (size_t)E);
    for (int k = 1; k < K1; ++k) {
      const cplx *Q = c->tlqk + ((size_t)m * K1 + k) * E;
      for (int i = 0; i < E; ++i) S[i] = cx(1, 0) * Q[i] + S[i];
    }
    conj_transpose(N, S, c->tlqa + (size_t)m * E);
  }
  free(U); free(Ua); free(tmp);
}

/* StoreTimeLocalTruncationMatrices (:1695-1712). */
static void tl_store(const oracle_ctx *c) {
  if (!c->tl) return;
  const size_t nq = (size_t)c->nb * c->N * c->N;
  memcpy(c->tlq_st, c->tlq, sizeof(cplx) * nq);
  memcpy(c->tlqk_st, c->tlqk, sizeof(cplx) * nq * (size_t)c->K1);
}

/* RestoreTimeLocalTruncationMatrices (:1714-1733). */
static void tl_restore(const oracle_ctx *c) {
  if (!c->tl) return;
  const int N = c->N, E = N * N;
  const size_t nq = (size_t)c->nb * E;
  memcpy(c->tlq, c->tlq_st, sizeof(cplx) * nq);
  memcpy(c->tlqk, c->tlqk_st, sizeof(cplx) * nq * (size_t)c->K1);
  for (int m = 0; m < c->nb; ++m) conj_transpose(N, c->tlq + (size_t)m * E, c->tlqa + (size_t)m * E);
}

void oracle_reset_time_local(oracle_ctx *c) {
  if (!c->tl) return;
  const size_t nq = (size_t)c->nb * c->N * c->N;
  memset(c->tlqk, 0, sizeof(cplx) * nq * (size_t)c->K1);
  memset(c->tlqk_st, 0, sizeof(cplx) * nq * (size_t)c->K1);
  memset(c->tlq, 0, sizeof(cplx) * nq);
  memset(c->tlq_st, 0, sizeof(cplx) * nq);
  memset(c->tlqa, 0, sizeof(cplx) * nq);
}

void oracle_get_time_local(const oracle_ctx *c, double *q) {
  const size_t nq = (size_t)c->nb * c->N * c->N;
  if (!c->tl) {
    memset(q, 0, sizeof(double) * 2 * nq);
    return;
  }
  memcpy(q, c->tlq, sizeof(cplx) * nq);
}

void oracle_reset_filter(oracle_ctx *c) {
  if (c->active) memset(c->active, 1, (size_t)c->M);
}

void oracle_get_active(const oracle_ctx *c, unsigned char *flags) {
  memcpy(flags, c->active, (size_t)c->M);
}

/* The active flags after a state update (RK4: every step, :2827-2850;
 * RKF45: every accepted step, :2359-2384): a node whose largest |element|
 * falls below the tolerance is deactivated, an inactive one whose largest
 * |element| exceeds it is reactivated. */
static void update_filter(const oracle_ctx *c, const cplx *y) {
  if (!(c->filter_tol > 0) || c->kind != ORACLE_BATH_INDEPENDENT || c->trunc <= 1) return;
  const int E = c->N * c->N;
  for (int64_t m = 0; m < c->M; ++m) {
    double mx = 0;
    for (int e = 0; e < E; ++e) {
      const double a = cabs(y[m * E + e]);
      if (a > mx) mx = a;
    }
    if (mx < c->filter_tol && c->active[m]) c->active[m] = 0;
    else if (mx > c->filter_tol && !c->active[m]) c->active[m] = 1;
  }
}

int64_t oracle_rk4(const oracle_ctx *c, double *state_d, double dt, double start_time,
                   double end_time, double output_min_step, double *traj,
                   double *traj_times, int64_t traj_capacity, int64_t *num_out) {
  /* Rk4Integrate, hierarchy_integrator.cc:2578-2939. */
  const int64_t total = c->M * c->N * c->N;
  const int E = c->N * c->N;
  cplx *y = (cplx *)state_d;
  cplx *x = (cplx *)malloc(sizeof(cplx) * (size_t)total);
  cplx *k0 = (cplx *)calloc((size_t)total, sizeof(cplx));
  cplx *k1 = (cplx *)calloc((size_t)total, sizeof(cplx));
  cplx *k2 = (cplx *)calloc((size_t)total, sizeof(cplx));
  cplx *k3 = (cplx *)calloc((size_t)total, sizeof(cplx));
  cplx *temp = (cplx *)malloc(sizeof(cplx) * (size_t)E);
  const cplx h2 = cx(dt / 2, 0), h6 = cx(dt / 6, 0), h1 = cx(dt, 0);
  const int output_factor = (int)ceil(output_min_step / dt); /* :2616-2617 */
  double time_now = start_time;
  int64_t i = -1, nout = 0;
  while (time_now < end_time) {
    i += 1;
    {
      cplx *live[] = {y};
      anneal_update(c, time_now, live, 1);                        /* :2688-2695 */
    }
    apply_all(c, y, k0, temp);                                   /* :2709-2711 */
    for (int64_t j = 0; j < total; ++j) x[j] = y[j] + k0[j] * h2; /* :2715-2718 */
    tl_update(c, dt / 2);                                         /* :2721 */
    {
      cplx *live[] = {y, x, k0};
      anneal_update(c, time_now + dt / 2, live, 3);               /* :2728-2737 */
    }
    apply_all(c, x, k1, temp);
    for (int64_t j = 0; j < total; ++j) x[j] = y[j] + k1[j] * h2; /* :2758-2761 */
    apply_all(c, x, k2, temp);
    for (int64_t j = 0; j < total; ++j) x[j] = y[j] + k2[j] * h1; /* :2777-2780 */
    tl_update(c, dt / 2);                                         /* :2784 */
    {
      cplx *live[] = {y, x, k0, k1, k2};
      anneal_update(c, time_now + dt, live, 5);                   /* :2792-2803 */
    }
    apply_all(c, x, k3, temp);
    for (int64_t j = 0; j < total; ++j)                           /* :2822-2825 */
      y[j] += h6 * (k0[j] + 2.0 * k1[j] + 2.0 * k2[j] + k3[j]);
    update_filter(c, y);                                          /* :2827-2850 */
    time_now += dt;                                               /* :2856 */
    if (output_factor > 0 && (i % output_factor) == 0) {          /* :2858 */
      if (traj && nout < traj_capacity) {
        memcpy(traj + 2 * nout * E, y, sizeof(cplx) * (size_t)E);
        if (traj_times) traj_times[nout] = time_now;
      }
      nout++;
    }
  }
  if (num_out) *num_out = nout;
  free(x); free(k0); free(k1); free(k2); free(k3); free(temp);
  return i + 1;
}

int64_t oracle_rkf45(const oracle_ctx *c, double *state_d, double dt0, double start_time,
                     double end_time, double tolerance, double min_dt,
                     int64_t *accepted_out, double *final_time, double *final_dt) {
  return oracle_rkf45_trace(c, state_d, dt0, start_time, end_time, tolerance, min_dt, accepted_out,
                            final_time, final_dt, NULL, 0);
}

int64_t oracle_rkf45_trace(const oracle_ctx *c, double *state_d, double dt0, double start_time,
                           double end_time, double tolerance, double min_dt, int64_t *accepted_out,
                           double *final_time, double *final_dt, double *err_trace, int64_t trace_cap) {
  /* Rkf45Integrate, hierarchy_integrator.cc:1797-2573.  The step-size
   * bookkeeping mirrors the reference: every tableau coefficient is scaled by
   * dt once and then multiplied in place by the grow/shrink factor, and the
   * last-step clamp permanently replaces the grow factor (:2415-2418). */
  const int64_t total = c->M * c->N * c->N;
  const int E = c->N * c->N;
  cplx *y = (cplx *)state_d;
  cplx *x = (cplx *)malloc(sizeof(cplx) * (size_t)total);
  cplx *k[6];
  for (int s = 0; s < 6; ++s) k[s] = (cplx *)calloc((size_t)total, sizeof(cplx));
  cplx *temp = (cplx *)malloc(sizeof(cplx) * (size_t)E);
  double mydt = dt0;
  cplx dtup = 1.1, dtdn = 0.5;
  /* Butcher tableau (:1937-1975); the fifth-order weight on k5 is 6/25. */
  cplx b10 = 2. / 9.;
  cplx b20 = 1. / 12., b21 = 1. / 4.;
  cplx b30 = 69. / 128., b31 = -243. / 128., b32 = 135. / 64.;
  cplx b40 = -17. / 12., b41 = 27. / 4., b42 = -27. / 5, b43 = 16. / 15;
  cplx b50 = 65. / 432., b51 = -5. / 16, b52 = 13. / 16., b53 = 4. / 27., b54 = 5. / 144.;
  cplx c50 = 1. / 9, c52 = 9. / 20, c53 = 16. / 45, c54 = 1. / 12;
  cplx c60 = 47. / 450, c62 = 12. / 25, c63 = 32. / 225, c64 = 1. / 30, c65 = 6. / 25;
  cplx *coef[] = {&b10, &b20, &b21, &b30, &b31, &b32, &b40, &b41, &b42, &b43,
                  &b50, &b51, &b52, &b53, &b54, &c50, &c52, &c53, &c54,
                  &c60, &c62, &c63, &c64, &c65};
  const int ncoef = (int)(sizeof(coef) / sizeof(coef[0]));
  const cplx dtc = cx(dt0, 0);
  for (int q = 0; q < ncoef; ++q) *coef[q] *= dtc;
  /* Stage offsets a1..a5 (:1937, :1947-1951), scaled with the step size. */
  double a[5] = {2. / 9, 1. / 3, 3. / 4, 1.0, 5. / 6};
  for (int s = 0; s < 5; ++s) a[s] *= mydt;
  double time_now = start_time;
  int64_t i = -1, accepted = 0;
  while (time_now < end_time) {
    i += 1;
    {
      cplx *live[] = {y};
      anneal_update(c, time_now, live, 1);                        /* :1988-1995 */
    }
    apply_all(c, y, k[0], temp);
    /* Time-local matrices and an annealing Hamiltonian follow the stage
     * times (:1988, :2028-2033, :2079-2084, :2132-2138, :2188-2194,
     * :2246-2252). */
    for (int64_t j = 0; j < total; ++j) x[j] = y[j] + k[0][j] * b10;
    tl_update(c, a[0]);
    {
      cplx *live[] = {y, x, k[0]};
      anneal_update(c, time_now + a[0], live, 3);
    }
    apply_all(c, x, k[1], temp);
    for (int64_t j = 0; j < total; ++j) x[j] = y[j] + k[0][j] * b20 + k[1][j] * b21;
    tl_update(c, a[1] - a[0]);
    {
      cplx *live[] = {y, x, k[0], k[1]};
      anneal_update(c, time_now + a[1], live, 4);
    }
    apply_all(c, x, k[2], temp);
    for (int64_t j = 0; j < total; ++j)
      x[j] = y[j] + k[0][j] * b30 + k[1][j] * b31 + k[2][j] * b32;
    tl_update(c, a[2] - a[1]);
    {
      cplx *live[] = {y, x, k[0], k[1], k[2]};
      anneal_update(c, time_now + a[2], live, 5);
    }
    apply_all(c, x, k[3], temp);
    for (int64_t j = 0; j < total; ++j)
      x[j] = y[j] + k[0][j] * b40 + k[1][j] * b41 + k[2][j] * b42 + k[3][j] * b43;
    tl_update(c, a[3] - a[2]);
    {
      cplx *live[] = {y, x, k[0], k[1], k[2], k[3]};
      anneal_update(c, time_now + a[3], live, 6);
    }
    apply_all(c, x, k[4], temp);
    for (int64_t j = 0; j < total; ++j)
      x[j] = y[j] + k[0][j] * b50 + k[1][j] * b51 + k[2][j] * b52 + k[3][j] * b53 +
             k[4][j] * b54;
    tl_restore(c);
    tl_update(c, a[4]);
    {
      /* k1 is not rotated at this stage (:2259-2263): no later sum reads it. */
      cplx *live[] = {y, x, k[0], k[2], k[3], k[4]};
      anneal_update(c, time_now + a[4], live, 6);
    }
    apply_all(c, x, k[5], temp);
    /* Fourth- and fifth-order solutions and the global max-abs difference
     * (:2317-2328, :2339-2351); x holds the fifth-order candidate. */
    double max_diff = 0;
    for (int64_t j = 0; j < total; ++j) {
      const cplx y4 = y[j] + k[0][j] * c50 + k[2][j] * c52 + k[3][j] * c53 + k[4][j] * c54;
      x[j] = y[j] + k[0][j] * c60 + k[2][j] * c62 + k[3][j] * c63 + k[4][j] * c64 +
             k[5][j] * c65;
      const double diff = cabs(y4 - x[j]);
      max_diff = (diff > max_diff) ? diff : max_diff;
    }
    /* The error estimate of every attempt, for callers that check the
     * accept decisions (test infrastructure). */
    if (err_trace && i < trace_cap) err_trace[i] = max_diff;
    /* Accept test (:2355) taken on the step size of this attempt. */
    if (max_diff < tolerance || mydt * creal(dtdn) < min_dt) {
      memcpy(y, x, sizeof(cplx) * (size_t)total);
      update_filter(c, y);                                        /* :2359-2384 */
      tl_update(c, mydt - a[4]);                                  /* :2388-2389 */
      tl_store(c);
      time_now += mydt;
      accepted += 1;
      int update_dt = max_diff < tolerance / 10;
      if (time_now + mydt > end_time) {
        update_dt = 1;
        dtup = cx((end_time - time_now) / mydt, 0);
      }
      if (update_dt) {
        mydt *= creal(dtup);
        for (int q = 0; q < ncoef; ++q) *coef[q] *= dtup;
        for (int s = 0; s < 5; ++s) a[s] *= creal(dtup);       /* :2403-2408 */
      }
    } else {
      mydt *= creal(dtdn);
      for (int q = 0; q < ncoef; ++q) *coef[q] *= dtdn;
      for (int s = 0; s < 5; ++s) a[s] *= creal(dtdn);         /* :2442-2447 */
      tl_restore(c);                                              /* :2479 */
    }
  }
  if (accepted_out) *accepted_out = accepted;
  if (final_time) *final_time = time_now;
  if (final_dt) *final_dt = mydt;
  free(x); for (int s = 0; s < 6; ++s) free(k[s]); free(temp);
  return i + 1;
}
