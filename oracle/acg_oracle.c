/*
 * ORACLE — test infrastructure only.  Nothing in the product links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
 * as the checker.
 *
 * Plain-C, single-threaded, FP64 restatement of the reference's solve phase
 * (Laplacians.jl v1.4.1), following the reference line by line:
 *   lap(a)          = sparse(Diagonal(a*ones(n))) - a        src/graphOps.jl:25
 *   mat*p           SparseArrays CSC mat-vec (column order)   called at src/pcg.jl:291
 *   LDLsolver       copy, forward!, ./d (d != 0), backward!, minus mean
 *                                                             src/approxChol.jl:1347-1366
 *   forward!        src/approxChol.jl:1369-1388
 *   backward!       src/approxChol.jl:1390-1408
 *   pcg             src/pcg.jl:256-445 (bestx, all stop rules, stag_test)
 *   f(b)            pcg(la, b .- mean(b), F; stag_test)       src/approxChol.jl:1624
 * Where the reference calls OpenBLAS (dot, norm) or Julia's pairwise/SIMD
 * `sum`/`mean`, this file sums sequentially in index order; those reductions
 * therefore agree with the reference to rounding, not bit for bit.
 * Compiled with -ffp-contract=off so that a*b+c is never fused (Julia does
 * not fuse either).
 *
 * Index arrays are 1-based int64 exactly as Julia stores them.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ---- Laplacian ---------------------------------------------------------- */

/* Number of stored entries of lap(a): nnz(a) + n (the diagonal is stored for
 * every vertex because a*ones is dense; sparse(Diagonal(d)) keeps zeros out,
 * but a connected graph has no zero degree). */
int64_t oracle_lap_nnz(int64_t n, const int64_t* a_colptr) { return a_colptr[n] - a_colptr[0] + n; }

/* la = sparse(Diagonal(a*ones(n))) - a, in CSC with sorted rows (1-based). */
void oracle_lap(int64_t n, const int64_t* a_colptr, const int64_t* a_rowval, const double* a_nzval,
                int64_t* l_colptr, int64_t* l_rowval, double* l_nzval) {
  double* deg = (double*)calloc((size_t)n, sizeof(double));
  /* a*ones(n): y[rowval[k]] += nzval[k]*1, column by column */
  for (int64_t c = 0; c < n; ++c)
    for (int64_t k = a_colptr[c] - 1; k < a_colptr[c + 1] - 1; ++k) deg[a_rowval[k] - 1] += a_nzval[k] * 1.0;
  int64_t p = 0;
  l_colptr[0] = 1;
  for (int64_t c = 0; c < n; ++c) {
    int diag_done = 0;
    for (int64_t k = a_colptr[c] - 1; k < a_colptr[c + 1] - 1; ++k) {
      int64_t r = a_rowval[k] - 1;
      if (!diag_done && r > c) {
        l_rowval[p] = c + 1; l_nzval[p] = deg[c]; ++p; diag_done = 1;
      }
      l_rowval[p] = r + 1;
      l_nzval[p] = 0.0 - a_nzval[k];
      ++p;
    }
    if (!diag_done) { l_rowval[p] = c + 1; l_nzval[p] = deg[c]; ++p; }
    l_colptr[c + 1] = p + 1;
  }
  free(deg);
}

/* q = L*p with SparseArrays' CSC kernel: zero q, then column by column
 * q[rowval[k]] += nzval[k]*p[col]. */
void oracle_spmv(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                 const double* p, double* q) {
  for (int64_t i = 0; i < n; ++i) q[i] = 0.0;
  for (int64_t c = 0; c < n; ++c) {
    double xj = p[c];
    for (int64_t k = colptr[c] - 1; k < colptr[c + 1] - 1; ++k) q[rowval[k] - 1] += nzval[k] * xj;
  }
}

/* ---- LDLinv application ------------------------------------------------- */

void oracle_forward(int64_t n, const int64_t* col, const int64_t* colptr, const int64_t* rowval,
                    const double* fval, double* y) {
  for (int64_t ii = 0; ii < n - 1; ++ii) {
    int64_t i = col[ii] - 1;
    int64_t j0 = colptr[ii] - 1;
    int64_t j1 = colptr[ii + 1] - 2;
    double yi = y[i];
    for (int64_t jj = j0; jj < j1; ++jj) {
      int64_t j = rowval[jj] - 1;
      y[j] += fval[jj] * yi;
      yi *= (1.0 - fval[jj]);
    }
    y[rowval[j1] - 1] += yi;
    y[i] = yi;
  }
}

void oracle_backward(int64_t n, const int64_t* col, const int64_t* colptr, const int64_t* rowval,
                     const double* fval, double* y) {
  for (int64_t ii = n - 2; ii >= 0; --ii) {
    int64_t i = col[ii] - 1;
    int64_t j0 = colptr[ii] - 1;
    int64_t j1 = colptr[ii + 1] - 2;
    double yi = y[i];
    yi = yi + y[rowval[j1] - 1];
    for (int64_t jj = j1 - 1; jj >= j0; --jj) {
      int64_t j = rowval[jj] - 1;
      yi = (1.0 - fval[jj]) * yi + fval[jj] * y[j];
    }
    y[i] = yi;
  }
}

static double seq_sum(int64_t n, const double* v) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += v[i];
  return s;
}

/* y = LDLsolver(ldli, b) */
void oracle_ldlsolve(int64_t n, const int64_t* col, const int64_t* colptr, const int64_t* rowval,
                     const double* fval, const double* d, const double* b, double* y) {
  memcpy(y, b, sizeof(double) * (size_t)n);
  oracle_forward(n, col, colptr, rowval, fval, y);
  for (int64_t i = 0; i < n; ++i)
    if (d[i] != 0.0) y[i] /= d[i];
  oracle_backward(n, col, colptr, rowval, fval, y);
  double mu = seq_sum(n, y) / (double)n;
  for (int64_t i = 0; i < n; ++i) y[i] = y[i] - mu;
}

/* ---- PCG ----------------------------------------------------------------- */

typedef struct {
  int64_t n;
  const int64_t *l_colptr, *l_rowval;
  const double* l_nzval;
  const int64_t *col, *colptr, *rowval;
  const double *fval, *d;
} oracle_problem;

static double dotp(int64_t n, const double* a, const double* b) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
static double norm2(int64_t n, const double* a) { return sqrt(dotp(n, a, a)); }
static double sumabs(int64_t n, const double* a) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += fabs(a[i]);
  return s;
}
static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Stop codes match include/acgpu.h: 0 converged, 1 maxits, 2 stag x, 3 stag r,
 * 4 rho stagnation, 5 inf, 6 stag p, 7 maxtime. */
int oracle_pcg(const oracle_problem* P, const double* b, double* bestx_out, double tol, int64_t maxits,
               double maxtime, int64_t stag_test, int64_t* its_out, double* nr_out) {
  const int64_t n = P->n;
  const double eps = 2.220446049250313e-16;
  int stop = 1;
  double nb = norm2(n, b);
  if (nb == 0.0) {
    memset(bestx_out, 0, sizeof(double) * (size_t)n);
    if (its_out) *its_out = 0;
    if (nr_out) *nr_out = 0.0;
    return 0;
  }
  double* x = (double*)calloc((size_t)n, sizeof(double));
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* q = (double*)malloc(sizeof(double) * (size_t)n);
  memset(bestx_out, 0, sizeof(double) * (size_t)n);
  double bestnr = 1.0;
  memcpy(r, b, sizeof(double) * (size_t)n);
  oracle_ldlsolve(n, P->col, P->colptr, P->rowval, P->fval, P->d, r, z);
  memcpy(p, z, sizeof(double) * (size_t)n);
  double rho = dotp(n, r, z);
  double best_rho = rho;
  int64_t stag_count = 0;
  double t1 = now_s();
  int64_t itcnt = 0;
  double nr = 1.0;
  stop = 1;
  while (itcnt < maxits) {
    itcnt = itcnt + 1;
    oracle_spmv(n, P->l_colptr, P->l_rowval, P->l_nzval, p, q);
    double pq = dotp(n, p, q);
    double al = rho / pq;
    if (itcnt % 10 == 0) {
      if (al * sumabs(n, p) < eps * sumabs(n, x)) { stop = 2; break; }
    }
    for (int64_t i = 0; i < n; ++i) x[i] = x[i] + al * p[i];
    if (itcnt % 10 == 0) {
      if (al * sumabs(n, q) < eps * sumabs(n, r)) { stop = 3; break; }
    }
    for (int64_t i = 0; i < n; ++i) r[i] = r[i] + (-al) * q[i];
    nr = norm2(n, r) / nb;
    if (nr < bestnr) {
      bestnr = nr;
      memcpy(bestx_out, x, sizeof(double) * (size_t)n);
    }
    if (nr < tol) { stop = 0; break; }
    oracle_ldlsolve(n, P->col, P->colptr, P->rowval, P->fval, P->d, r, z);
    double oldrho = rho;
    rho = dotp(n, z, r);
    int stagged = 0;
    if (rho < best_rho * (1.0 - 1.0 / (double)stag_test)) {
      best_rho = rho;
      stag_count = 0;
    } else {
      if (stag_test > 0) {
        if (best_rho > (1.0 - 1.0 / (double)stag_test) * rho) {
          stag_count += 1;
          if (stag_count > stag_test) stagged = 1;
        }
      }
    }
    if (stagged) { stop = 4; break; }
    if (isinf(rho)) { stop = 5; break; }
    double beta = rho / oldrho;
    if (isinf(beta)) { stop = 5; break; }
    if (itcnt % 10 == 0) {
      if (beta * sumabs(n, p) < eps * sumabs(n, z)) { stop = 6; break; }
    }
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    if ((now_s() - t1) > maxtime) { stop = 7; break; }
    stop = 1;
  }
  if (its_out) *its_out = itcnt;
  if (nr_out) *nr_out = nr;
  free(x); free(r); free(z); free(p); free(q);
  return stop;
}

/* The closure f(b) of src/approxChol.jl:1624: pcg(la, b .- mean(b), F). */
int oracle_solve(const oracle_problem* P, const double* b, double* x, double tol, int64_t maxits,
                 double maxtime, int64_t stag_test, int64_t* its_out, double* nr_out) {
  const int64_t n = P->n;
  double* bm = (double*)malloc(sizeof(double) * (size_t)n);
  double mu = seq_sum(n, b) / (double)n;
  for (int64_t i = 0; i < n; ++i) bm[i] = b[i] - mu;
  int rc = oracle_pcg(P, bm, x, tol, maxits, maxtime, stag_test, its_out, nr_out);
  free(bm);
  return rc;
}
