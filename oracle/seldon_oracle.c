/*
 * CPU restatement of Seldon's sparse Krylov path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle the GPU path is checked against.  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it; the
 * product library never links or calls it.  It is pinned bit-for-bit against
 * the reference itself (oracle/_ref/libseldon_ref.so, built from the Seldon
 * headers by oracle/Makefile) and against golden vectors generated from the
 * reference (tests/golden/).
 *
 * Each function restates one reference routine in plain C, keeping its exact
 * floating-point operation order (compile with -ffp-contract=off so products
 * and sums are rounded separately, as in the reference loops).  Citations are
 * file:line within the Seldon tree.
 *
 * Conventions: CSR arrays are 0-based int32 (ptr[m+1], ind[nnz]); values and
 * vectors are double.  A "sym" matrix stores only the upper triangle,
 * diagonal included (matrix_sparse/Matrix_SymSparse.cxx:1031-1032).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int m, n, nnz;
  const int* ptr;
  const int* ind;
  const double* val;
  int sym;
} orc_csr;

/* ---------------------------------------------------------------- BLAS-1 */

/* Functions_Vector.cxx:69-74 -> Vector::operator*= : X(i) *= alpha. */
void orc_scal(int n, double alpha, double* x) {
  for (int i = 0; i < n; i++) x[i] *= alpha;
}

/* Functions_Vector.cxx:85-105: no-op when alpha == 0, else Y(i) += alpha*X(i). */
void orc_axpy(int n, double alpha, const double* x, double* y) {
  if (alpha == 0.0) return;
  for (int i = 0; i < n; i++) y[i] += alpha * x[i];
}

/* Functions_Vector.cxx:240-246 (Y.Copy(X), vector/Vector.cxx:581-586). */
void orc_copy(int n, const double* x, double* y) {
  memcpy(y, x, (size_t)n * sizeof(double));
}

/* Functions_Vector.cxx:330-346: sequential sum from i = 0. */
double orc_dot(int n, const double* x, const double* y) {
  double v = 0.0;
  for (int i = 0; i < n; i++) v += x[i] * y[i];
  return v;
}

/* Functions_Vector.cxx:540-549: unscaled sqrt(sum x_i^2). */
double orc_nrm2(int n, const double* x) {
  double v = 0.0;
  for (int i = 0; i < n; i++) v += x[i] * x[i];
  return sqrt(v);
}

/* Functions_Vector.cxx:612-649: old-BLAS drotg semantics.  On exit *a = r,
 * *b = z; r takes the sign of the larger-magnitude input. */
void orc_genrot(double* a_in, double* b_in, double* c_, double* s_) {
  double a = *a_in, b = *b_in;
  double roe = (fabs(a) > fabs(b)) ? a : b;
  double scal = fabs(a) + fabs(b);
  double r, z;
  if (scal != 0.0) {
    double a_scl = a / scal;
    double b_scl = b / scal;
    r = scal * sqrt(a_scl * a_scl + b_scl * b_scl);
    if (roe < 0.0) r *= -1.0;
    *c_ = a / r;
    *s_ = b / r;
    z = 1.0;
    if (fabs(a) > fabs(b))
      z = *s_;
    else if (fabs(b) >= fabs(a) && *c_ != 0.0)
      z = 1.0 / *c_;
  } else {
    *c_ = 1.0;
    *s_ = 0.0;
    r = 0.0;
    z = 0.0;
  }
  *a_in = r;
  *b_in = z;
}

/* Functions_Vector.cxx:681-687. */
void orc_applyrot(double* x, double* y, double c, double s) {
  double temp = c * *x + s * *y;
  *y = c * *y - s * *x;
  *x = temp;
}

/* Upper-triangular back-substitution H y = s, H column-major with leading
 * dimension ld.  Gmres.cxx:166 calls Solve(ColUpTriang), which Seldon routes
 * to cblas_dtrsv (computation/interfaces/Blas_2.cxx:3226-3238); this is the
 * netlib DTRSV column sweep (UPLO=U, TRANS=N, DIAG=N). */
void orc_trsv_upper(int n, const double* H, int ld, double* s) {
  for (int j = n - 1; j >= 0; j--)
    if (s[j] != 0.0) {
      s[j] = s[j] / H[j + (size_t)j * ld];
      double t = s[j];
      for (int i = j - 1; i >= 0; i--) s[i] = s[i] - t * H[i + (size_t)j * ld];
    }
}

/* ---------------------------------------------------------------- SpMV */

/* MltAdd on RowSparse, Functions_MatVect.cxx:398-431:
 * Y *= beta (always, even for beta == 0), then Y(i) += alpha * sum_j. */
void orc_mltadd_rowsparse(int m, const int* ptr, const int* ind,
                          const double* val, double alpha, const double* x,
                          double beta, double* y) {
  orc_scal(m, beta, y);
  for (int i = 0; i < m; i++) {
    double temp = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) temp += val[j] * x[ind[j]];
    y[i] += alpha * temp;
  }
}

/* MltAdd on RowSymSparse (upper stored), Functions_MatVect.cxx:526-564:
 * row pass over the stored part, then a scatter of the strict upper part
 * for rows i < m-1. */
void orc_mltadd_rowsymsparse(int m, const int* ptr, const int* ind,
                             const double* val, double alpha, const double* x,
                             double beta, double* y) {
  orc_scal(m, beta, y);
  for (int i = 0; i < m; i++) {
    double temp = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) temp += val[j] * x[ind[j]];
    y[i] += alpha * temp;
  }
  for (int i = 0; i < m - 1; i++)
    for (int j = ptr[i]; j < ptr[i + 1]; j++)
      if (ind[j] != i) y[ind[j]] += alpha * val[j] * x[i];
}

/* MltAdd(SeldonTrans) on RowSparse, Functions_MatVect.cxx:729-758:
 * Y *= beta, then Y(ind[j]) += alpha * data[j] * X(i) row by row. */
void orc_mltadd_rowsparse_trans(int m, int n, const int* ptr, const int* ind,
                                const double* val, double alpha,
                                const double* x, double beta, double* y) {
  orc_scal(n, beta, y);
  for (int i = 0; i < m; i++)
    for (int j = ptr[i]; j < ptr[i + 1]; j++) y[ind[j]] += alpha * val[j] * x[i];
}

/* C entry used by tests: sym/trans dispatch as in Functions_MatVect.cxx
 * (RowSymSparse Trans reduces to NoTrans, :915-927). */
void orc_mltadd(int m, int n, const int* ptr, const int* ind, const double* val,
                int sym, int trans, double alpha, const double* x, double beta,
                double* y) {
  if (sym)
    orc_mltadd_rowsymsparse(m, ptr, ind, val, alpha, x, beta, y);
  else if (trans)
    orc_mltadd_rowsparse_trans(m, n, ptr, ind, val, alpha, x, beta, y);
  else
    orc_mltadd_rowsparse(m, ptr, ind, val, alpha, x, beta, y);
}

static void csr_mlt(const orc_csr* A, const double* x, double* y) {
  /* Mlt(M, X, Y): Y.Fill(0); MltAdd(1, M, X, 0, Y) -- Functions_MatVect.cxx:72-81 */
  memset(y, 0, (size_t)A->m * sizeof(double));
  orc_mltadd(A->m, A->n, A->ptr, A->ind, A->val, A->sym, 0, 1.0, x, 0.0, y);
}

static void csr_residual(const orc_csr* A, const double* x, double* r) {
  /* MltAdd(-1, A, x, 1, r) */
  orc_mltadd(A->m, A->n, A->ptr, A->ind, A->val, A->sym, 0, -1.0, x, 1.0, r);
}

/* Matrix_Sparse::operator()(i, i) lookup, Matrix_Sparse.cxx:1051-1083:
 * advance while k < b-1 and ind[k] < i, then test ind[k] == i. */
double orc_diag_entry(const int* ptr, const int* ind, const double* val, int i) {
  int a = ptr[i], b = ptr[i + 1];
  if (a == b) return 0.0;
  int k = a;
  while (k < b - 1 && ind[k] < i) k++;
  return ind[k] == i ? val[k] : 0.0;
}

/* ---------------------------------------------------------------- SOR */

/* SOR on RowSparse, Relaxation_MatVect.cxx:41-95. */
void orc_sor_rowsparse(int m, const int* ptr, const int* ind, const double* val,
                       double* x, const double* b, double omega, int iter,
                       int type_ssor) {
  if (type_ssor % 2 == 0)
    for (int it = 0; it < iter; it++)
      for (int j = 0; j < m; j++) {
        double temp = 0.0;
        double ajj = orc_diag_entry(ptr, ind, val, j);
        for (int k = ptr[j]; k < ptr[j + 1]; k++) temp += val[k] * x[ind[k]];
        temp = b[j] - temp + ajj * x[j];
        x[j] = (1.0 - omega) * x[j] + omega * temp / ajj;
      }
  if (type_ssor % 3 == 0)
    for (int it = 0; it < iter; it++)
      for (int j = m - 1; j >= 0; j--) {
        double temp = 0.0;
        double ajj = orc_diag_entry(ptr, ind, val, j);
        for (int k = ptr[j]; k < ptr[j + 1]; k++) temp += val[k] * x[ind[k]];
        temp = b[j] - temp + ajj * x[j];
        x[j] = (1.0 - omega) * x[j] + omega * temp / ajj;
      }
}

/* SOR on RowSymSparse (upper stored), Relaxation_MatVect.cxx:176-298. */
void orc_sor_rowsymsparse(int m, const int* ptr, const int* ind,
                          const double* val, double* x, const double* b,
                          double omega, int iter, int type_ssor) {
  double* y = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
  if (type_ssor % 2 == 0)
    for (int it = 0; it < iter; it++) {
      for (int j = 0; j < m; j++) {
        double temp = 0.0, ajj = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; k++) {
          int p = ind[k];
          double v = val[k];
          if (p == j)
            ajj += v;
          else
            temp += v * x[p];
        }
        temp = b[j] - temp;
        x[j] = (1.0 - omega) / omega * ajj * x[j] + temp;
      }
      for (int j = 0; j < m; j++) {
        double ajj = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; k++)
          if (ind[k] == j) ajj += val[k];
        x[j] *= omega / ajj;
        for (int k = ptr[j]; k < ptr[j + 1]; k++)
          if (ind[k] != j) x[ind[k]] -= val[k] * x[j];
      }
    }
  if (type_ssor % 3 == 0)
    for (int it = 0; it < iter; it++) {
      memset(y, 0, (size_t)m * sizeof(double));
      for (int j = 0; j < m; j++) {
        double ajj = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; k++) {
          int p = ind[k];
          double v = val[k];
          if (p == j)
            ajj += v;
          else
            y[p] += v * x[j];
        }
        x[j] = (1.0 - omega) / omega * ajj * x[j] + b[j] - y[j];
      }
      for (int j = m - 1; j >= 0; j--) {
        double temp = 0.0, ajj = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; k++) {
          int p = ind[k];
          double v = val[k];
          if (p == j)
            ajj += v;
          else
            temp += v * x[p];
        }
        x[j] = (x[j] - temp) * omega / ajj;
      }
    }
  free(y);
}

void orc_sor(int m, const int* ptr, const int* ind, const double* val, int sym,
             double* x, const double* b, double omega, int iter, int type_ssor) {
  if (sym)
    orc_sor_rowsymsparse(m, ptr, ind, val, x, b, omega, iter, type_ssor);
  else
    orc_sor_rowsparse(m, ptr, ind, val, x, b, omega, iter, type_ssor);
}

/* ---------------------------------------------------------------- Iteration */

/* Iteration<Titer>, Iterative.hxx:47-108 / Iterative.cxx:80-354. */
typedef struct {
  double tolerance, facteur_reste;
  int max_iter, nb_iter, error_code, fail_convergence, init_guess_null;
  /* residual log: every Finished() call appends (nb_iter, relative residual). */
  double* hist;
  int* hist_it;
  int hist_cap, hist_len;
} orc_iter;

static int it_init(orc_iter* it, int n, const double* r) {
  /* Iterative.cxx:235-249 */
  double nr = orc_nrm2(n, r);
  if (nr == 0.0) return -1;
  it->facteur_reste = 1.0 / nr;
  it->nb_iter = 0;
  return 0;
}

static int it_finished(orc_iter* it, double res) {
  /* Iterative.cxx:299-319 (the vector form :272-295 is Norm2 then this). */
  double reste = it->facteur_reste * res;
  if (it->hist && it->hist_len < it->hist_cap) {
    it->hist[it->hist_len] = reste;
    it->hist_it[it->hist_len] = it->nb_iter;
    it->hist_len++;
  }
  return (reste < it->tolerance) || (it->nb_iter >= it->max_iter);
}

static void it_fail(orc_iter* it, int code) {
  /* Iterative.cxx:324-331 */
  it->fail_convergence = 1;
  it->error_code = code;
}

static int it_error_code(const orc_iter* it) {
  /* Iterative.cxx:344-354 */
  if (it->nb_iter >= it->max_iter) return -2;
  if (it->fail_convergence) return it->error_code;
  return 0;
}

/* ---------------------------------------------------------------- preconditioners */

typedef struct {
  int kind; /* 0 identity, 1 Jacobi, 2 SOR */
  double omega;
  int nb_iter, symmetric;
  double* diag;
} orc_prec;

/* Preconditioner_Base::Solve = Copy (Iterative.cxx:60-65); Jacobi
 * z_i = r_i / A(i,i) (not in the reference); SorPreconditioner::Solve zeros z
 * then runs SOR type 0 (symmetric) or 2 (Precond_Ssor.cxx:62-74). */
static void prec_solve(const orc_prec* M, const orc_csr* A, const double* r,
                       double* z) {
  int n = A->m;
  if (M->kind == 0) {
    orc_copy(n, r, z);
  } else if (M->kind == 1) {
    for (int i = 0; i < n; i++) z[i] = r[i] / M->diag[i];
  } else {
    memset(z, 0, (size_t)n * sizeof(double));
    orc_sor(n, A->ptr, A->ind, A->val, A->sym, z, r, M->omega, M->nb_iter,
            M->symmetric ? 0 : 2);
  }
}

/* ---------------------------------------------------------------- solvers */

/* Cg, computation/solver/iterative/Cg.cxx:45-116. */
static int orc_cg_impl(const orc_csr* A, double* x, const double* b,
                       const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  double rho = 1.0, rho_1 = 1.0, alpha, beta, delta;
  size_t bytes = (size_t)N * sizeof(double);
  double *p = malloc(bytes), *q = malloc(bytes), *r = malloc(bytes),
         *z = malloc(bytes);
  memcpy(p, b, bytes); memcpy(q, b, bytes); memcpy(r, b, bytes); memcpy(z, b, bytes);
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r))) {
    prec_solve(M, A, r, z);
    rho = orc_dot(N, r, z);
    if (rho == 0.0) { it_fail(it, 1); break; }
    if (it->nb_iter == 0)
      orc_copy(N, z, p);
    else {
      beta = rho / rho_1;
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, z, p);
    }
    csr_mlt(A, p, q);
    delta = orc_dot(N, p, q);
    if (delta == 0.0) { it_fail(it, 2); break; }
    alpha = rho / delta;
    orc_axpy(N, alpha, p, x);
    orc_axpy(N, -alpha, q, r);
    rho_1 = rho;
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  free(p); free(q); free(r); free(z);
  return code;
}

/* BiCgStab, computation/solver/iterative/BiCgStab.cxx:43-145. */
static int orc_bicgstab_impl(const orc_csr* A, double* x, const double* b,
                             const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  double rho_1, rho_2 = 0.0, alpha = 0.0, beta, omega = 0.0, sigma;
  size_t bytes = (size_t)N * sizeof(double);
  double *p = malloc(bytes), *phat = malloc(bytes), *s = malloc(bytes),
         *shat = malloc(bytes), *t = malloc(bytes), *v = malloc(bytes),
         *r = malloc(bytes), *rtilde = malloc(bytes);
  double* all[8] = {p, phat, s, shat, t, v, r, rtilde};
  for (int k = 0; k < 8; k++) memcpy(all[k], b, bytes);
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  orc_copy(N, r, rtilde);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r))) {
    rho_1 = orc_dot(N, rtilde, r);
    if (rho_1 == 0.0) { it_fail(it, 1); break; }
    if (it->nb_iter == 0)
      orc_copy(N, r, p);
    else {
      if (omega == 0.0) { it_fail(it, 2); break; }
      beta = (rho_1 / rho_2) * (alpha / omega);
      orc_axpy(N, -omega, v, p);
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, r, p);
    }
    prec_solve(M, A, p, phat);
    csr_mlt(A, phat, v);
    sigma = orc_dot(N, rtilde, v);
    if (sigma == 0.0) { it_fail(it, 3); break; }
    alpha = rho_1 / sigma;
    orc_copy(N, r, s);
    orc_axpy(N, -alpha, v, s);
    it->nb_iter++;
    if (it_finished(it, orc_nrm2(N, s))) {
      orc_axpy(N, alpha, phat, x);
      break;
    }
    prec_solve(M, A, s, shat);
    csr_mlt(A, shat, t);
    omega = orc_dot(N, t, s) / orc_dot(N, t, t);
    orc_axpy(N, alpha, phat, x);
    orc_axpy(N, omega, shat, x);
    orc_copy(N, s, r);
    orc_axpy(N, -omega, t, r);
    rho_2 = rho_1;
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  for (int k = 0; k < 8; k++) free(all[k]);
  return code;
}

/* Gmres(m), computation/solver/iterative/Gmres.cxx:44-183.  Left
 * preconditioning, modified Gram-Schmidt, Givens rotations; the Hessenberg is
 * kept column-major in an (m+1)x(m+1) array. */
static int orc_gmres_impl(const orc_csr* A, double* x, const double* b,
                          const orc_prec* M, orc_iter* outer, int m) {
  const int N = A->m;
  if (N <= 0) return 0;
  if (m < 1) m = 1;
  size_t bytes = (size_t)N * sizeof(double);
  int ld = m + 1;
  double* V = calloc((size_t)(m + 1) * N, sizeof(double));
  double* H = calloc((size_t)ld * ld, sizeof(double));
  double *w = calloc(N, sizeof(double)), *r = calloc(N, sizeof(double)),
         *u = calloc(N, sizeof(double));
  double* s = calloc(m + 1, sizeof(double));
  double* rc = calloc(m + 1, sizeof(double));
  double* rs = calloc(m + 1, sizeof(double));
  int code;

  orc_copy(N, b, w);
  if (!outer->init_guess_null)
    csr_residual(A, x, w);
  else
    memset(x, 0, bytes);
  prec_solve(M, A, w, r);
  double beta = orc_nrm2(N, r);
  if (it_init(outer, N, r) != 0) { code = it_error_code(outer); goto out; }

  outer->nb_iter = 0;
  while (!it_finished(outer, beta)) {
    double* V0 = V;
    orc_copy(N, r, V0);
    orc_scal(N, 1.0 / beta, V0);
    memset(s, 0, (size_t)(m + 1) * sizeof(double));
    s[0] = beta;
    int i = 0;
    /* Iteration inner(outer): copies tolerance and facteur_reste; its
     * max_iter is outer's count + m (Gmres.cxx:114-116). */
    orc_iter inner = *outer;
    inner.max_iter = outer->nb_iter + m;
    int stop;
    do {
      double* Vi = V + (size_t)i * N;
      csr_mlt(A, Vi, u);
      prec_solve(M, A, u, w);
      for (int k = 0; k <= i; k++) {
        double h = orc_dot(N, V + (size_t)k * N, w);
        H[k + (size_t)i * ld] = h;
        orc_axpy(N, -h, V + (size_t)k * N, w);
      }
      double hi_ip1 = orc_nrm2(N, w);
      double* Vn = V + (size_t)(i + 1) * N;
      orc_copy(N, w, Vn);
      if (hi_ip1 != 0.0) orc_scal(N, 1.0 / hi_ip1, Vn);
      for (int k = 0; k < i; k++)
        orc_applyrot(&H[k + (size_t)i * ld], &H[k + 1 + (size_t)i * ld], rc[k],
                     rs[k]);
      if (hi_ip1 != 0.0) {
        orc_genrot(&H[i + (size_t)i * ld], &hi_ip1, &rc[i], &rs[i]);
        orc_applyrot(&s[i], &s[i + 1], rc[i], rs[i]);
      }
      inner.nb_iter++;
      outer->nb_iter++;
      i++;
      stop = it_finished(&inner, fabs(s[i]));
    } while (!stop);
    /* the inner log entries belong to the caller's history */
    outer->hist_len = inner.hist_len;

    orc_trsv_upper(i, H, ld, s);
    for (int k = 0; k < i; k++) orc_axpy(N, s[k], V + (size_t)k * N, x);

    orc_copy(N, b, w);
    csr_residual(A, x, w);
    prec_solve(M, A, w, r);
    beta = orc_nrm2(N, r);
  }
  code = it_error_code(outer);
out:
  free(V); free(H); free(w); free(r); free(u); free(s); free(rc); free(rs);
  return code;
}

/* Cgs, computation/solver/iterative/Cgs.cxx:45-132.  Right preconditioning;
 * the test is on the unpreconditioned residual and the count advances by two
 * per loop (after each product). */
static int orc_cgs_impl(const orc_csr* A, double* x, const double* b,
                        const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  double rho_1, rho_2 = 0.0, alpha, beta, delta;
  size_t bytes = (size_t)N * sizeof(double);
  double *p = malloc(bytes), *phat = malloc(bytes), *q = malloc(bytes),
         *qhat = malloc(bytes), *vhat = malloc(bytes), *u = malloc(bytes),
         *uhat = malloc(bytes), *r = malloc(bytes), *rtilde = malloc(bytes);
  double* all[9] = {p, phat, q, qhat, vhat, u, uhat, r, rtilde};
  for (int k = 0; k < 9; k++) memcpy(all[k], b, bytes);
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  orc_copy(N, r, rtilde);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r))) {
    rho_1 = orc_dot(N, rtilde, r);
    if (rho_1 == 0.0) { it_fail(it, 1); break; }
    if (it->nb_iter == 0) {
      orc_copy(N, r, u);
      orc_copy(N, u, p);
    } else {
      /* u = r + beta q;  p = beta (beta p + q) + u */
      beta = rho_1 / rho_2;
      orc_copy(N, r, u);
      orc_axpy(N, beta, q, u);
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, q, p);
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, u, p);
    }
    prec_solve(M, A, p, phat);
    csr_mlt(A, phat, vhat);
    it->nb_iter++;
    delta = orc_dot(N, rtilde, vhat);
    if (delta == 0.0) { it_fail(it, 2); break; }
    alpha = rho_1 / delta;
    orc_copy(N, u, q);
    orc_axpy(N, -alpha, vhat, q);
    orc_axpy(N, 1.0, q, u);
    prec_solve(M, A, u, uhat);
    orc_axpy(N, alpha, uhat, x);
    csr_mlt(A, uhat, qhat);
    orc_axpy(N, -alpha, qhat, r);
    rho_2 = rho_1;
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  for (int k = 0; k < 9; k++) free(all[k]);
  return code;
}

/* TfQmr, computation/solver/iterative/TfQmr.cxx:44-243.  Left
 * preconditioning; two half steps per loop, each ending with the scalar
 * test Finished(kappa) (Iterative.cxx:299-319) on the quasi-residual bound
 * kappa = tau sqrt(m + 1). */
static int orc_tfqmr_impl(const orc_csr* A, double* x, const double* b,
                          const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *tmp = malloc(bytes), *r0 = malloc(bytes), *v = malloc(bytes),
         *h = malloc(bytes), *w = malloc(bytes), *y1 = malloc(bytes),
         *g = malloc(bytes), *y0 = malloc(bytes), *rtilde = malloc(bytes),
         *d = malloc(bytes);
  double* all[10] = {tmp, r0, v, h, w, y1, g, y0, rtilde, d};
  for (int k = 0; k < 10; k++) memcpy(all[k], b, bytes);
  double sigma, alpha, beta, eta, rho, rho0, c, kappa, tau, theta;
  int code;
  memset(tmp, 0, bytes);
  /* 1. r0 = M^{-1} (b - A x) */
  orc_copy(N, b, tmp);
  if (!it->init_guess_null)
    csr_residual(A, x, tmp);
  else
    memset(x, 0, bytes);
  prec_solve(M, A, tmp, r0);
  if (it_init(it, N, r0) != 0) { code = it_error_code(it); goto out; }
  /* 2.-3. w = y = r0; g = v = M^{-1} A y */
  orc_copy(N, r0, w);
  orc_copy(N, r0, y1);
  orc_copy(N, y1, v);
  csr_mlt(A, v, tmp);
  prec_solve(M, A, tmp, v);
  it->nb_iter++;
  orc_copy(N, v, g);
  /* 4.-8. */
  memset(d, 0, bytes);
  tau = orc_nrm2(N, r0);
  theta = 0.0;
  eta = 0.0;
  orc_copy(N, r0, rtilde);
  rho = orc_dot(N, rtilde, r0);
  rho0 = rho;
  it->nb_iter = 0;
  for (;;) {
    sigma = orc_dot(N, rtilde, v);
    if (sigma == 0.0) { it_fail(it, 1); break; }
    alpha = rho / sigma;
    orc_copy(N, y1, y0);
    orc_axpy(N, -alpha, v, y0);
    orc_copy(N, y0, h);
    csr_mlt(A, h, tmp);
    prec_solve(M, A, tmp, h);
    /* first half step (m = 2k - 1) */
    orc_axpy(N, -alpha, g, w);
    if (alpha == 0.0) { it_fail(it, 2); break; }
    orc_scal(N, theta * theta * eta / alpha, d);
    orc_axpy(N, 1.0, y1, d);
    if (tau == 0.0) { it_fail(it, 3); break; }
    theta = orc_nrm2(N, w) / tau;
    c = 1.0 / sqrt(1.0 + theta * theta);
    tau = tau * c * theta;
    eta = c * c * alpha;
    orc_axpy(N, eta, d, x);
    kappa = tau * sqrt(2. * (it->nb_iter + 1));
    if (it_finished(it, kappa)) break;
    it->nb_iter++;
    /* second half step (m = 2k) */
    orc_copy(N, h, g);
    orc_axpy(N, -alpha, g, w);
    orc_scal(N, theta * theta * eta / alpha, d);
    orc_axpy(N, 1.0, y0, d);
    if (tau == 0.0) { it_fail(it, 4); break; }
    theta = orc_nrm2(N, w) / tau;
    c = 1.0 / sqrt(1.0 + theta * theta);
    tau = tau * c * theta;
    eta = c * c * alpha;
    orc_axpy(N, eta, d, x);
    kappa = tau * sqrt(2. * (it->nb_iter + 1) + 1.);
    if (it_finished(it, kappa)) break;
    /* 22.-26. */
    rho0 = rho;
    rho = orc_dot(N, rtilde, w);
    if (rho0 == 0.0) { it_fail(it, 5); break; }
    beta = rho / rho0;
    orc_copy(N, w, y1);
    orc_axpy(N, beta, y0, y1);
    orc_copy(N, y1, g);
    csr_mlt(A, g, tmp);
    prec_solve(M, A, tmp, g);
    orc_scal(N, beta * beta, v);
    orc_axpy(N, beta, h, v);
    orc_axpy(N, 1.0, g, v);
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  for (int k = 0; k < 10; k++) free(all[k]);
  return code;
}

/* MinRes, computation/solver/iterative/MinRes.cxx:46-153.  Symmetric A and
 * M; the test is on the recurrence's residual estimate np (||b|| times the
 * product of the |s| of the rotations so far). */
static int orc_minres_impl(const orc_csr* A, double* x, const double* b,
                           const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *u_old = malloc(bytes), *u = malloc(bytes), *r = malloc(bytes),
         *v_old = malloc(bytes), *v = malloc(bytes), *w_old = malloc(bytes),
         *w = malloc(bytes), *z = malloc(bytes), *w_oold = malloc(bytes);
  double* all[9] = {u_old, u, r, v_old, v, w_old, w, z, w_oold};
  for (int k = 0; k < 9; k++) memcpy(all[k], b, bytes);
  double dp, beta, ibeta, beta_old, alpha, eta, ceta;
  double cold, coold, c, soold, sold, s, rho0, rho1, rho2, rho3, np;
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  memset(u_old, 0, bytes); memset(v_old, 0, bytes); memset(w_old, 0, bytes);
  memset(w, 0, bytes); memset(w_oold, 0, bytes);
  prec_solve(M, A, r, z);
  dp = orc_dot(N, r, z);
  dp = sqrt(dp);
  beta = dp;
  eta = beta;
  orc_copy(N, r, v);
  orc_copy(N, z, u);
  ibeta = 1.0 / beta;
  orc_scal(N, ibeta, v);
  orc_scal(N, ibeta, u);
  c = 1.0; s = 0.0; cold = 1.0; sold = 0.0;
  np = orc_nrm2(N, b);
  it->nb_iter = 0;
  while (!it_finished(it, np)) {
    csr_mlt(A, u, r);
    alpha = orc_dot(N, r, u);
    prec_solve(M, A, r, z);
    orc_axpy(N, -alpha, v, r);
    orc_axpy(N, -alpha, u, z);
    orc_axpy(N, -beta, v_old, r);
    orc_axpy(N, -beta, u_old, z);
    beta_old = beta;
    dp = orc_dot(N, r, z);
    beta = sqrt(dp);
    /* QR factorization */
    coold = cold; cold = c; soold = sold; sold = s;
    rho0 = cold * alpha - coold * sold * beta_old;
    rho1 = sqrt(rho0 * rho0 + beta * beta);
    rho2 = sold * alpha + coold * cold * beta_old;
    rho3 = soold * beta_old;
    if (rho1 == 0.0) { it_fail(it, 1); break; }
    c = rho0 / rho1;
    s = beta / rho1;
    orc_copy(N, w_old, w_oold);
    orc_copy(N, w, w_old);
    orc_copy(N, u, w);
    orc_axpy(N, -rho2, w_old, w);
    orc_axpy(N, -rho3, w_oold, w);
    orc_scal(N, 1. / rho1, w);
    ceta = c * eta;
    orc_axpy(N, ceta, w, x);
    eta = -s * eta;
    orc_copy(N, v, v_old);
    orc_copy(N, u, u_old);
    orc_copy(N, r, v);
    orc_copy(N, z, u);
    if (beta == 0.0) { it_fail(it, 2); break; }
    ibeta = 1.0 / beta;
    orc_scal(N, ibeta, v);
    orc_scal(N, ibeta, u);
    np *= fabs(s);
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  for (int k = 0; k < 9; k++) free(all[k]);
  return code;
}

/* Gcr(m), computation/solver/iterative/Gcr.cxx:45-141.  Restarted
 * generalized conjugate residuals, left preconditioned, the test on
 * ||M^{-1}(b - A x)|| / ||b||.  Each cycle runs an inner Iteration copied
 * from the outer one (Iterative.cxx:114-124) whose limit is the outer count
 * plus m; both test the same residual, and both tests are logged.  Where
 * the reference never returns -- a cycle whose inner loop takes no step (a
 * breakdown at its first product, or m = 0), after which every cycle
 * repeats it -- this stops after that cycle. */
static int orc_gcr_impl(const orc_csr* A, double* x, const double* b,
                        const orc_prec* M, orc_iter* outer, int m) {
  const int N = A->m;
  if (N <= 0) return 0;
  if (it_init(outer, N, b) != 0) return it_error_code(outer);
  size_t bytes = (size_t)N * sizeof(double);
  const int nm = m > 0 ? m : 0;
  double* P = calloc((size_t)(nm + 1) * N, sizeof(double));
  double* Wv = calloc((size_t)(nm + 1) * N, sizeof(double));
  double* beta = calloc((size_t)(nm + 1), sizeof(double));
  double *r = malloc(bytes), *q = malloc(bytes), *u = malloc(bytes);
  memcpy(r, b, bytes); memcpy(q, b, bytes); memcpy(u, b, bytes);
  orc_copy(N, b, u);
  if (!outer->init_guess_null)
    csr_residual(A, x, u);
  else
    memset(x, 0, bytes);
  prec_solve(M, A, u, r);
  double alpha, delta, normr = orc_nrm2(N, r);
  outer->nb_iter = 0;
  while (!it_finished(outer, orc_nrm2(N, r))) {
    orc_iter inner = *outer;
    inner.max_iter = outer->nb_iter + m;
    orc_copy(N, r, P);
    orc_scal(N, 1.0 / normr, P);
    int j = 0;
    while (!it_finished(&inner, orc_nrm2(N, r))) {
      double *pj = P + (size_t)j * N, *wj = Wv + (size_t)j * N;
      csr_mlt(A, pj, u);
      prec_solve(M, A, u, wj);
      beta[j] = orc_dot(N, wj, wj);
      if (beta[j] == 0.0) { it_fail(outer, 1); break; }
      alpha = orc_dot(N, wj, r) / beta[j];
      orc_axpy(N, alpha, pj, x);
      orc_axpy(N, -alpha, wj, r);
      inner.nb_iter++;
      outer->nb_iter++;
      csr_mlt(A, r, u);
      prec_solve(M, A, u, q);
      double* pn = P + (size_t)(j + 1) * N;
      orc_copy(N, r, pn);
      for (int i = 0; i <= j; i++) {
        delta = -orc_dot(N, Wv + (size_t)i * N, q) / beta[i];
        orc_axpy(N, delta, P + (size_t)i * N, pn);
      }
      inner.nb_iter++;
      outer->nb_iter++;
      j++;
    }
    outer->hist_len = inner.hist_len;
    if (j == 0) break; /* the reference would repeat this cycle for ever */
    normr = orc_nrm2(N, r);
  }
  int code = it_error_code(outer);
  free(P); free(Wv); free(beta); free(r); free(q); free(u);
  return code;
}

/* BiCgStabl(l), computation/solver/iterative/BiCgStabl.cxx:43-180, with
 * l = the restart parameter.  Right preconditioning: x gathers u's in the
 * preconditioned coordinates and is mapped back by M^{-1} at the end; the
 * test is on ||r_0|| / ||b||, the count advances by two per BiCG step.  A
 * breakdown ends the BiCG part only; the MR part and the loop go on.  tau
 * and the gammas carry over from cycle to cycle, as the reference's do.
 * Where the reference can repeat a cycle for ever -- one that counts no
 * iteration (a breakdown at the first step) -- this stops after it. */
static int orc_bicgstabl_impl(const orc_csr* A, double* x, const double* b,
                              const orc_prec* M, orc_iter* it, int m) {
  const int N = A->m;
  if (N <= 0) return 0;
  /* l = 0 reads gamma(1) past the end of a one-entry vector in the
   * reference: no result to restate */
  if (m < 1) return -100;
  const int l = m;
  size_t bytes = (size_t)N * sizeof(double);
  double *q = malloc(bytes), *r0 = malloc(bytes);
  memcpy(q, b, bytes); memcpy(r0, b, bytes);
  double* R = calloc((size_t)(l + 1) * N, sizeof(double));
  double* U = calloc((size_t)(l + 1) * N, sizeof(double));
  double* gamma = calloc((size_t)(l + 1), sizeof(double));
  double* gamma_p = calloc((size_t)(l + 1), sizeof(double));
  double* gamma_t = calloc((size_t)(l + 1), sizeof(double));
  double* tau = calloc((size_t)(l + 1) * (l + 1), sizeof(double));
#define TAU(i, j) tau[(size_t)(i) * (l + 1) + (j)]
#define RV(i) (R + (size_t)(i) * N)
#define UV(i) (U + (size_t)(i) * N)
  double rho_0, rho_1, alpha, beta, omega, sigma;
  int code;
  orc_copy(N, b, RV(0));
  if (!it->init_guess_null)
    csr_residual(A, x, RV(0));
  else
    memset(x, 0, bytes);
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, RV(0), r0);
  rho_0 = 1.0; alpha = 0.0; omega = 1.0;
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, RV(0)))) {
    const int start = it->nb_iter;
    rho_0 *= -omega;
    /* Bi-CG part */
    for (int j = 0; j < l; j++) {
      rho_1 = orc_dot(N, RV(j), r0);
      if (rho_0 == 0.0) { it_fail(it, 1); break; }
      beta = alpha * (rho_1 / rho_0);
      rho_0 = rho_1;
      for (int i = 0; i <= j; i++) {
        orc_scal(N, -beta, UV(i));
        orc_axpy(N, 1.0, RV(i), UV(i));
      }
      prec_solve(M, A, UV(j), q);
      csr_mlt(A, q, UV(j + 1));
      it->nb_iter++;
      sigma = orc_dot(N, UV(j + 1), r0);
      if (sigma == 0.0) { it_fail(it, 2); break; }
      alpha = rho_1 / sigma;
      orc_axpy(N, alpha, UV(0), x);
      for (int i = 0; i <= j; i++) orc_axpy(N, -alpha, UV(i + 1), RV(i));
      prec_solve(M, A, RV(j), q);
      csr_mlt(A, q, RV(j + 1));
      it->nb_iter++;
    }
    /* MR part, modified Gram-Schmidt */
    for (int j = 1; j <= l; j++) {
      for (int i = 1; i < j; i++) {
        if (gamma[i] != 0.0) {
          TAU(i, j) = orc_dot(N, RV(j), RV(i)) / gamma[i];
          orc_axpy(N, -TAU(i, j), RV(i), RV(j));
        }
      }
      gamma[j] = orc_dot(N, RV(j), RV(j));
      if (gamma[j] != 0.0) gamma_p[j] = orc_dot(N, RV(0), RV(j)) / gamma[j];
    }
    /* gamma = tau^{-1} gamma' */
    gamma[l] = gamma_p[l];
    omega = gamma[l];
    for (int j = l - 1; j >= 1; j--) {
      sigma = 0.0;
      for (int i = j + 1; i <= l; i++) sigma += TAU(j, i) * gamma[i];
      gamma[j] = gamma_p[j] - sigma;
    }
    /* gamma'' = T S gamma */
    for (int j = 1; j <= l - 1; j++) {
      sigma = 0.0;
      for (int i = j + 1; i <= l - 1; i++) sigma += TAU(j, i) * gamma[i + 1];
      gamma_t[j] = gamma[j + 1] + sigma;
    }
    /* update */
    orc_axpy(N, gamma[1], RV(0), x);
    orc_axpy(N, -gamma_p[l], RV(l), RV(0));
    orc_axpy(N, -gamma[l], UV(l), UV(0));
    for (int j = 1; j <= l - 1; j++) {
      orc_axpy(N, -gamma[j], UV(j), UV(0));
      orc_axpy(N, gamma_t[j], RV(j), x);
      orc_axpy(N, -gamma_p[j], RV(j), RV(0));
    }
    if (it->nb_iter == start) break; /* the reference may repeat this for ever */
  }
  /* change of coordinates (right preconditioning) */
  orc_copy(N, x, q);
  prec_solve(M, A, q, x);
  code = it_error_code(it);
out:
#undef TAU
#undef RV
#undef UV
  free(q); free(r0); free(R); free(U); free(gamma); free(gamma_p); free(gamma_t); free(tau);
  return code;
}

/* QCgs, computation/solver/iterative/QCgs.cxx:46-165: Cgs with a
 * quasi-minimal smoothing step (a 2 x 2 least-squares fit on
 * r_qcgs - r and v per loop).  The test is on ||r_qcgs|| / ||b||; x is
 * replaced by M^{-1} x_qcgs at the end, breakdown or not. */
static int orc_qcgs_impl(const orc_csr* A, double* x, const double* b,
                         const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *p = malloc(bytes), *q = malloc(bytes), *r = malloc(bytes),
         *rtilde = malloc(bytes), *u = malloc(bytes), *phat = malloc(bytes),
         *r_q = malloc(bytes), *x_q = malloc(bytes), *v = malloc(bytes);
  double* all[9] = {p, q, r, rtilde, u, phat, r_q, x_q, v};
  for (int k = 0; k < 9; k++) memcpy(all[k], b, bytes);
  double rho_1, rho_2, mu, nu, alpha, beta, sigma, delta;
  double b00, b11, b10, m00, m11, m10, rn0, rn1;
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  orc_copy(N, r, rtilde);
  rho_1 = 1.0;
  memset(q, 0, bytes);
  memset(p, 0, bytes);
  orc_copy(N, r, r_q);
  orc_copy(N, x, x_q);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r_q))) {
    rho_2 = orc_dot(N, rtilde, r);
    if (rho_1 == 0.0) { it_fail(it, 1); break; }
    beta = rho_2 / rho_1;
    orc_copy(N, r, u);
    orc_axpy(N, beta, q, u);
    orc_scal(N, beta, p);
    orc_axpy(N, 1.0, q, p);
    orc_scal(N, beta, p);
    orc_axpy(N, 1.0, u, p);
    prec_solve(M, A, p, phat);
    csr_mlt(A, phat, v);
    it->nb_iter++;
    sigma = orc_dot(N, rtilde, v);
    if (sigma == 0.0) { it_fail(it, 2); break; }
    alpha = rho_2 / sigma;
    orc_copy(N, u, q);
    orc_axpy(N, -alpha, v, q);
    orc_axpy(N, 1.0, q, u);
    orc_axpy(N, alpha, u, x);
    prec_solve(M, A, u, phat);
    csr_mlt(A, phat, u);
    orc_axpy(N, -alpha, u, r);
    orc_copy(N, r_q, u);
    orc_axpy(N, -1.0, r, u);
    b00 = orc_dot(N, u, u);
    b11 = orc_dot(N, v, v);
    b10 = orc_dot(N, u, v);
    /* inverse of the symmetric 2 x 2 matrix (b(0,1) is b(1,0)) */
    delta = b00 * b11 - b10 * b10;
    if (delta == 0.0) { it_fail(it, 3); break; }
    m00 = b11 / delta;
    m11 = b00 / delta;
    m10 = -b10 / delta;
    rn0 = -orc_dot(N, u, r);
    rn1 = -orc_dot(N, v, r);
    mu = m00 * rn0 + m10 * rn1;
    nu = m10 * rn0 + m11 * rn1;
    /* smoothing step */
    orc_copy(N, r, r_q);
    orc_axpy(N, mu, u, r_q);
    orc_axpy(N, nu, v, r_q);
    orc_scal(N, mu, x_q);
    orc_axpy(N, 1.0 - mu, x, x_q);
    orc_axpy(N, -nu, p, x_q);
    rho_1 = rho_2;
    it->nb_iter++;
  }
  prec_solve(M, A, x_q, x);
  code = it_error_code(it);
out:
  for (int k = 0; k < 9; k++) free(all[k]);
  return code;
}

/* M^{-T} r: SorPreconditioner::TransSolve sweeps backward (type 3) when
 * the preconditioner is not symmetric (Precond_Ssor.cxx:78-90); the
 * identity and Jacobi are their own transposes. */
static void prec_trans_solve(const orc_prec* M, const orc_csr* A, const double* r,
                             double* z) {
  if (M->kind != 2) {
    prec_solve(M, A, r, z);
    return;
  }
  memset(z, 0, (size_t)A->m * sizeof(double));
  orc_sor(A->m, A->ptr, A->ind, A->val, A->sym, z, r, M->omega, M->nb_iter,
          M->symmetric ? 0 : 3);
}

/* Mlt(SeldonTrans, M, X, Y) (Functions_MatVect.cxx:122-130) passes its
 * flag as the base type SeldonTranspose, so the generic MltAdd runs
 * (:1279-1317): Y(i) = 0 + 1 * sum_j M(j, i) X(j), j increasing, over every
 * j (the absent entries add zeros, which change no sum).  For RowSparse
 * that is column i's entries in increasing row order, as the column
 * scatter below adds them; for RowSymSparse, M(j, i) = M(i, j), so row i of
 * the full symmetric matrix in increasing column order: the strict lower
 * part (`lp/li/lv`, the upper part transposed, built once by the caller)
 * then the stored upper row. */
static void csr_mlt_trans(const orc_csr* A, const int* lp, const int* li,
                          const double* lv, const double* x, double* y) {
  memset(y, 0, (size_t)A->n * sizeof(double));
  if (!A->sym) {
    orc_mltadd(A->m, A->n, A->ptr, A->ind, A->val, 0, 1, 1.0, x, 0.0, y);
    return;
  }
  for (int i = 0; i < A->m; i++) {
    double t = 0.0;
    for (int k = lp[i]; k < lp[i + 1]; k++) t += lv[k] * x[li[k]];
    for (int k = A->ptr[i]; k < A->ptr[i + 1]; k++) t += A->val[k] * x[A->ind[k]];
    y[i] += 1.0 * t;
  }
}

/* The strict lower part of a RowSymSparse matrix as CSR (the strict upper
 * part transposed), columns increasing within each row. */
static void sym_lower(const orc_csr* A, int** lp, int** li, double** lv) {
  const int n = A->m;
  int* p = calloc((size_t)n + 1, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int k = A->ptr[i]; k < A->ptr[i + 1]; k++)
      if (A->ind[k] > i) p[A->ind[k] + 1]++;
  for (int i = 0; i < n; i++) p[i + 1] += p[i];
  int* fill = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) fill[i] = p[i];
  int* c = malloc(sizeof(int) * (size_t)(p[n] > 0 ? p[n] : 1));
  double* v = malloc(sizeof(double) * (size_t)(p[n] > 0 ? p[n] : 1));
  for (int i = 0; i < n; i++)
    for (int k = A->ptr[i]; k < A->ptr[i + 1]; k++)
      if (A->ind[k] > i) {
        const int q = fill[A->ind[k]]++;
        c[q] = i;
        v[q] = A->val[k];
      }
  free(fill);
  *lp = p;
  *li = c;
  *lv = v;
}

/* BiCg, computation/solver/iterative/BiCg.cxx:46-134: biconjugate
 * gradients, M^{-1} on the residual and M^{-T} on the shadow residual, one
 * product with A and one with A^T per loop. */
static int orc_bicg_impl(const orc_csr* A, double* x, const double* b,
                         const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *r = malloc(bytes), *z = malloc(bytes), *p = malloc(bytes),
         *q = malloc(bytes), *rt = malloc(bytes), *zt = malloc(bytes),
         *pt = malloc(bytes), *qt = malloc(bytes);
  double* all[8] = {r, z, p, q, rt, zt, pt, qt};
  for (int k = 0; k < 8; k++) memcpy(all[k], b, bytes);
  double rho_1, rho_2 = 0.0, alpha, beta, delta;
  int code;
  int *lp = NULL, *li = NULL;
  double* lv = NULL;
  if (A->sym) sym_lower(A, &lp, &li, &lv);
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  orc_copy(N, r, rt);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r))) {
    /* z = M^{-1} r, zt = M^{-T} rt (SOR's TransSolve sweeps backward) */
    prec_solve(M, A, r, z);
    prec_trans_solve(M, A, rt, zt);
    rho_1 = orc_dot(N, z, rt);
    if (rho_1 == 0.0) { it_fail(it, 1); break; }
    if (it->nb_iter == 0) {
      orc_copy(N, z, p);
      orc_copy(N, zt, pt);
    } else {
      beta = rho_1 / rho_2;
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, z, p);
      orc_scal(N, beta, pt);
      orc_axpy(N, 1.0, zt, pt);
    }
    csr_mlt(A, p, q);
    it->nb_iter++;
    csr_mlt_trans(A, lp, li, lv, pt, qt);
    delta = orc_dot(N, pt, q);
    if (delta == 0.0) { it_fail(it, 2); break; }
    alpha = rho_1 / delta;
    orc_axpy(N, alpha, p, x);
    orc_axpy(N, -alpha, q, r);
    orc_axpy(N, -alpha, qt, rt);
    rho_2 = rho_1;
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  for (int k = 0; k < 8; k++) free(all[k]);
  free(lp); free(li); free(lv);
  return code;
}

/* Cgne, computation/solver/iterative/Cgne.cxx:40-127: CG on the normal
 * equations A^T A x = A^T b, M^{-T} then M^{-1} on r.  The test is on
 * ||r|| / ||A^T b||, and the first one on ||A^T b|| itself even from an
 * initial guess; the count advances by two per loop. */
static int orc_cgne_impl(const orc_csr* A, double* x, const double* b,
                         const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *p = malloc(bytes), *q = malloc(bytes), *r = malloc(bytes), *z = malloc(bytes);
  memcpy(p, b, bytes); memcpy(q, b, bytes); memcpy(r, b, bytes); memcpy(z, b, bytes);
  int *lp = NULL, *li = NULL;
  double* lv = NULL;
  if (A->sym) sym_lower(A, &lp, &li, &lv);
  double rho = 1.0, rho_1 = 0.0, alpha, beta, delta, dp;
  int code;
  csr_mlt_trans(A, lp, li, lv, b, q);
  if (it_init(it, N, q) != 0) { code = it_error_code(it); goto out; }
  if (!it->init_guess_null) {
    csr_mlt(A, x, p);
    csr_mlt_trans(A, lp, li, lv, p, r);
    orc_scal(N, -1.0, r);
    orc_axpy(N, 1.0, q, r);
  } else {
    orc_copy(N, q, r);
    memset(x, 0, bytes);
  }
  dp = orc_nrm2(N, q);
  it->nb_iter = 0;
  while (!it_finished(it, dp)) {
    prec_trans_solve(M, A, r, q);
    prec_solve(M, A, q, z);
    rho = orc_dot(N, r, z);
    if (rho == 0.0) { it_fail(it, 1); break; }
    if (it->nb_iter == 0)
      orc_copy(N, z, p);
    else {
      beta = rho / rho_1;
      orc_scal(N, beta, p);
      orc_axpy(N, 1.0, z, p);
    }
    csr_mlt(A, p, q);
    csr_mlt_trans(A, lp, li, lv, q, z);
    delta = orc_dot(N, p, z);
    if (delta == 0.0) { it_fail(it, 2); break; }
    alpha = rho / delta;
    orc_axpy(N, alpha, p, x);
    orc_axpy(N, -alpha, z, r);
    rho_1 = rho;
    dp = orc_nrm2(N, r);
    it->nb_iter += 2;
  }
  code = it_error_code(it);
out:
  free(p); free(q); free(r); free(z); free(lp); free(li); free(lv);
  return code;
}

/* BiCgcr.cxx:44-118: biconjugate conjugate residuals.  One product a step;
 * the count starts at 1 (the initial product a = A p is counted) and the
 * test is on the unpreconditioned residual v. */
static int orc_bicgcr_impl(const orc_csr* A, double* x, const double* b,
                           const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *v = calloc(N, sizeof(double)), *w = calloc(N, sizeof(double)),
         *s = calloc(N, sizeof(double)), *z = calloc(N, sizeof(double)),
         *p = calloc(N, sizeof(double)), *a = calloc(N, sizeof(double));
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  memcpy(v, b, bytes);
  if (!it->init_guess_null)
    csr_residual(A, x, v);
  else
    memset(x, 0, bytes);
  it->nb_iter = 0;
  prec_solve(M, A, v, s);
  orc_copy(N, s, p);
  csr_mlt(A, p, a);
  prec_solve(M, A, a, w);
  it->nb_iter++;
  while (!it_finished(it, orc_nrm2(N, v))) {
    double rho = orc_dot(N, w, v), mu = orc_dot(N, w, a);
    if (mu == 0.0) { it_fail(it, 1); break; }
    double alpha = rho / mu;
    orc_axpy(N, alpha, p, x);
    orc_axpy(N, -alpha, a, v);
    orc_axpy(N, -alpha, w, s);
    csr_mlt(A, s, z);
    double tau = orc_dot(N, w, z);
    if (tau == 0.0) { it_fail(it, 2); break; }
    double beta = tau / mu;
    orc_scal(N, -beta, p);
    orc_axpy(N, 1.0, s, p);
    orc_scal(N, -beta, a);
    orc_axpy(N, 1.0, z, a);
    prec_solve(M, A, a, w);
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  free(v); free(w); free(s); free(z); free(p); free(a);
  return code;
}

/* Lsqr.cxx:40-135: Golub-Kahan bidiagonalisation on A and A^T.  The
 * preconditioner is not used.  The initial guess enters only the first test
 * (rnorm = ||b - A x0||): x is zeroed and u starts from b either way.  The
 * test is on |phi_bar| after the first, and the count advances by two a
 * loop. */
static int orc_lsqr_impl(const orc_csr* A, double* x, const double* b, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *v = malloc(bytes), *v1 = malloc(bytes), *u = malloc(bytes),
         *u1 = malloc(bytes), *w = malloc(bytes);
  memcpy(v, b, bytes); memcpy(v1, b, bytes); memcpy(u, b, bytes);
  memcpy(u1, b, bytes); memcpy(w, b, bytes);
  int *lp = NULL, *li = NULL;
  double* lv = NULL;
  if (A->sym) sym_lower(A, &lp, &li, &lv);
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, u);
  if (!it->init_guess_null)
    csr_residual(A, x, u);
  else
    memset(x, 0, bytes);
  double rnorm = orc_nrm2(N, u);
  orc_copy(N, b, u);
  double beta = orc_nrm2(N, u);
  orc_scal(N, 1.0 / beta, u);
  csr_mlt_trans(A, lp, li, lv, u, v);
  double alpha = orc_nrm2(N, v);
  orc_scal(N, 1.0 / alpha, v);
  orc_copy(N, v, w);
  memset(x, 0, bytes);
  double phi_bar = beta, rho_bar = alpha;
  it->nb_iter = 0;
  while (!it_finished(it, rnorm)) {
    csr_mlt(A, v, u1);
    orc_axpy(N, -alpha, u, u1);
    beta = orc_nrm2(N, u1);
    if (beta == 0.0) { it_fail(it, 1); break; }
    orc_scal(N, 1.0 / beta, u1);
    csr_mlt_trans(A, lp, li, lv, u1, v1);
    orc_axpy(N, -beta, v, v1);
    alpha = orc_nrm2(N, v1);
    if (alpha == 0.0) { it_fail(it, 2); break; }
    orc_scal(N, 1.0 / alpha, v1);
    double rho = sqrt(rho_bar * rho_bar + beta * beta);
    if (rho == 0.0) { it_fail(it, 3); break; }
    double c = rho_bar / rho, s = beta / rho;
    double theta = s * alpha;
    rho_bar = -c * alpha;
    double phi = c * phi_bar;
    phi_bar = s * phi_bar;
    orc_axpy(N, phi / rho, w, x);
    orc_scal(N, -theta / rho, w);
    orc_axpy(N, 1.0, v1, w);
    rnorm = fabs(phi_bar);
    double* t = u1; u1 = u; u = t;
    t = v1; v1 = v; v = t;
    it->nb_iter += 2;
  }
  code = it_error_code(it);
out:
  free(v); free(v1); free(u); free(u1); free(w); free(lp); free(li); free(lv);
  return code;
}

/* QmrSym.cxx:41-165: QMR for symmetric systems, one product a step.  Its
 * Fail codes are 1, 3, 4, 5 and 6 (the messages number them #1 to #5). */
static int orc_qmrsym_impl(const orc_csr* A, double* x, const double* b,
                           const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *r = malloc(bytes), *y = malloc(bytes), *v = malloc(bytes),
         *pt = malloc(bytes), *p = malloc(bytes), *d = malloc(bytes), *s = malloc(bytes);
  memcpy(r, b, bytes); memcpy(y, b, bytes); memcpy(v, b, bytes); memcpy(pt, b, bytes);
  memcpy(p, b, bytes); memcpy(d, b, bytes); memcpy(s, b, bytes);
  double delta, ep = 0.0, beta, rho, rho_1, theta_1, gamma_1;
  double theta = 0.0, gamma = 1.0, eta = -1.0;
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  orc_copy(N, r, v);
  prec_solve(M, A, v, y);
  rho = orc_nrm2(N, y);
  it->nb_iter = 0;
  while (!it_finished(it, orc_nrm2(N, r))) {
    if (rho == 0.0) { it_fail(it, 1); break; }
    orc_scal(N, 1. / rho, v);
    orc_scal(N, 1. / rho, y);
    delta = orc_dot(N, v, y);
    if (delta == 0.0) { it_fail(it, 3); break; }
    if (it->nb_iter == 0)
      orc_copy(N, y, p);
    else {
      orc_scal(N, -(rho * delta / ep), p);
      orc_axpy(N, 1.0, y, p);
    }
    csr_mlt(A, p, pt);
    ep = orc_dot(N, p, pt);
    if (ep == 0.0) { it_fail(it, 4); break; }
    beta = ep / delta;
    if (beta == 0.0) { it_fail(it, 5); break; }
    orc_scal(N, -beta, v);
    orc_axpy(N, 1.0, pt, v);
    prec_solve(M, A, v, y);
    rho_1 = rho;
    rho = orc_nrm2(N, y);
    gamma_1 = gamma;
    theta_1 = theta;
    theta = rho / (gamma_1 * beta);
    gamma = 1.0 / sqrt(1.0 + theta * theta);
    if (gamma == 0.0) { it_fail(it, 6); break; }
    eta = -eta * rho_1 * gamma * gamma / (beta * gamma_1 * gamma_1);
    if (it->nb_iter == 0) {
      orc_copy(N, p, d);
      orc_scal(N, eta, d);
      orc_copy(N, pt, s);
      orc_scal(N, eta, s);
    } else {
      double tmp = theta_1 * theta_1 * gamma * gamma;
      orc_scal(N, tmp, d);
      orc_axpy(N, eta, p, d);
      orc_scal(N, tmp, s);
      orc_axpy(N, eta, pt, s);
    }
    orc_axpy(N, 1.0, d, x);
    orc_axpy(N, -1.0, s, r);
    it->nb_iter++;
  }
  code = it_error_code(it);
out:
  free(r); free(y); free(v); free(pt); free(p); free(d); free(s);
  return code;
}

/* Symmlq.cxx:45-161: SYMMLQ (Lanczos with an LQ factorisation).  The first
 * test is on ||b|| even from an initial guess; later ones on the estimate
 * s_prod / |c|.  x takes its last correction ceta_bar * w_bar after the
 * loop, whichever way the loop ended.  No Fail code. */
static int orc_symmlq_impl(const orc_csr* A, double* x, const double* b,
                           const orc_prec* M, orc_iter* it) {
  const int N = A->m;
  if (N <= 0) return 0;
  size_t bytes = (size_t)N * sizeof(double);
  double *r = malloc(bytes), *z = malloc(bytes), *u = malloc(bytes), *v = malloc(bytes),
         *w = calloc(N, sizeof(double)), *u_old = calloc(N, sizeof(double)),
         *v_old = calloc(N, sizeof(double)), *w_bar = calloc(N, sizeof(double));
  memcpy(r, b, bytes); memcpy(z, b, bytes); memcpy(u, b, bytes); memcpy(v, b, bytes);
  double alpha, beta, ibeta, beta_old, beta1, ceta = 0.0, ceta_oold, ceta_old, ceta_bar;
  double c, cold, s, sold, coold, soold, rho0, rho1, rho2, rho3, dp, np, s_prod;
  int code;
  if (it_init(it, N, b) != 0) { code = it_error_code(it); goto out; }
  orc_copy(N, b, r);
  if (!it->init_guess_null)
    csr_residual(A, x, r);
  else
    memset(x, 0, bytes);
  ceta_oold = 0.0; ceta_old = 0.0;
  c = 1.0; cold = 1.0; s = 0.0; sold = 0.0;
  prec_solve(M, A, r, z);
  dp = orc_dot(N, r, z);
  dp = sqrt(dp); beta = dp; beta1 = beta;
  s_prod = fabs(beta1);
  orc_copy(N, r, v); orc_copy(N, z, u);
  ibeta = 1.0 / beta;
  orc_scal(N, ibeta, v); orc_scal(N, ibeta, u);
  orc_copy(N, u, w_bar);
  np = orc_nrm2(N, b);
  it->nb_iter = 0;
  while (!it_finished(it, np)) {
    if (it->nb_iter != 0) {
      orc_copy(N, v, v_old); orc_copy(N, u, u_old);
      ibeta = 1.0 / beta;
      orc_copy(N, r, v); orc_scal(N, ibeta, v);
      orc_copy(N, z, u); orc_scal(N, ibeta, u);
      orc_copy(N, w_bar, w); orc_scal(N, c, w); orc_axpy(N, s, u, w);
      orc_scal(N, -s, w_bar); orc_axpy(N, c, u, w_bar);
      orc_axpy(N, ceta, w, x);
      ceta_oold = ceta_old;
      ceta_old = ceta;
    }
    csr_mlt(A, u, r);
    alpha = orc_dot(N, u, r);
    prec_solve(M, A, r, z);
    orc_axpy(N, -alpha, v, r);
    orc_axpy(N, -alpha, u, z);
    orc_axpy(N, -beta, v_old, r);
    orc_axpy(N, -beta, u_old, z);
    beta_old = beta;
    dp = orc_dot(N, r, z);
    beta = sqrt(dp);
    coold = cold; cold = c; soold = sold; sold = s;
    rho0 = cold * alpha - coold * sold * beta_old;
    rho1 = sqrt(rho0 * rho0 + beta * beta);
    rho2 = sold * alpha + coold * cold * beta_old;
    rho3 = soold * beta_old;
    c = rho0 / rho1; s = beta / rho1;
    if (it->nb_iter == 0)
      ceta = beta1 / rho1;
    else
      ceta = -(rho2 * ceta_old + rho3 * ceta_oold) / rho1;
    s_prod *= fabs(s);
    if (c == 0.0)
      np = s_prod * 1e16;
    else
      np = s_prod / fabs(c);
    it->nb_iter++;
  }
  if (c == 0.0)
    ceta_bar = ceta * 1e15;
  else
    ceta_bar = ceta / c;
  orc_axpy(N, ceta_bar, w_bar, x);
  code = it_error_code(it);
out:
  free(r); free(z); free(u); free(v); free(w); free(u_old); free(v_old); free(w_bar);
  return code;
}

/* C entry used by tests.  which: 0 Cg, 1 BiCgStab, 2 Gmres, 3 Cgs, 4 TfQmr,
 * 5 MinRes, 6 Gcr, 7 BiCgStabl, 8 QCgs, 9 BiCg, 10 CoCg, 11 Cgne, 12 BiCgcr,
 * 13 Lsqr, 14 QmrSym, 15 Symmlq.
 * precond: 0 identity, 1 Jacobi, 2 SOR (omega, sor_iter, sor_sym).
 * hist/hist_it (may be NULL) receive the relative residual and iteration
 * number of every Finished() test, hist_len their count.
 * Returns Iteration::ErrorCode(); *nb_iter the final iteration count. */
int orc_solve(int which, int m, int nnz, const int* ptr, const int* ind,
              const double* val, int sym, int precond, double omega,
              int sor_iter, int sor_sym, double* x, const double* b, double tol,
              int max_iter, int restart, int init_guess_null, int* nb_iter,
              double* hist, int* hist_it, int hist_cap, int* hist_len) {
  orc_csr A = {m, m, nnz, ptr, ind, val, sym};
  orc_iter it;
  memset(&it, 0, sizeof(it));
  it.tolerance = tol;
  it.max_iter = max_iter;
  it.init_guess_null = init_guess_null;
  it.hist = hist;
  it.hist_it = hist_it;
  it.hist_cap = hist ? hist_cap : 0;
  orc_prec M = {precond, omega, sor_iter, sor_sym, NULL};
  if (precond == 1) {
    M.diag = malloc((size_t)(m > 0 ? m : 1) * sizeof(double));
    for (int i = 0; i < m; i++) M.diag[i] = orc_diag_entry(ptr, ind, val, i);
  }
  int code;
  if (which == 0)
    code = orc_cg_impl(&A, x, b, &M, &it);
  else if (which == 1)
    code = orc_bicgstab_impl(&A, x, b, &M, &it);
  else if (which == 3)
    code = orc_cgs_impl(&A, x, b, &M, &it);
  else if (which == 4)
    code = orc_tfqmr_impl(&A, x, b, &M, &it);
  else if (which == 5)
    code = orc_minres_impl(&A, x, b, &M, &it);
  else if (which == 6)
    code = orc_gcr_impl(&A, x, b, &M, &it, restart);
  else if (which == 7)
    code = orc_bicgstabl_impl(&A, x, b, &M, &it, restart);
  else if (which == 8)
    code = orc_qcgs_impl(&A, x, b, &M, &it);
  else if (which == 9)
    code = orc_bicg_impl(&A, x, b, &M, &it);
  else if (which == 10)
    code = orc_cg_impl(&A, x, b, &M, &it); /* CoCg: Cg's steps in real arithmetic */
  else if (which == 11)
    code = orc_cgne_impl(&A, x, b, &M, &it);
  else if (which == 12)
    code = orc_bicgcr_impl(&A, x, b, &M, &it);
  else if (which == 13)
    code = orc_lsqr_impl(&A, x, b, &it);
  else if (which == 14)
    code = orc_qmrsym_impl(&A, x, b, &M, &it);
  else if (which == 15)
    code = orc_symmlq_impl(&A, x, b, &M, &it);
  else
    code = orc_gmres_impl(&A, x, b, &M, &it, restart);
  free(M.diag);
  if (nb_iter) *nb_iter = it.nb_iter;
  if (hist_len) *hist_len = it.hist_len;
  return code;
}

/* ------------------------------------------------- coordinate -> CSR */

/* Sizes of the matrix ConvertMatrix_from_Coordinates builds
 * (matrix_sparse/Matrix_Conversions.cxx:1300-1313 RowSparse: m = max(largest
 * row - index + 1, A.GetM()), n likewise, GetNormInf of an empty vector
 * being 0; 1410-1421 RowSymSparse: m = n = largest row - index + 1, entries
 * below the diagonal dropped, an empty input returning early).  Returns -1
 * for an index below `index` (ReadCoordinateMatrix's check,
 * Matrix_Sparse.cxx:1912-1921). */
int orc_coo_sizes(int nnz, const int* row, const int* col, int index,
                  int m_min, int n_min, int sym, int* m, int* n,
                  int* nnz_out) {
  long long rmax = 0, cmax = 0;
  int kept = 0;
  for (int i = 0; i < nnz; i++) {
    long long r = (long long)row[i] - index, c = (long long)col[i] - index;
    if (r < 0 || c < 0) return -1;
    if (r > rmax) rmax = r;
    if (c > cmax) cmax = c;
    if (r <= c) kept++;
  }
  if (sym) {
    *m = nnz > 0 ? (int)(rmax + 1) : m_min;
    *n = *m;
    *nnz_out = kept;
  } else {
    *m = (int)(rmax + 1 > m_min ? rmax + 1 : m_min);
    *n = (int)(cmax + 1 > n_min ? cmax + 1 : n_min);
    *nnz_out = nnz;
  }
  return 0;
}

/* Stable merge sort of key[lo..hi) carrying val (equal keys keep their
 * order, as Seldon's MergeSort does: vector/Functions_Arrays.cxx:412-500). */
static void stable_sort_kv(int* key, double* val, int lo, int hi, int* tk,
                           double* tv) {
  if (hi - lo < 2) return;
  int mid = lo + (hi - lo) / 2;
  stable_sort_kv(key, val, lo, mid, tk, tv);
  stable_sort_kv(key, val, mid, hi, tk, tv);
  int a = lo, b = mid, o = lo;
  while (a < mid && b < hi) {
    if (key[b] < key[a]) { tk[o] = key[b]; tv[o++] = val[b++]; }
    else { tk[o] = key[a]; tv[o++] = val[a++]; }
  }
  while (a < mid) { tk[o] = key[a]; tv[o++] = val[a++]; }
  while (b < hi) { tk[o] = key[b]; tv[o++] = val[b++]; }
  memcpy(key + lo, tk + lo, sizeof(int) * (hi - lo));
  memcpy(val + lo, tv + lo, sizeof(double) * (hi - lo));
}

/* The CSR arrays (ptr[m+1], ind/vout[nnz_out] from orc_coo_sizes):
 * Matrix_Conversions.cxx:1315-1333 (RowSparse) and 1423-1466 (RowSymSparse).
 * Steps: drop the lower part (sym), order by row keeping input order among
 * equal rows, count rows into ptr, order each row by column keeping the
 * previous order among equal columns. */
void orc_coo_to_csr(int nnz, const int* row, const int* col,
                    const double* val, int index, int m, int sym, int* ptr,
                    int* ind, double* vout) {
  int* cnt = (int*)calloc((size_t)m + 1, sizeof(int));
  int* fill = (int*)malloc(sizeof(int) * ((size_t)m + 1));
  int* tk = (int*)malloc(sizeof(int) * ((size_t)nnz + 1));
  double* tv = (double*)malloc(sizeof(double) * ((size_t)nnz + 1));
  for (int i = 0; i < nnz; i++) {
    int r = row[i] - index, c = col[i] - index;
    if (sym && r > c) continue;
    cnt[r + 1]++;
  }
  for (int i = 0; i < m; i++) cnt[i + 1] += cnt[i];
  memcpy(ptr, cnt, sizeof(int) * ((size_t)m + 1));
  memcpy(fill, cnt, sizeof(int) * ((size_t)m + 1));
  for (int i = 0; i < nnz; i++) {
    int r = row[i] - index, c = col[i] - index;
    if (sym && r > c) continue;
    ind[fill[r]] = c;
    vout[fill[r]] = val[i];
    fill[r]++;
  }
  for (int i = 0; i < m; i++) stable_sort_kv(ind, vout, ptr[i], ptr[i + 1], tk, tv);
  free(cnt);
  free(fill);
  free(tk);
  free(tv);
}

/* ------------------------------------------------- ILUT preconditioner */

/* SolveLU on Seldon's incomplete factor, with the permutations of
 * IlutPreconditioning::Solve / TransSolve
 * (computation/solver/preconditioner/IlutPreconditioning.cxx:329-374).
 * The factor rows are flat CSR arrays in stored order:
 *   sym = 0: ArrayRowSparse, row i = L part (columns < i), then 1/U(i,i),
 *            then the U part (SparseSolver.cxx:533-611);
 *   sym = 1: ArrayRowSymSparse, row i = 1/D(i) at position 0, then row i of
 *            L^T (SparseSolver.cxx:852-882); the transposed solve is the
 *            same solve.
 * The loops keep Seldon's order of operations, scatter form included. */
static void orc_solve_lu(int n, const int* fp, const int* fi, const double* fv,
                         int sym, int trans, double* x) {
  if (sym) {
    for (int ic = 0; ic < n; ic++)
      for (int k = fp[ic] + 1; k < fp[ic + 1]; k++) x[fi[k]] -= fv[k] * x[ic];
    for (int ic = 0; ic < n; ic++) x[ic] *= fv[fp[ic]];
    for (int ic = n - 1; ic >= 0; ic--) {
      double tmp = x[ic];
      for (int k = fp[ic] + 1; k < fp[ic + 1]; k++) tmp -= fv[k] * x[fi[k]];
      x[ic] = tmp;
    }
    return;
  }
  if (trans) {
    for (int i = 0; i < n; i++) {
      int k = fp[i];
      while (fi[k] < i) k++;
      x[i] *= fv[k];
      for (int q = k + 1; q < fp[i + 1]; q++) x[fi[q]] -= fv[q] * x[i];
    }
    for (int i = n - 1; i >= 0; i--)
      for (int k = fp[i]; fi[k] < i; k++) x[fi[k]] -= fv[k] * x[i];
  } else {
    for (int i = 0; i < n; i++)
      for (int k = fp[i]; fi[k] < i; k++) x[i] -= fv[k] * x[fi[k]];
    for (int i = n - 1; i >= 0; i--) {
      int k = fp[i];
      while (fi[k] < i) k++;
      const double inv_diag = fv[k];
      for (int q = k + 1; q < fp[i + 1]; q++) x[i] -= fv[q] * x[fi[q]];
      x[i] *= inv_diag;
    }
  }
}

void orc_ilut_solve(int n, const int* fp, const int* fi, const double* fv,
                    int sym, const int* perm_row, const int* perm_col,
                    int trans, const double* r, double* z) {
  double* t = (double*)malloc(sizeof(double) * ((size_t)n + 1));
  if (sym || !trans) {
    for (int i = 0; i < n; i++) t[perm_row[i]] = r[i];
    orc_solve_lu(n, fp, fi, fv, sym, 0, t);
    if (sym)
      for (int i = 0; i < n; i++) z[i] = t[perm_row[i]];
    else
      for (int i = 0; i < n; i++) z[perm_col[i]] = t[i];
  } else {
    for (int i = 0; i < n; i++) t[i] = r[perm_col[i]];
    orc_solve_lu(n, fp, fi, fv, 0, 1, t);
    for (int i = 0; i < n; i++) z[i] = t[perm_row[i]];
  }
  free(t);
}
