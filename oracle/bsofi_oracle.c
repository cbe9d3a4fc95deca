/*
 * bsofi_oracle.c -- CPU restatement of the reference BSOF/I algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it.  The product library (bsofi_b200/libbsofi_b200.so) never links,
 * loads or calls it.
 *
 * What it restates (reference file:line):
 *   oracle_bsof        src/bsofi_cpu.c:86-118   (lapackXbsof)
 *   oracle_bstri       src/bsofi_cpu.c:146-177  (lapackXbstri)
 *   oracle_bsoi        src/bsofi_cpu.c:211-248  (lapackXbsoi_ormqr, the
 *                                                route of hybridXbsoiH,
 *                                                src/bsofi_callback.c:156)
 *   oracle_cpyzero_l   src/bsofi_lapack.c:260-281 (lapackXcpyzero 'L')
 * The reference calls LAPACK/BLAS (dgeqrf, dormqr, dtrtri, dtrmm, dgemm) through
 * src/bsofi_lapack.c:130-250.  LAPACK is an unpinned third-party dependency of
 * the reference; its published unblocked algorithms are restated here:
 *   geqr2/larfg   LAPACK dgeqr2 + dlarfg (beta = -sign(alpha)*||(alpha,x)||,
 *                 tau = (beta-alpha)/beta, v = x/(alpha-beta); tau = 0 and
 *                 H = I when x == 0)
 *   orm2r         LAPACK dorm2r (left/right, transposed)
 *   trti2         LAPACK dtrti2 (upper, non-unit), with dtrtri's exact-zero
 *                 diagonal check (info = i)
 *   trmm / gemm   BLAS dtrmm / dgemm definitions
 * Differences from LAPACK: no scaled 2-norm (dnrm2) and no dlarfg rescaling
 * loop for |beta| < safmin; vectors are summed in plain order.  Results agree
 * with the compiled reference to rounding (the tests pin this).
 *
 * Layout: column-major, leading dimension lda >= n*L, N = n*L.
 */
#include <math.h>
#include <stddef.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(j) * (size_t)(ld) + (size_t)(i))

/* dlarfg: on exit *alpha = beta, x = v(2:m), *tau set. */
static void larfg(int m, double *alpha, double *x, double *tau)
{
  double xnorm2 = 0.0, beta;
  int i;
  if (m <= 1) { *tau = 0.0; return; }
  for (i = 0; i < m - 1; i++) xnorm2 += x[i] * x[i];
  if (xnorm2 == 0.0) { *tau = 0.0; return; }
  beta = -copysign(sqrt((*alpha) * (*alpha) + xnorm2), *alpha);
  *tau = (beta - *alpha) / beta;
  {
    double scal = 1.0 / (*alpha - beta);
    for (i = 0; i < m - 1; i++) x[i] *= scal;
  }
  *alpha = beta;
}

/* Apply H = I - tau v v^T from the left to C (m x nc); v(0) = 1 implicit. */
static void larf_left(int m, int nc, const double *v, double tau,
                      double *C, int ldc)
{
  int i, j;
  if (tau == 0.0) return;
  for (j = 0; j < nc; j++) {
    double *c = C + IDX(0, j, ldc);
    double w = c[0];
    for (i = 1; i < m; i++) w += v[i] * c[i];
    w *= tau;
    c[0] -= w;
    for (i = 1; i < m; i++) c[i] -= w * v[i];
  }
}

/* Apply H = I - tau v v^T from the right to C (mr x m); v(0) = 1 implicit. */
static void larf_right(int mr, int m, const double *v, double tau,
                       double *C, int ldc)
{
  int i, j;
  if (tau == 0.0) return;
  for (i = 0; i < mr; i++) {
    double w = C[IDX(i, 0, ldc)];
    for (j = 1; j < m; j++) w += C[IDX(i, j, ldc)] * v[j];
    w *= tau;
    C[IDX(i, 0, ldc)] -= w;
    for (j = 1; j < m; j++) C[IDX(i, j, ldc)] -= w * v[j];
  }
}

/* dgeqr2: Householder QR of A (m x n), reflectors below the diagonal. */
void oracle_geqr2(int m, int n, double *A, int lda, double *tau)
{
  int k = m < n ? m : n, i;
  double v[4096];
  for (i = 0; i < k; i++) {
    double *a = A + IDX(i, i, lda);
    larfg(m - i, a, a + 1, &tau[i]);
    if (i < n - 1) {
      int r;
      v[0] = 1.0;
      for (r = 1; r < m - i; r++) v[r] = a[r];
      larf_left(m - i, n - i - 1, v, tau[i], A + IDX(i, i + 1, lda), lda);
    }
  }
}

/* dorm2r SIDE='L', TRANS='T': C (m x nc) <- Q^T C, Q = H(0)...H(k-1). */
void oracle_orm2r_lt(int m, int nc, int k, const double *V, int ldv,
                     const double *tau, double *C, int ldc)
{
  double v[4096];
  int i, r;
  for (i = 0; i < k; i++) {
    v[0] = 1.0;
    for (r = 1; r < m - i; r++) v[r] = V[IDX(i + r, i, ldv)];
    larf_left(m - i, nc, v, tau[i], C + IDX(i, 0, ldc), ldc);
  }
}

/* dorm2r SIDE='R', TRANS='T': C (mr x m) <- C Q^T, Q = H(0)...H(k-1). */
void oracle_orm2r_rt(int mr, int m, int k, const double *V, int ldv,
                     const double *tau, double *C, int ldc)
{
  double v[4096];
  int i, r;
  for (i = k - 1; i >= 0; i--) {
    v[0] = 1.0;
    for (r = 1; r < m - i; r++) v[r] = V[IDX(i + r, i, ldv)];
    larf_right(mr, m - i, v, tau[i], C + IDX(0, i, ldc), ldc);
  }
}

/* dtrtri UPLO='U', DIAG='N' (unblocked dtrti2 order).  Returns info. */
int oracle_trtri_u(int n, double *A, int lda)
{
  int i, j, k;
  for (i = 0; i < n; i++)
    if (A[IDX(i, i, lda)] == 0.0) return i + 1;
  for (j = 0; j < n; j++) {
    double ajj;
    A[IDX(j, j, lda)] = 1.0 / A[IDX(j, j, lda)];
    ajj = -A[IDX(j, j, lda)];
    /* x = A(0:j, j) <- triu(A(0:j,0:j)) * x  (dtrmv upper, no-trans) */
    for (k = 0; k < j; k++) {
      double t = A[IDX(k, j, lda)];
      for (i = 0; i < k; i++) A[IDX(i, j, lda)] += t * A[IDX(i, k, lda)];
      A[IDX(k, j, lda)] = t * A[IDX(k, k, lda)];
    }
    for (i = 0; i < j; i++) A[IDX(i, j, lda)] *= ajj;
  }
  return 0;
}

/* dtrmm SIDE='R', UPLO='U', TRANSA='N', DIAG='N': B (m x n) <- alpha B U. */
static void trmm_run(int m, int n, double alpha, const double *U, int ldu,
                     double *B, int ldb)
{
  int i, j, k;
  for (j = n - 1; j >= 0; j--) {
    double t = alpha * U[IDX(j, j, ldu)];
    for (i = 0; i < m; i++) B[IDX(i, j, ldb)] *= t;
    for (k = 0; k < j; k++) {
      double u = alpha * U[IDX(k, j, ldu)];
      if (u != 0.0)
        for (i = 0; i < m; i++) B[IDX(i, j, ldb)] += u * B[IDX(i, k, ldb)];
    }
  }
}

/* dtrmm SIDE='L', UPLO='U', TRANSA='N', DIAG='N': B (m x n) <- alpha U B. */
static void trmm_lun(int m, int n, double alpha, const double *U, int ldu,
                     double *B, int ldb)
{
  int i, j, k;
  for (j = 0; j < n; j++) {
    for (k = 0; k < m; k++) {
      double t = alpha * B[IDX(k, j, ldb)];
      if (t != 0.0) {
        for (i = 0; i < k; i++) B[IDX(i, j, ldb)] += t * U[IDX(i, k, ldu)];
        t *= U[IDX(k, k, ldu)];
      }
      B[IDX(k, j, ldb)] = t;
    }
  }
}

/* dgemm 'N','N': C (m x n) <- alpha A B + beta C, K inner. */
static void gemm_nn(int m, int n, int K, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta,
                    double *C, int ldc)
{
  int i, j, k;
  for (j = 0; j < n; j++) {
    if (beta != 1.0)
      for (i = 0; i < m; i++) C[IDX(i, j, ldc)] *= beta;
    for (k = 0; k < K; k++) {
      double t = alpha * B[IDX(k, j, ldb)];
      if (t != 0.0)
        for (i = 0; i < m; i++) C[IDX(i, j, ldc)] += t * A[IDX(i, k, lda)];
    }
  }
}

/* lapackXcpyzero('L', m, n, A, lda, B, ldb), src/bsofi_lapack.c:260-281. */
void oracle_cpyzero_l(int m, int n, double *A, int lda, double *B, int ldb)
{
  int i, j;
  for (j = 0; j < n; j++)
    for (i = j + 1; i < m; i++) {
      B[IDX(i, j, ldb)] = A[IDX(i, j, lda)];
      A[IDX(i, j, lda)] = 0.0;
    }
}

#define BLK(i, j) (A + IDX((size_t)(i) * n, (size_t)(j) * n, lda))

/* lapackXbsof, src/bsofi_cpu.c:86-118. */
int oracle_bsof(int n, int L, double *A, int lda, double *tau)
{
  int i;
  double *t = tau;
  for (i = 0; i < L - 2; i++) {
    oracle_geqr2(2 * n, n, BLK(i, i), lda, t);
    oracle_orm2r_lt(2 * n, n, n, BLK(i, i), lda, t, BLK(i, i + 1), lda);
    oracle_orm2r_lt(2 * n, n, n, BLK(i, i), lda, t, BLK(i, L - 1), lda);
    t += n;
  }
  oracle_geqr2(2 * n, 2 * n, BLK(L - 2, L - 2), lda, t);
  return 0;
}

/* lapackXbstri, src/bsofi_cpu.c:146-177.  Like the reference, info is the
 * value returned by the last triangular inversion performed. */
int oracle_bstri(int n, int L, double *A, int lda)
{
  int i, info = 0;
  if (L <= 2) return oracle_trtri_u(n * L, BLK(0, 0), lda);
  info = oracle_trtri_u(3 * n, BLK(L - 3, L - 3), lda);
  if (L > 3) {
    trmm_run(n * (L - 3), n, 1.0, BLK(L - 1, L - 1), lda, BLK(0, L - 1), lda);
    for (i = L - 4; i >= 0; i--) {
      info = oracle_trtri_u(n, BLK(i, i), lda);
      trmm_lun(n, n, -1.0, BLK(i, i), lda, BLK(i, L - 1), lda);
      trmm_lun(n, n, -1.0, BLK(i, i), lda, BLK(i, i + 1), lda);
      gemm_nn(n, n * (L - i - 2), n, 1.0, BLK(i, i + 1), lda,
              BLK(i + 1, i + 2), lda, 1.0, BLK(i, i + 2), lda);
      trmm_run(n, n, 1.0, BLK(i + 1, i + 1), lda, BLK(i, i + 1), lda);
    }
  }
  return info;
}

/* lapackXbsoi_ormqr, src/bsofi_cpu.c:211-248.  work >= 4 n^2 doubles. */
int oracle_bsoi(int n, int L, double *A, int lda, const double *tau,
                double *work)
{
  int N = n * L, i, ldq = 2 * n;
  const double *t = tau + (size_t)(L - 2) * n;
  double *Q = work;
  memset(Q, 0, sizeof(double) * 4 * (size_t)n * n);
  oracle_cpyzero_l(2 * n, 2 * n, BLK(L - 2, L - 2), lda, Q, ldq);
  oracle_orm2r_rt(N, 2 * n, 2 * n, Q, ldq, t, BLK(0, L - 2), lda);
  for (i = L - 3; i >= 0; i--) {
    t -= n;
    oracle_cpyzero_l(2 * n, n, BLK(i, i), lda, Q, ldq);
    oracle_orm2r_rt(N, 2 * n, n, Q, ldq, t, BLK(0, i), lda);
  }
  return 0;
}

/* Full BSOF -> BSTRI -> BSOI, the route of hybridXbsoftriH + hybridXbsoiH
 * without CUDA (src/bsofi_callback.c:130-157). */
int oracle_bsofi(int n, int L, double *A, int lda, double *tau, double *work)
{
  int info;
  oracle_bsof(n, L, A, lda, tau);
  info = oracle_bstri(n, L, A, lda);
  if (info != 0) return info;
  return oracle_bsoi(n, L, A, lda, tau, work);
}
