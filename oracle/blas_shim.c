/*
 * Test infrastructure only (oracle build). Not part of the product.
 *
 * Minimal sequential BLAS/LAPACK routines that the reference VCP3D sources
 * link against (src/Makefile:36-37 links -llapack -lblas; no BLAS/LAPACK is
 * installed here). Each routine is written from the routine's documented
 * semantics, not from any BLAS source:
 *
 *   ddot_   x . y, summed sequentially from i = 0 upward
 *           (called by CG_EntropyVarMassMatrix, src/CG_MassMatrix.cpp:60-74)
 *   daxpy_  y := a x + y
 *           (src/CG_MassMatrix.cpp:27-45)
 *   dgetrf_ LU factorisation with partial (row) pivoting, A = P L U
 *   dgetri_ inverse from the dgetrf_ factors
 *           (both called by InverseMatrix, src/StandAloneFunctions.cpp:144-180)
 *   dgtsv_  tridiagonal solve (only referenced by the wall model,
 *           src/WallModel.cpp; never called on the configured cases)
 *
 * The summation order of ddot_ is not pinned by the reference (it links an
 * unversioned system BLAS), so the oracle build fixes it to the plain
 * sequential order above.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

double ddot_(const int *n, const double *x, const int *incx,
             const double *y, const int *incy)
{
  double s = 0.0;
  int ix = (*incx >= 0) ? 0 : (1 - *n) * (*incx);
  int iy = (*incy >= 0) ? 0 : (1 - *n) * (*incy);
  for (int i = 0; i < *n; ++i, ix += *incx, iy += *incy) s += x[ix] * y[iy];
  return s;
}

void daxpy_(const int *n, const double *a, const double *x, const int *incx,
            double *y, const int *incy)
{
  if (*n <= 0 || *a == 0.0) return;
  int ix = (*incx >= 0) ? 0 : (1 - *n) * (*incx);
  int iy = (*incy >= 0) ? 0 : (1 - *n) * (*incy);
  for (int i = 0; i < *n; ++i, ix += *incx, iy += *incy) y[iy] += (*a) * x[ix];
}

/* Column-major LU with partial pivoting. ipiv is 1-based as in LAPACK. */
void dgetrf_(const int *m, const int *n, double *a, const int *lda, int *ipiv,
             int *info)
{
  const int M = *m, N = *n, L = *lda;
  const int mn = M < N ? M : N;
  *info = 0;
  for (int j = 0; j < mn; ++j) {
    int p = j;
    double best = fabs(a[j + j * L]);
    for (int i = j + 1; i < M; ++i) {
      const double v = fabs(a[i + j * L]);
      if (v > best) { best = v; p = i; }
    }
    ipiv[j] = p + 1;
    if (a[p + j * L] == 0.0) { if (*info == 0) *info = j + 1; continue; }
    if (p != j)
      for (int c = 0; c < N; ++c) {
        const double t = a[j + c * L]; a[j + c * L] = a[p + c * L]; a[p + c * L] = t;
      }
    const double inv = 1.0 / a[j + j * L];
    for (int i = j + 1; i < M; ++i) a[i + j * L] *= inv;
    for (int c = j + 1; c < N; ++c) {
      const double f = a[j + c * L];
      for (int i = j + 1; i < M; ++i) a[i + c * L] -= a[i + j * L] * f;
    }
  }
}

/* Inverse of A from its dgetrf_ factors: solve A X = I column by column,
 * then write X back into a. */
void dgetri_(const int *n, double *a, const int *lda, const int *ipiv,
             double *work, const int *lwork, int *info)
{
  const int N = *n, L = *lda;
  (void)work; (void)lwork;
  *info = 0;
  for (int i = 0; i < N; ++i)
    if (a[i + i * L] == 0.0) { *info = i + 1; return; }
  double *x = (double *)malloc(sizeof(double) * (size_t)N * (size_t)N);
  for (int c = 0; c < N; ++c) {
    double *col = x + (size_t)c * N;
    for (int i = 0; i < N; ++i) col[i] = (i == c) ? 1.0 : 0.0;
    for (int i = 0; i < N; ++i) {           /* apply the row interchanges */
      const int p = ipiv[i] - 1;
      if (p != i) { const double t = col[i]; col[i] = col[p]; col[p] = t; }
    }
    for (int i = 0; i < N; ++i)             /* unit lower triangular solve */
      for (int k = 0; k < i; ++k) col[i] -= a[i + k * L] * col[k];
    for (int i = N - 1; i >= 0; --i) {      /* upper triangular solve */
      for (int k = i + 1; k < N; ++k) col[i] -= a[i + k * L] * col[k];
      col[i] /= a[i + i * L];
    }
  }
  for (int c = 0; c < N; ++c)
    for (int i = 0; i < N; ++i) a[i + c * L] = x[i + (size_t)c * N];
  free(x);
}

/* Tridiagonal solve by Gaussian elimination without pivoting.
 * dl: sub-diagonal (n-1), d: diagonal (n), du: super-diagonal (n-1). */
void dgtsv_(const int *n, const int *nrhs, double *dl, double *d, double *du,
            double *b, const int *ldb, int *info)
{
  const int N = *n, R = *nrhs, L = *ldb;
  *info = 0;
  for (int i = 1; i < N; ++i) {
    if (d[i - 1] == 0.0) { *info = i; return; }
    const double f = dl[i - 1] / d[i - 1];
    d[i] -= f * du[i - 1];
    for (int r = 0; r < R; ++r) b[i + r * L] -= f * b[i - 1 + r * L];
  }
  if (d[N - 1] == 0.0) { *info = N; return; }
  for (int r = 0; r < R; ++r) {
    b[N - 1 + r * L] /= d[N - 1];
    for (int i = N - 2; i >= 0; --i)
      b[i + r * L] = (b[i + r * L] - du[i] * b[i + 1 + r * L]) / d[i];
  }
}
