/* Linear least squares for the oracle build of the reference code.
 *
 * The reference's fit generator, Interpolation::create
 * (elec/Interpolation.cc:276-292), solves min ||A x - b||_2 with LAPACK's
 * DGELS (trans = 'N', one right-hand side, A of m rows >= n columns,
 * column-major with lda = m), first asking for the workspace size
 * (lwork = -1).  LAPACK is not installed here; the reference links the
 * system LAPACK, so no version is pinned.  This file restates the published
 * method DGELS uses for a full-rank overdetermined system, QR factorisation
 * by Householder reflections (Golub and Van Loan, Matrix Computations,
 * 4th ed., Alg. 5.1.1 and 5.2.1, Sec. 5.3.3):
 *   for j = 0 .. n-1: the reflection H_j = I - 2 v v^T / (v^T v) that maps
 *   A[j:m, j] onto beta e_1 (beta = -sign(A_jj) ||A[j:m, j]||), applied to
 *   the remaining columns and to b;
 *   then R x = (Q^T b)[0:n) by back substitution; x overwrites b[0:n).
 * Column norms are accumulated with scaling (as the reference BLAS DNRM2
 * does) so no intermediate overflows.  A zero column norm (rank
 * deficiency) returns info = j + 1, as DGELS reports an exactly singular R.
 *
 * Test infrastructure: only the oracle build links it.
 */
#include <math.h>
#include <stddef.h>

static double scaled_norm(const double* x, int n)
{
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    const double a = fabs(x[i]);
    if (a == 0.0) continue;
    if (scale < a) {
      ssq = 1.0 + ssq * (scale / a) * (scale / a);
      scale = a;
    } else {
      ssq += (a / scale) * (a / scale);
    }
  }
  return scale * sqrt(ssq);
}

int dgels_(char* trans, int* m, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, double* work, int* lwork,
           int* info)
{
  const int M = *m, N = *n, LDA = *lda;
  (void)ldb;
  *info = 0;
  if (*lwork == -1) {          /* workspace query: this method needs none */
    work[0] = 1.0;
    return 0;
  }
  if ((*trans != 'N' && *trans != 'n') || *nrhs != 1 || M < N || N < 0 || LDA < M) {
    *info = -1;
    return 0;
  }
  for (int j = 0; j < N; ++j) {
    double* col = a + (size_t)j * LDA;
    const double norm = scaled_norm(col + j, M - j);
    if (norm == 0.0) {
      *info = j + 1;
      return 0;
    }
    const double alpha = col[j];
    const double beta = alpha >= 0.0 ? -norm : norm;
    /* v = (alpha - beta, col[j+1:m]); v^T v = 2 norm (norm + |alpha|) */
    const double v0 = alpha - beta;
    const double vtv = v0 * v0 + (norm * norm - alpha * alpha);
    for (int k = j + 1; k < N; ++k) {
      double* ck = a + (size_t)k * LDA;
      double s = v0 * ck[j];
      for (int i = j + 1; i < M; ++i) s += col[i] * ck[i];
      const double f = 2.0 * s / vtv;
      ck[j] -= f * v0;
      for (int i = j + 1; i < M; ++i) ck[i] -= f * col[i];
    }
    {
      double s = v0 * b[j];
      for (int i = j + 1; i < M; ++i) s += col[i] * b[i];
      const double f = 2.0 * s / vtv;
      b[j] -= f * v0;
      for (int i = j + 1; i < M; ++i) b[i] -= f * col[i];
    }
    col[j] = beta;               /* R's diagonal */
  }
  for (int i = N - 1; i >= 0; --i) {
    double s = b[i];
    for (int k = i + 1; k < N; ++k) s -= a[(size_t)k * LDA + i] * b[k];
    b[i] = s / a[(size_t)i * LDA + i];
  }
  return 0;
}
