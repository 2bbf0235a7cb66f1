/*
 * CPU restatement of the reference's solve-phase kernels — TEST
 * INFRASTRUCTURE (the oracle).  Only the tests, the smoke check and the CPU
 * baseline of bench.py load this library; the product never does.
 *
 * Every function repeats the loop order of the reference routine it names, so
 * that on the same inputs the results agree with the reference to the last
 * bit (the parity tests check this against outputs of the reference itself).
 * Citations are to ParGeMSLR (Hitenze/pargemslr) source files.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* y = alpha*A*x + beta*y for a CSR matrix, trans 'N'
 * (CsrMatrixPMatVecHostTemplate, SRC/matrices/matrixops.cpp:5139-5330):
 * y is first scaled by beta (set to zero when beta == 0), then every row sum
 * r = sum_j a_ij x_j is accumulated in CSR order and added as y_i += alpha*r
 * (y_i += r when alpha == 1). */
void oracle_csr_matvec(int nrows, const int *ia, const int *ja, const double *aa, double alpha,
                       const double *x, double beta, double *y)
{
   int i, j;
   if (beta != 1.0)
   {
      if (beta != 0.0)
         for (i = 0; i < nrows; i++) y[i] *= beta;
      else
         for (i = 0; i < nrows; i++) y[i] = 0.0;
   }
   if (alpha == 0.0) return;
   for (i = 0; i < nrows; i++)
   {
      double r = 0.0;
      for (j = ia[i]; j < ia[i + 1]; j++) r += aa[j] * x[ja[j]];
      if (alpha != 1.0)
         y[i] += alpha * r;
      else
         y[i] += r;
   }
}

/* ILU solve without internal permutation (IluClass::SolveHost,
 * SRC/preconditioners/ilu.cpp:3677-3790): x = rhs; forward sweep with the
 * strictly lower L (unit diagonal); backward sweep with the strictly upper U
 * followed by x_i *= D_i, D holding the INVERSE diagonal. */
void oracle_ilu_solve(int n, const int *li, const int *lj, const double *la, const int *ui, const int *uj,
                      const double *ua, const double *d, const double *rhs, double *x)
{
   int i, j;
   for (i = 0; i < n; i++) x[i] = rhs[i];
   for (i = 0; i < n; i++)
      for (j = li[i]; j < li[i + 1]; j++) x[i] -= la[j] * x[lj[j]];
   for (i = n - 1; i >= 0; i--)
   {
      for (j = ui[i]; j < ui[i + 1]; j++) x[i] -= ua[j] * x[uj[j]];
      x[i] *= d[i];
   }
}

/* Level sets of a triangular factor (IluClass::BuildLevels,
 * SRC/preconditioners/ilu.cpp:832-1062): level(i) = 1 + max level of the
 * entries of row i (lower: sweep from row 0, upper: from row n-1); rows are
 * listed by level, then by index.  level_ptr needs n+1 entries; returns the
 * number of levels, or -1 if the factor is not strictly triangular. */
int oracle_build_levels(char uplo, int n, const int *ia, const int *ja, int *level_ptr, int *order)
{
   int *lev = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
   int t, i, j, l, max_level = 0, nlev;
   for (i = 0; i < n; i++) lev[i] = -1;
   for (t = 0; t < n; t++)
   {
      i = uplo == 'U' ? n - 1 - t : t;
      l = -1;
      for (j = ia[i]; j < ia[i + 1]; j++)
      {
         int c = ja[j];
         if (uplo == 'U' ? c <= i : c >= i)
         {
            free(lev);
            return -1;
         }
         if (lev[c] > l) l = lev[c];
      }
      lev[i] = l + 1;
      if (lev[i] > max_level) max_level = lev[i];
   }
   nlev = n > 0 ? max_level + 1 : 0;
   for (l = 0; l <= nlev; l++) level_ptr[l] = 0;
   for (i = 0; i < n; i++) level_ptr[lev[i] + 1]++;
   for (l = 0; l < nlev; l++) level_ptr[l + 1] += level_ptr[l];
   {
      int *pos = (int *)malloc(sizeof(int) * (nlev > 0 ? nlev : 1));
      for (l = 0; l < nlev; l++) pos[l] = level_ptr[l];
      for (i = 0; i < n; i++) order[pos[lev[i]]++] = i;
      free(pos);
   }
   free(lev);
   return nlev;
}

/* y = A^T x for a column-major dense A (m x k, leading dimension m), the 'C'
 * branch with alpha = 1, beta = 0 of DenseMatrixPMatVecTemplate
 * (SRC/matrices/matrixops.cpp:101-330): y_c accumulates a_jc x_j over j. */
void oracle_dense_matvec_t(int m, int k, const double *a, const double *x, double *y)
{
   int c, j;
   for (c = 0; c < k; c++) y[c] = 0.0;
   for (c = 0; c < k; c++)
   {
      const double *col = a + (size_t)c * m;
      for (j = 0; j < m; j++) y[c] += col[j] * x[j];
   }
}

/* y = A x for a column-major dense A, the 'N' branch with alpha = 1,
 * beta = 0: column by column, y_j += a_jc x_c. */
void oracle_dense_matvec_n(int m, int k, const double *a, const double *x, double *y)
{
   int c, j;
   for (j = 0; j < m; j++) y[j] = 0.0;
   for (c = 0; c < k; c++)
   {
      const double *col = a + (size_t)c * m;
      for (j = 0; j < m; j++) y[j] += col[j] * x[c];
   }
}

/* dot, axpy and scale of VectorPDotTemplate / VectorPAxpyTemplate /
 * VectorPScaleTemplate (SRC/vectors/vectorops.cpp), single-threaded. */
double oracle_dot(int n, const double *x, const double *y)
{
   double t = 0.0;
   int i;
   for (i = 0; i < n; i++) t += x[i] * y[i];
   return t;
}

void oracle_axpy(int n, double a, const double *x, double *y)
{
   int i;
   if (a == 1.0)
      for (i = 0; i < n; i++) y[i] += x[i];
   else
      for (i = 0; i < n; i++) y[i] += a * x[i];
}

void oracle_scale(int n, double a, double *x)
{
   int i;
   for (i = 0; i < n; i++) x[i] *= a;
}

/* Modified Gram-Schmidt without re-orthogonalisation as FlexGmres calls it
 * (PargemslrMgs with tol_reorth = -1, SRC/matrices/matrixops.cpp:10728-10806):
 * column k+1 of V (leading dimension n) against columns 0..k; H is
 * column-major with leading dimension ldh; w is scaled by 1/||w||. */
void oracle_mgs(int n, double *V, int k, double *H, int ldh)
{
   double *w = V + (size_t)(k + 1) * n;
   double t;
   int i;
   for (i = 0; i <= k; i++)
   {
      const double *v = V + (size_t)i * n;
      t = oracle_dot(n, v, w);
      H[i + (size_t)k * ldh] = t;
      oracle_axpy(n, -t, v, w);
   }
   t = sqrt(fabs(oracle_dot(n, w, w)));
   H[(k + 1) + (size_t)k * ldh] = t;
   oracle_scale(n, 1.0 / t, w);
}
