/*
 * eigensolve_lanczos_tbgpu.c -- the reference's Lanczos driver entry point
 * running on libtbgpu.so.
 *
 * Compiled inside the NEMO-3D tree in place of the eigensolve_lanczos of
 * eigen/src/lanczos.c:1823-2089, against the tree's own declaration
 * (eigen/include/lanczos.h:365-391) and nml allocation routines, it keeps
 * the callers (lanczos_driver, nemo3d/src/base/eigsys3d_par.c:361-390)
 * unchanged and runs the solve on the GPU:
 *
 *   argument[0]   the libtbgpu context (tbgpu_ctx *), in the slot where the
 *                 reference's driver passes its qd_struct
 *                 (eigsys3d_par.c:280); the context applies H itself, so the
 *                 matmul pointer is not called (tbgpu_matvect_mult is that
 *                 product behind the same signature);
 *   start vector  r_0, or r_n when r_0 is NULL (the reference's first pass
 *                 starts from r_n and reruns from r_0);
 *   *pValue       allocated with nml_dv_new(imax), the eigenvalues found in
 *                 ascending order, as the reference returns them;
 *   fn_tridiag,   the state the reference saves (saveTridiagonalMatrix,
 *   fn_eigval     saveEigenvalues, lanczos.c:1692-1713, 1780-1792) in its
 *                 binary formats; restoreState reads them back (keeping
 *                 iterations - 200 of the stored matrix, as
 *                 restoreTridiagonalMatrix does) and only the eigenvectors
 *                 are computed;
 *   r_0 != NULL   *pCValue = nml_dcv_new(n) holds (value, 0) and
 *                 *pCVector = nml_dcm_new(n, length) the eigenvectors, from a
 *                 rerun of the recurrence on the saved matrix (every value's
 *                 Ritz vector on the whole matrix);
 *   r_n, q_n, q_n1 are not written (the recurrence's vectors stay on the
 *                 GPU); fn_trace is not written; verbose prints the
 *                 eigenvalues as the reference does.
 *
 * Errors: the reference exits the process; this returns the negative libtbgpu
 * status (tbgpu_error_string describes it).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lanczos.h"
#include "tbgpu.h"

/* eigenvectors of the n values from the tridiagonal matrix (alpha, beta) of
 * `iterations` steps into the rows of M (nml_dcm_new(n, length)) */
static int vectors_into(tbgpu_ctx *ctx, int iterations, const double *alpha,
                        const double *beta, int n, const double *values,
                        const nml_dcscalar *start, nml_dcmatrix *M, size_t length) {
  int contiguous = 1, k, rc;
  tbgpu_dcomplex *buf;
  for (k = 1; k < n; ++k)
    if (M[k] != M[0] + (size_t)k * length) contiguous = 0;
  buf = contiguous ? (tbgpu_dcomplex *)M[0]
                   : (tbgpu_dcomplex *)malloc(sizeof(tbgpu_dcomplex) * length * (size_t)n);
  if (!buf) return TBGPU_E_NOMEM;
  rc = tbgpu_eigenvectors_from_tridiagonal(ctx, iterations, alpha, beta, n, values,
                                           (const tbgpu_dcomplex *)start, buf, n);
  if (!contiguous) {
    if (rc > 0)
      for (k = 0; k < n; ++k)
        memcpy(M[k], buf + (size_t)k * length, sizeof(tbgpu_dcomplex) * length);
    free(buf);
  }
  return rc < 0 ? rc : 0;
}

int eigensolve_lanczos(nml_dvector **pValue, int ConvCheckStartIter, int ConvCheckSkipRate,
                       int imax, int requested1, int requested2, nml_extent length,
                       int *argument[], nml_dscalar emin1, nml_dscalar emax1,
                       nml_dscalar emin2, nml_dscalar emax2, nml_dscalar tolerance,
                       int verbose, const char *fn_trace, const char *fn_tridiag,
                       const char *fn_eigval, nml_dcvector *r_n, const nml_dcvector *r_0,
                       nml_dcvector *q_n, nml_dcvector *q_n1, nml_dcvector **pCValue,
                       nml_dcmatrix **pCVector,
                       void (*matmul)(const int **, nml_dcscalar *, const nml_dcscalar *),
                       int restoreState) {
  tbgpu_ctx *ctx = argument ? (tbgpu_ctx *)argument[0] : NULL;
  const nml_dcscalar *start = r_0 ? r_0 : r_n;
  double *alpha = NULL, *beta = NULL;
  int eigenvalues = 0, iterations = 0, rc = 0, k;
  (void)fn_trace;
  (void)q_n;
  (void)q_n1;
  (void)matmul;
  if (!ctx || !pValue || !start || (long)length != tbgpu_dimension(ctx)) return TBGPU_E_ARG;

  if (restoreState) {
    int procs = 0;
    iterations = tbgpu_read_tridiagonal_file(fn_tridiag, 0, NULL, NULL, &procs);
    if (iterations < 0) return iterations;
    eigenvalues = tbgpu_read_eigenvalue_file(fn_eigval, 0, NULL);
    if (eigenvalues < 0) return eigenvalues;
    alpha = (double *)malloc(sizeof(double) * (size_t)iterations);
    beta = (double *)malloc(sizeof(double) * (size_t)iterations);
    *pValue = nml_dv_new((nml_extent)(eigenvalues > 0 ? eigenvalues : 1));
    if (!alpha || !beta || !*pValue) {
      rc = TBGPU_E_NOMEM;
    } else {
      tbgpu_read_tridiagonal_file(fn_tridiag, iterations, alpha, beta, NULL);
      tbgpu_read_eigenvalue_file(fn_eigval, eigenvalues, *pValue);
      if (procs != 1 && verbose)
        printf("ACHTUNG!!!:  you are running on a different number of processors\n"
               "from the run that generated your tridiagonal matrix\n");
    }
  } else {
    int *conv = (int *)malloc(sizeof(int) * (size_t)imax);
    *pValue = nml_dv_new((nml_extent)imax);
    if (!conv || !*pValue) {
      free(conv);
      return TBGPU_E_NOMEM;
    }
    eigenvalues = tbgpu_eigensolve_lanczos(ctx, ConvCheckStartIter, ConvCheckSkipRate, imax,
                                           requested1, requested2, emin1, emax1, emin2, emax2,
                                           tolerance, (const tbgpu_dcomplex *)start, *pValue,
                                           conv, &iterations, NULL, 0);
    if (eigenvalues < 0) {
      free(conv);
      return eigenvalues;
    }
    if (verbose)
      for (k = 0; k < eigenvalues; ++k)
        printf("Eigenvalue: %.8e  in %d iterations\n", (*pValue)[k], conv[k]);
    free(conv);
    alpha = (double *)malloc(sizeof(double) * (size_t)(iterations + 1));
    beta = (double *)malloc(sizeof(double) * (size_t)(iterations + 1));
    if (!alpha || !beta) {
      rc = TBGPU_E_NOMEM;
    } else {
      iterations = tbgpu_get_tridiagonal(ctx, alpha, beta, iterations + 1);
      /* save state = {tridiagonal matrix, eigenvalues} */
      if (fn_tridiag) tbgpu_write_tridiagonal_file(fn_tridiag, alpha, beta, iterations, 1);
      if (fn_eigval) tbgpu_write_eigenvalue_file(fn_eigval, *pValue, eigenvalues);
    }
  }

  if (!rc && r_0 && eigenvalues > 0) {
    *pCValue = nml_dcv_new((nml_extent)eigenvalues);
    *pCVector = nml_dcm_new((nml_extent)eigenvalues, length);
    if (!*pCValue || !*pCVector) {
      rc = TBGPU_E_NOMEM;
    } else {
      for (k = 0; k < eigenvalues; ++k) {
        (*pCValue)[k].r = (*pValue)[k];
        (*pCValue)[k].i = 0.0;
      }
      rc = vectors_into(ctx, iterations, alpha, beta, eigenvalues, *pValue, r_0, *pCVector,
                        (size_t)length);
    }
  }
  free(alpha);
  free(beta);
  return rc < 0 ? rc : eigenvalues;
}
