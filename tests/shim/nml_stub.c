/* nml_stub.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The three nml allocation routines the eigensolve_lanczos drop-in calls
 * (nml_dv_new, nml_dcv_new, nml_dcm_new), written on the interface the
 * reference's nml headers declare (a vector keeps its length in the word
 * before its first element; a matrix is an array of row pointers into one
 * block).  In the NEMO-3D build these come from its nml library, whose
 * sources are generated by a template tool; the tests link these instead.
 */
#include <stdlib.h>

#include "nml_dcmatrix.h"
#include "nml_dcvector.h"
#include "nml_dvector.h"

static void *with_length(size_t n, size_t elem) {
  char *raw = (char *)calloc(1, 16 + elem * (n > 0 ? n : 1));
  if (!raw) return NULL;
  *(nml_extent *)(raw + 16 - sizeof(nml_extent)) = (nml_extent)n;
  return raw + 16;
}

nml_dvector *nml_dv_new(nml_extent n) { return (nml_dvector *)with_length(n, sizeof(nml_dvector)); }

nml_dcvector *nml_dcv_new(nml_extent n) {
  return (nml_dcvector *)with_length(n, sizeof(nml_dcvector));
}

nml_dcmatrix *nml_dcm_new(nml_extent m, nml_extent n) {
  nml_dcmatrix *rows = (nml_dcmatrix *)with_length(m, sizeof(nml_dcmatrix));
  nml_dcscalar *data = (nml_dcscalar *)with_length(m * n, sizeof(nml_dcscalar));
  nml_extent i;
  if (!rows || !data) return NULL;
  for (i = 0; i < m; ++i) rows[i] = data + i * n;
  return rows;
}
