// ref_lanczos_driver.cc -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
//
// Links the reference's own Lanczos driver (eigen/src/lanczos.c, compiled
// where it lies by oracle/build_ref.sh, with the reference's fake MPI layer
// eigen/src/mpi_fake.c) into oracle/_ref/libref_lanczos.so, so that the CPU
// baseline of the benchmark and the tests can run the reference's
// eigenvaluesLanczos -- its recurrence, convergence windows, dstebz
// bisection and ghost handling -- on a real Hamiltonian.  The H*x it calls
// through its matmul pointer is the oracle's restatement of the reference's
// stored product (orc_hx, oracle/tb_oracle.c): the reference's own
// Hmult_stored needs its XML-driven geometry set-up and is not built.
// Nothing of the product uses this file.
//
// What the link needs besides those sources:
//  * the nml routines lanczos.c calls, written here on the interface the
//    reference's nml headers declare (a vector keeps its length in the word
//    before its first element; tridiagonal bands are three vectors reached
//    through a pointer to the middle one, T[-1], T[0], T[+1]); the nml
//    library's own sources are generated by a template tool;
//  * LAPACK's dstebz, forwarded to the dstebz that scipy's bundled OpenBLAS
//    exports (the reference builds its vendored Fortran LAPACK, and no
//    Fortran compiler is present here);
//  * the MPI rank globals of a serial run.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "lanczos.h"

extern "C" {
#include "tb_oracle.h"
}

// ---------------------------------------------------------------- serial MPI
int mpi_n3d_id = 0;
int mpi_n3d_masterid = 0;
int mpi_n3d_numprocs = 1;

// ---------------------------------------------------------------- nml
namespace {
void *with_length(size_t n, size_t elem) {
  char *raw = static_cast<char *>(calloc(1, 16 + elem * (n > 0 ? n : 1)));
  if (!raw) {
    fprintf(stderr, "ref_lanczos_driver: out of memory\n");
    exit(2);
  }
  *reinterpret_cast<nml_extent *>(raw + 16 - sizeof(nml_extent)) = n;
  return raw + 16;
}
template <typename T>
nml_extent length_of(const T *p) {
  return *reinterpret_cast<const nml_extent *>(reinterpret_cast<const char *>(p) -
                                               sizeof(nml_extent));
}
void release(const void *p) {
  if (p) free(const_cast<char *>(static_cast<const char *>(p)) - 16);
}
}  // namespace

nml_dvector *nml_dv_new(nml_extent n) { return static_cast<nml_dvector *>(with_length(n, sizeof(double))); }
void nml_dv_delete(nml_dvector *p) { release(p); }
nml_extent nml_dv_extent(const nml_dvector *p) { return length_of(p); }
nml_dvector *nml_dv_clone(const nml_dvector *p) {
  const nml_extent n = length_of(p);
  nml_dvector *q = nml_dv_new(n);
  memcpy(q, p, sizeof(double) * n);
  return q;
}
nml_dvector *nml_dv_ssub(nml_dvector *p, nml_dscalar x) {
  const nml_extent n = length_of(p);
  for (nml_extent i = 0; i < n; ++i) p[i] -= x;
  return p;
}
nml_ivector *nml_iv_new(nml_extent n) { return static_cast<nml_ivector *>(with_length(n, sizeof(int))); }
void nml_iv_delete(nml_ivector *p) { release(p); }
nml_dcvector *nml_dcv_new(nml_extent n) {
  return static_cast<nml_dcvector *>(with_length(n, sizeof(nml_dcvector)));
}
nml_dscalar nml_dcv_ssqr(const nml_dcvector *p) {
  const nml_extent n = length_of(p);
  nml_dscalar s = 0.0;
  for (nml_extent i = 0; i < n; ++i) s += p[i].r * p[i].r + p[i].i * p[i].i;
  return s;
}
nml_dcscalar nml_dcmplx(nml_double r, nml_double i) {
  nml_dcscalar z;
  z.r = r;
  z.i = i;
  return z;
}
nml_dmatrix *nml_dm_new(nml_extent m, nml_extent n) {
  nml_dmatrix *rows = static_cast<nml_dmatrix *>(with_length(m, sizeof(nml_dmatrix)));
  double *data = static_cast<double *>(with_length(m * n, sizeof(double)));
  for (nml_extent i = 0; i < m; ++i) rows[i] = data + i * n;
  return rows;
}
void nml_dm_delete(nml_dmatrix *p) {
  if (!p) return;
  release(p[0]);
  release(p);
}
nml_dcmatrix *nml_dcm_new(nml_extent m, nml_extent n) {
  nml_dcmatrix *rows = static_cast<nml_dcmatrix *>(with_length(m, sizeof(nml_dcmatrix)));
  nml_dcscalar *data = static_cast<nml_dcscalar *>(with_length(m * n, sizeof(nml_dcscalar)));
  for (nml_extent i = 0; i < m; ++i) rows[i] = data + i * n;
  return rows;
}
// three bands of m entries, reached through a pointer to the middle one
nml_d3bands *nml_d3_new(nml_extent m) {
  nml_d3bands *b = static_cast<nml_d3bands *>(with_length(3, sizeof(nml_d3bands)));
  for (int k = 0; k < 3; ++k) b[k] = nml_dv_new(m);
  return b + 1;
}
void nml_d3_delete(nml_d3bands *p) {
  if (!p) return;
  for (int k = -1; k <= 1; ++k) nml_dv_delete(p[k]);
  release(p - 1);
}
nml_extent nml_d3_extent(const nml_d3bands *p) { return length_of(p[0]); }
nml_d3bands *nml_d3_clone(const nml_d3bands *p) {
  const nml_extent m = length_of(p[0]);
  nml_d3bands *q = nml_d3_new(m);
  for (int k = -1; k <= 1; ++k) memcpy(q[k], p[k], sizeof(double) * m);
  return q;
}
void nml_memory_report(char *) {}
void error(char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  exit(3);
}

// ---------------------------------------------------------------- LAPACK
extern "C" void scipy_dstebz_(const char *, const char *, const int *, const double *,
                              const double *, const int *, const int *, const double *,
                              const double *, const double *, int *, int *, double *, int *,
                              int *, double *, int *, int *, size_t, size_t);
extern "C" void dstebz(const char *range, const char *order, const int *n, const double *vl,
                       const double *vu, const int *il, const int *iu, const double *abstol,
                       const nml_dvector *d, const nml_dvector *e, int *m, int *nsplit,
                       nml_dvector *w, nml_ivector *iblock, nml_ivector *isplit,
                       nml_dvector *work, nml_ivector *iwork, int *info) {
  scipy_dstebz_(range, order, n, vl, vu, il, iu, abstol, d, e, m, nsplit, w, iblock, isplit,
                work, iwork, info, 1, 1);
}

// ---------------------------------------------------------------- H*x
// argList[0]: the oracle's stored Hamiltonian, argList[1]: &shift
struct OracleH {
  int norb, nspin;
  long natoms;
  const int *atom_slot, *nbr;
  const signed char *wrap;
  const double *kvec, *onsite, *blocks;
};

static void oracle_matmul(const int **argList, nml_dcscalar *y, const nml_dcscalar *x) {
  const OracleH *h = reinterpret_cast<const OracleH *>(argList[0]);
  const double shift = argList[1] ? *reinterpret_cast<const double *>(argList[1]) : 0.0;
  orc_hx(h->norb, h->nspin, h->natoms, h->atom_slot, h->nbr, h->wrap, h->kvec, h->onsite,
         h->blocks, shift, reinterpret_cast<const double *>(x), reinterpret_cast<double *>(y));
}

// The reference's first pass (eigenvaluesLanczos, lanczos.c:1282-1357) from
// the start vector r0 (2*length doubles): values[imax] ascending,
// conv_iterations[imax], *iterations; returns the number of values found.
extern "C" int ref_eigenvalues_lanczos(const OracleH *h, long length, const double *r0,
                                       int conv_start, int conv_skip, int imax, int requested1,
                                       int requested2, double emin1, double emax1, double emin2,
                                       double emax2, double tolerance, double *values,
                                       int *conv_iterations, int *iterations) {
  nml_dvector *value = nml_dv_new(imax);
  nml_ivector *conv = nml_iv_new(imax);
  nml_d3bands *T = nml_d3_new(imax);
  nml_dcvector *r_n = nml_dcv_new(length), *q_n = nml_dcv_new(length),
               *q_n1 = nml_dcv_new(length);
  memcpy(r_n, r0, sizeof(nml_dcscalar) * length);
  double shift = 0.0;
  const int *args[3] = {reinterpret_cast<const int *>(h), reinterpret_cast<const int *>(&shift),
                        nullptr};
  nml_extent its = 0;
  const nml_extent ne =
      eigenvaluesLanczos(value, conv, T, &its, r_n, q_n, q_n1, length, requested1, requested2,
                         conv_start, conv_skip, imax, emin1, emax1, emin2, emax2, tolerance,
                         100.0 * tolerance, oracle_matmul, args, nullptr, nullptr, 0);
  for (nml_extent k = 0; k < ne; ++k) {
    values[k] = value[k];
    conv_iterations[k] = conv[k];
  }
  *iterations = int(its);
  nml_dv_delete(value);
  nml_iv_delete(conv);
  nml_d3_delete(T);
  release(r_n);
  release(q_n);
  release(q_n1);
  return int(ne);
}
