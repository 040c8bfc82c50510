// ref_lanczos_driver.cc -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
//
// Links the reference's own Lanczos drivers (eigen/src/lanczos.c and
// eigen/src/lanczos_blk.c, compiled where they lie by oracle/build_ref.sh,
// with the reference's fake MPI layer eigen/src/mpi_fake.c) into
// oracle/_ref/libref_lanczos.so, so that the CPU baseline of the benchmark
// and the tests can run the reference's eigenvaluesLanczos -- its
// recurrence, convergence windows, dstebz bisection and ghost handling --
// and its block Lanczos (block_Lanczos_QR, single_iteration, the zhbevx
// band solve and the Method-4 convergence test) on a real Hamiltonian.  The H*x it calls
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
//  * LAPACK's dstebz, zhbevx, zgbtrf and zgbtrs, forwarded to the routines
//    scipy's bundled OpenBLAS exports (the reference builds its vendored
//    Fortran LAPACK, and no Fortran compiler is present here);
//  * ARPACK's znaupd/zneupd, which only lanczos_blk.c's eigenvector routine
//    calls (ARPACK is not present): stubs that stop the process if reached;
//  * the MPI rank globals of a serial run;
//  * Allreduce_MPI_sp as a function with MPI's meaning (copy `count`
//    doubles).  lanczos_blk.c is compiled with the reference's
//    NoGnuStatementExpre switch, which selects this function (and the
//    complex-pointer overload of oracle/ref_blk_compat.h): the serial
//    build's default statement-expression macro copies `count` elements of
//    the pointer's own type, and dot_product (lanczos_blk.c:172) passes a
//    complex pointer with count 2 (MPI's two doubles), writing 32 bytes into
//    the caller's 16-byte result on the stack.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <vector>

#include "lanczos.h"
#include "ref_blk_compat.h"

extern "C" {
#include "tb_oracle.h"
}

// ---------------------------------------------------------------- serial MPI
int mpi_n3d_id = 0;
int mpi_n3d_masterid = 0;
int mpi_n3d_numprocs = 1;

void Allreduce_MPI_sp(double *pa, double *pb, int count, MPI_Datatype, MPI_Op, MPI_Comm) {
  for (int i = 0; i < count; ++i) pb[i] = pa[i];
}
void Allreduce_MPI_sp(nml_dcomplex *pa, nml_dcomplex *pb, int count, MPI_Datatype d, MPI_Op o,
                      MPI_Comm c) {
  Allreduce_MPI_sp(reinterpret_cast<double *>(pa), reinterpret_cast<double *>(pb), count, d, o,
                   c);
}

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
void nml_dcm_delete(nml_dcmatrix *p) {
  if (!p) return;
  release(p[0]);
  release(p);
}
void nml_dcv_delete(nml_dcvector *p) { release(p); }
void *nml_malloc(size_t n) {
  void *p = calloc(1, n > 0 ? n : 1);
  if (!p) {
    fprintf(stderr, "ref_lanczos_driver: out of memory\n");
    exit(2);
  }
  return p;
}
void nml_free(void *p) { free(p); }
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

// the band solves of lanczos_blk.c (FORTRAN_UNDERSCORE names); the complex
// type is two doubles in both
extern "C" void scipy_zhbevx_(const char *, const char *, const char *, const int *, const int *,
                              void *, const int *, void *, const int *, const double *,
                              const double *, const int *, const int *, const double *, int *,
                              double *, void *, const int *, void *, double *, int *, int *,
                              int *, size_t, size_t, size_t);
extern "C" void scipy_zgbtrf_(const int *, const int *, const int *, const int *, void *,
                              const int *, int *, int *);
extern "C" void scipy_zgbtrs_(const char *, const int *, const int *, const int *, const int *,
                              const void *, const int *, const int *, void *, const int *, int *,
                              size_t);
extern "C" {
void zhbevx_(char *jobz, char *range, char *uplo, int *n, int *kd, void *ab, int *ldab, void *q,
             int *ldq, double *vl, double *vu, int *il, int *iu, double *abstol, int *m,
             double *w, void *z, int *ldz, void *work, double *rwork, int *iwork, int *ifail,
             int *info) {
  scipy_zhbevx_(jobz, range, uplo, n, kd, ab, ldab, q, ldq, vl, vu, il, iu, abstol, m, w, z, ldz,
                work, rwork, iwork, ifail, info, 1, 1, 1);
}
void zgbtrf_(int *m, int *n, int *kl, int *ku, void *ab, int *ldab, int *ipiv, int *info) {
  scipy_zgbtrf_(m, n, kl, ku, ab, ldab, ipiv, info);
}
void zgbtrs_(char *trans, int *n, int *kl, int *ku, int *nrhs, void *ab, int *ldab, int *ipiv,
             void *b, int *ldb, int *info) {
  scipy_zgbtrs_(trans, n, kl, ku, nrhs, ab, ldab, ipiv, b, ldb, info, 1);
}
void znaupd_() {
  fprintf(stderr, "ref_lanczos_driver: ARPACK znaupd is not available\n");
  exit(4);
}
void zneupd_() {
  fprintf(stderr, "ref_lanczos_driver: ARPACK zneupd is not available\n");
  exit(4);
}
}

// lanczos_blk.c's routines (declared there, not in a header)
void block_Lanczos_QR(std::vector<nml_dcvector *> *R, std::vector<nml_dcvector *> *Q,
                      nml_dcmatrix *Beta, nml_extent m, int p);
int block_lanczos_blocktridiagonal(
    nml_dvector *eigv_conv, nml_dcmatrix *triad, nml_extent *pIterations, int p,
    std::vector<nml_dcvector *> *R_n, std::vector<nml_dcvector *> *Q_n,
    std::vector<nml_dcvector *> *Q_n1, nml_extent length, int requested1, int requested2,
    int ConvCheckStartIter, int ConvCheckSkipRate, int imax, nml_dscalar emin1,
    nml_dscalar emax1, nml_dscalar emin2, nml_dscalar emax2, nml_dscalar tolerance,
    nml_dscalar resolution, void (*matmul)(const int **, nml_dcscalar *, const nml_dcscalar *),
    const int *argument[], FILE *fp_trace, FILE *fp_log, int verbose, int *tridiag_size,
    double deflation_tolerance, int max_no_success, int *found_vb, int *found_cb,
    int deflation_on, int conv_method);

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

// The reference's block Lanczos eigenvalue pass as eigensolve_blk_lanczos
// runs it (lanczos_blk.c:2208-2255): the start block r0 (p vectors of
// 2*length doubles, back to back) orthonormalised by block_Lanczos_QR, then
// block_lanczos_blocktridiagonal with resolution 100*tolerance, no
// deflation, no trace or log files.  values[imax*p] ascending (the
// reference sorts them), *found_vb, *found_cb, *iterations as the routine
// leaves them; returns the number of eigenvalues.  max_no_success <= 0 means
// no limit.  The routine prints progress lines on stdout.
extern "C" int ref_block_lanczos(const OracleH *h, long length, int p, const double *r0,
                                 int conv_start, int conv_skip, int imax, int requested1,
                                 int requested2, double emin1, double emax1, double emin2,
                                 double emax2, double tolerance, int max_no_success,
                                 double *values, int *found_vb, int *found_cb, int *iterations) {
  std::vector<nml_dcvector *> R_n, Q_n, Q_n1, Q_start;
  for (int i = 0; i < p; ++i) {
    nml_dcvector *r = nml_dcv_new(length);
    memcpy(r, r0 + size_t(i) * 2 * length, sizeof(nml_dcscalar) * length);
    Q_start.push_back(r);
    R_n.push_back(nml_dcv_new(length));
    Q_n.push_back(nml_dcv_new(length));
    Q_n1.push_back(nml_dcv_new(length));
  }
  nml_dcmatrix *tri = nml_dcm_new(nml_extent(imax) * p, p + 1);
  nml_dcmatrix *Beta = nml_dcm_new(p, p);
  block_Lanczos_QR(&Q_start, &Q_n, Beta, length, p);
  nml_dvector *value = nml_dv_new(nml_extent(imax) * p);
  double shift = 0.0;
  const int *args[3] = {reinterpret_cast<const int *>(h), reinterpret_cast<const int *>(&shift),
                        nullptr};
  nml_extent its = 0;
  int tridiag_size = 0, fvb = 0, fcb = 0;
  const int ne = block_lanczos_blocktridiagonal(
      value, tri, &its, p, &R_n, &Q_n, &Q_n1, length, requested1, requested2, conv_start,
      conv_skip, imax, emin1, emax1, emin2, emax2, tolerance, 100.0 * tolerance, oracle_matmul,
      args, nullptr, nullptr, 0, &tridiag_size, 0.0,
      max_no_success > 0 ? max_no_success : (1 << 30), &fvb, &fcb, 0, 4);
  for (int k = 0; k < ne; ++k) values[k] = value[k];
  *found_vb = fvb;
  *found_cb = fcb;
  *iterations = int(its);
  nml_dv_delete(value);
  nml_dcm_delete(tri);
  nml_dcm_delete(Beta);
  for (int i = 0; i < p; ++i) {
    release(R_n[i]);
    release(Q_n[i]);
    release(Q_n1[i]);
    release(Q_start[i]);
  }
  return ne;
}
