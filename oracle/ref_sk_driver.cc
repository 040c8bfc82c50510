// ref_sk_driver.cc -- TEST INFRASTRUCTURE ONLY.
//
// A small driver that links the reference's own Slater-Koster routines
// (nemo3d/src/ham/mb_ham_spds_micro.c, compiled where it lies by
// oracle/build_ref.sh) so that the oracle's restatement of them can be
// checked against the real thing.  Nothing of the product uses it.
//
// The reference's vector/matrix helpers come from its nml library, whose
// sources are generated by a template tool; the few the routines call are
// implemented here on the interface the nml headers declare (a vector keeps
// its length in the word before its first element).
//
// Protocol (binary, native endian) on stdin, answers on stdout, one record
// per command until end of input:
//   int32 cmd = 1  bond block, h3d_offdiag_diag_corr (mb_ham_spds_micro.c:597)
//       int32 nbasis, spin_model (1: Basis_Spin 1/0 halves, -1: no spin),
//             this_cation, with_strain
//       double nnv[3], nnv0[3], a0, param[35], strain[33]
//     -> double ho[nbasis][nbasis][2], hd[nbasis][nbasis][2]
//   int32 cmd = 2  on-site block, h3d_diag (mb_ham_spds_micro.c:1453)
//       int32 nbasis, spin_model, cation; double param[35]
//     -> double h[nbasis][nbasis][2]
//   int32 cmd = 3  param_sp3s_2_sp3d5s (mb_ham_spds_micro.c:2984)
//       double param_in[15], a0 -> double param_out[35]
//   int32 cmd = 4  dangling-bond passivation,
//                  h3d_diag_dangling_bond_shift_zincblende
//                  (mb_ham_spds_micro.c:1910-2150), on a closed box
//       int32 nbasis (10: sp3s* with spin, 20: sp3d5s* with spin), nx, ny, nz
//       double DanglingBondEnergyShift
//       uint8 occupied[nx][ny][nz][8] (the reference's AtomType != 0)
//       int32 count, then count pairs (cell index, atom in cell) with cell
//             index (i * ny + j) * nz + k
//     -> per pair double h[nbasis][nbasis][2], the routine's additions to a
//        zero on-site block
//     The cell's neighbour map, positions and neighbour counts come from the
//     reference's own Cell::Initialize (nemo3d/src/base/Cell.c, compiled where
//     it lies) for the zincblende crystal.
// The basis and spin arrays are the ones basis_init builds
// (nemo3d/src/base/ham3d_final.c:597-619).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mb_ham_spds_micro.h"
#include "mb_ham_spds_micro2.h"

// ---------------------------------------------------------------- nml helpers
namespace {
template <typename T>
T *nml_alloc(long n) {
  // 16-byte header holding the length, then the elements
  char *raw = static_cast<char *>(calloc(1, 16 + sizeof(T) * (n > 0 ? n : 1)));
  if (!raw) {
    fprintf(stderr, "ref_sk_driver: out of memory\n");
    exit(2);
  }
  *reinterpret_cast<nml_extent *>(raw + 8) = static_cast<nml_extent>(n);
  return reinterpret_cast<T *>(raw + 16);
}
template <typename T>
void nml_free(T *p) {
  if (p) free(reinterpret_cast<char *>(p) - 16);
}
template <typename T>
nml_extent nml_len(const T *p) {
  return *reinterpret_cast<const nml_extent *>(reinterpret_cast<const char *>(p) - 8);
}
}  // namespace

rvectr Rvectr(int n) { return nml_alloc<double>(n); }
cvectr Cvectr(int n) { return nml_alloc<nml_dcomplex>(n); }
ivectr Ivectr(int n) { return nml_alloc<int>(n); }
void rm_rvectr(rvectr *p) { if (p) { nml_free(*p); *p = NULL; } }
void rm_cvectr(cvectr *p) { if (p) { nml_free(*p); *p = NULL; } }
void rm_ivectr(ivectr *p) { if (p) { nml_free(*p); *p = NULL; } }
nml_extent nml_dv_extent(const nml_dvector *p) { return nml_len(p); }
nml_extent nml_iv_extent(const nml_ivector *p) { return nml_len(p); }
rvectr check_rvectr(rvectr p, int n) {
  if (!p) return Rvectr(n);
  if (nml_len(p) != static_cast<nml_extent>(n)) {
    nml_free(p);
    return Rvectr(n);
  }
  return p;
}
rmatrix Rmatrix(int n, int m) {
  rmatrix rows = nml_alloc<double *>(n);
  double *data = nml_alloc<double>(static_cast<long>(n) * m);
  for (int i = 0; i < n; ++i) rows[i] = data + static_cast<long>(i) * m;
  return rows;
}
void rm_rmatrix(rmatrix *p) {
  if (p && *p) {
    nml_free((*p)[0]);
    nml_free(*p);
    *p = NULL;
  }
}
void rm_cmatrix(cmatrix *p) {
  if (p && *p) {
    nml_free((*p)[0]);
    nml_free(*p);
    *p = NULL;
  }
}
// 3-D tensors with lower bounds (the nml i3tensor/r3tensor interface):
// t[i][j][k] for lb3 <= i <= ub3, lb2 <= j <= ub2, lb1 <= k <= ub1
template <typename T>
T ***tensor3(int lb3, int ub3, int lb2, int ub2, int lb1, int ub1) {
  const int n3 = ub3 - lb3 + 1, n2 = ub2 - lb2 + 1, n1 = ub1 - lb1 + 1;
  T ***p = static_cast<T ***>(calloc(n3, sizeof(T **)));
  T **rows = static_cast<T **>(calloc(size_t(n3) * n2, sizeof(T *)));
  T *data = static_cast<T *>(calloc(size_t(n3) * n2 * n1, sizeof(T)));
  if (!p || !rows || !data) {
    fprintf(stderr, "ref_sk_driver: out of memory\n");
    exit(2);
  }
  for (int a = 0; a < n3; ++a) {
    p[a] = rows + size_t(a) * n2 - lb2;
    for (int b = 0; b < n2; ++b) rows[size_t(a) * n2 + b] = data + (size_t(a) * n2 + b) * n1 - lb1;
  }
  return p - lb3;
}
i3tensor I3tensor(int a, int b, int c, int d, int e, int f) { return tensor3<int>(a, b, c, d, e, f); }
r3tensor R3tensor(int a, int b, int c, int d, int e, int f) {
  return tensor3<double>(a, b, c, d, e, f);
}
void rm_i3tensor(i3tensor *p, int) { if (p) *p = NULL; }  // the driver's tensors live until exit
void rm_r3tensor(r3tensor *p, int) { if (p) *p = NULL; }

complex Complex(double r, double i) {
  complex z;
  z.r = r;
  z.i = i;
  return z;
}
complex cadd(complex a, complex b) { return Complex(a.r + b.r, a.i + b.i); }
complex cmul(complex a, complex b) {
  return Complex(a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r);
}
complex cconj(complex a) { return Complex(a.r, -a.i); }
// the master-rank output stream Cell::Initialize writes its notices to
ostream_N3D cout_master;
// only reached for tilted periodic crystals, which the driver never builds
int geo_struct::get_cindx_tilted(int, int, int) {
  fprintf(stderr, "ref_sk_driver: tilted crystals are not supported\n");
  exit(7);
}
void die(char *s, ...) {
  fprintf(stderr, "reference die(): %s\n", s);
  exit(3);
}

// ---------------------------------------------------------------- driver
namespace {
cmatrix cmat(int n) {
  cmatrix rows = nml_alloc<nml_dcomplex *>(n);
  nml_dcomplex *data = nml_alloc<nml_dcomplex>(static_cast<long>(n) * n);
  for (int i = 0; i < n; ++i) rows[i] = data + static_cast<long>(i) * n;
  return rows;
}
bool rd(void *p, size_t bytes) { return fread(p, 1, bytes, stdin) == bytes; }
void wr_cmat(cmatrix h, int n) {
  for (int i = 0; i < n; ++i) fwrite(h[i], sizeof(nml_dcomplex), n, stdout);
}
// basis_init (ham3d_final.c:597-619) for the models with 10 or 20 states
void basis(int nbasis, int spin_model, ivectr an, ivectr ca, ivectr sp) {
  if (spin_model == 1) {
    for (int i = 0; i < nbasis / 2; ++i) {
      sp[i] = 1;
      sp[i + nbasis / 2] = 0;
      an[i] = an[i + nbasis / 2] = i;
      ca[i] = ca[i + nbasis / 2] = i + 10;
    }
  } else {
    for (int i = 0; i < nbasis; ++i) {
      sp[i] = -1;
      an[i] = i;
      ca[i] = i + 10;
    }
  }
}
}  // namespace

int main() {
  int32_t cmd;
  while (rd(&cmd, 4)) {
    if (cmd == 1) {
      int32_t h[4];
      double geo[7];
      if (!rd(h, sizeof(h)) || !rd(geo, sizeof(geo))) return 4;
      const int nb = h[0];
      if (nb != 10 && nb != 20) return 5;
      rvectr par = Rvectr(sp3d5s_nparam), str = Rvectr(sp3d5s_nstrain);
      if (!rd(par, sizeof(double) * sp3d5s_nparam) || !rd(str, sizeof(double) * sp3d5s_nstrain))
        return 4;
      rvectr nnv = Rvectr(3), nnv0 = Rvectr(3);
      for (int d = 0; d < 3; ++d) {
        nnv[d] = geo[d];
        nnv0[d] = geo[3 + d];
      }
      ivectr an = Ivectr(nb), ca = Ivectr(nb), sp = Ivectr(nb);
      basis(nb, h[1], an, ca, sp);
      cmatrix ho = cmat(nb), hd = cmat(nb);
      h3d_offdiag_diag_corr(ho, hd, nnv, nnv0, h[2] ? ca : an, h[2] ? an : ca, sp, par,
                            h[3] ? str : NULL, geo[6], nb);
      wr_cmat(ho, nb);
      wr_cmat(hd, nb);
      rm_cmatrix(&ho);
      rm_cmatrix(&hd);
      rm_ivectr(&an);
      rm_ivectr(&ca);
      rm_ivectr(&sp);
      rm_rvectr(&nnv);
      rm_rvectr(&nnv0);
      rm_rvectr(&par);
      rm_rvectr(&str);
    } else if (cmd == 2) {
      int32_t h[3];
      if (!rd(h, sizeof(h))) return 4;
      const int nb = h[0];
      if (nb != 10 && nb != 20) return 5;
      rvectr par = Rvectr(sp3d5s_nparam);
      if (!rd(par, sizeof(double) * sp3d5s_nparam)) return 4;
      ivectr an = Ivectr(nb), ca = Ivectr(nb), sp = Ivectr(nb);
      basis(nb, h[1], an, ca, sp);
      cmatrix hm = cmat(nb);
      h3d_diag(hm, h[2] ? ca : an, sp, par, nb);
      wr_cmat(hm, nb);
      rm_cmatrix(&hm);
      rm_ivectr(&an);
      rm_ivectr(&ca);
      rm_ivectr(&sp);
      rm_rvectr(&par);
    } else if (cmd == 3) {
      rvectr pin = Rvectr(sp3s_nparam);
      double a0;
      if (!rd(pin, sizeof(double) * sp3s_nparam) || !rd(&a0, 8)) return 4;
      rvectr pout = param_sp3s_2_sp3d5s(pin, NULL, a0, 1.0, 1.0, 1.0);
      fwrite(pout, sizeof(double), sp3d5s_nparam, stdout);
      rm_rvectr(&pout);
      rm_rvectr(&pin);
    } else if (cmd == 4) {
      int32_t h[4];
      double shift;
      if (!rd(h, sizeof(h)) || !rd(&shift, 8)) return 4;
      const int nb = h[0], nx = h[1], ny = h[2], nz = h[3];
      if ((nb != 10 && nb != 20) || nx < 1 || ny < 1 || nz < 1) return 5;
      const long ncell = long(nx) * ny * nz;
      unsigned char *occ = static_cast<unsigned char *>(malloc(ncell * 8));
      if (!occ || !rd(occ, ncell * 8)) return 4;
      // the routine reads opt, hd, geo and BandModel of the structure; the
      // rest of it stays zero (no constructors run)
      QD_struct *d = static_cast<QD_struct *>(calloc(1, sizeof(QD_struct)));
      top_struct *opt = new top_struct();
      opt->Dev.StructFile = "NULL";
      opt->Dev.CrystalStruct = Dev_struct::Zincblende;
      Cell *cell = new Cell();
      cell->Initialize(*opt);
      memcpy(static_cast<void *>(&d->geo.cellgeom), static_cast<void *>(cell), sizeof(Cell));
      d->opt.ExecParam.Phys.DanglingBondEnergyShift = shift;
      d->BandModel = nb == 10 ? BM_10_sp3ss_spin : BM_20_sp3d5ss_spin;
      d->geo.N_Cell = int(ncell);
      d->geo.ijk__cell = I3tensor(-1, nx, -1, ny, -1, nz);
      for (int i = -1; i <= nx; ++i)
        for (int j = -1; j <= ny; ++j)
          for (int k = -1; k <= nz; ++k)
            d->geo.ijk__cell[i][j][k] =
                (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) ? -1
                                                                           : (i * ny + j) * nz + k;
      d->geo.cell__ijk = static_cast<int **>(calloc(ncell, sizeof(int *)));
      d->geo.AtomType = static_cast<nml_bscalar **>(calloc(ncell, sizeof(nml_bscalar *)));
      for (long l = 0; l < ncell; ++l) {
        d->geo.cell__ijk[l] = static_cast<int *>(calloc(3, sizeof(int)));
        d->geo.cell__ijk[l][0] = int(l / (long(ny) * nz));
        d->geo.cell__ijk[l][1] = int((l / nz) % ny);
        d->geo.cell__ijk[l][2] = int(l % nz);
        d->geo.AtomType[l] = static_cast<nml_bscalar *>(calloc(8, sizeof(nml_bscalar)));
        for (int m = 0; m < 8; ++m) d->geo.AtomType[l][m] = occ[l * 8 + m] != 0;
      }
      int32_t count;
      if (!rd(&count, 4)) return 4;
      for (int q = 0; q < count; ++q) {
        int32_t ca[2];
        if (!rd(ca, sizeof(ca)) || ca[0] < 0 || ca[0] >= ncell || ca[1] < 0 || ca[1] > 7) return 4;
        d->hd = cmat(nb);
        h3d_diag_dangling_bond_shift_zincblende(d, ca[0], ca[1]);
        wr_cmat(d->hd, nb);
        rm_cmatrix(&d->hd);
      }
      free(occ);
    } else {
      return 6;
    }
  }
  fflush(stdout);
  return 0;
}
