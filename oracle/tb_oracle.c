/*
 * tb_oracle.c -- CPU oracle for the NEMO-3D tight-binding hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see tb_oracle.h).  A plain-C restatement of the
 * reference algorithm, written for readability and checked against the
 * reference's golden eigenvalue files and, where the reference compiles here,
 * against the reference's own routines (oracle/_ref).  Paths cited are
 * relative to the NEMO-3D source tree.
 */
#include "tb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Host threads of the oracle's OpenMP loops (the CPU baseline times the
 * reference's serial path with 1 and the parallel restatement with all). */
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* The reference's sqrt(3) constant (mb_ham_spds_micro.c:42).  It is not the
 * correctly rounded sqrt(3); H entries only agree to 1e-12 with it. */
#define SQR3 1.73205080757

/* --- parameter vector layout (mb_ham_spds_micro.h:100-264) --------------- */
enum { pE_sa = 0, pE_pa, pE_sc, pE_pc, pE_sta, pE_stc, pE_da, pE_dc, pE_La,
       pE_Lc };
enum { eta_ssts = 0, eta_ststs, eta_sss, eta_sps, eta_pps, eta_ppp, eta_sds,
       eta_stps, eta_pds, eta_pdp, eta_const, eta_dds, eta_ddp, eta_ddd,
       eta_stds, eta_cat_shift, eta_an_shift };
#define STR(i) (ORC_NPV + (i))

/* orbital types and the orbital order s*, s, px, py, pz, dxy, dyz, dzx,
 * dx2-y2, dz2 (mb_ham_spds_micro.h:97-116, ham3d_final.c:601-610) */
enum { T_SST = 0, T_S = 1, T_P = 2, T_D = 3 };
static const int orb_type[10] = {T_SST, T_S, T_P, T_P, T_P,
                                 T_D, T_D, T_D, T_D, T_D};

/* ------------------------------------------------------------------------ */
/* param_init (base/mat3d.c:133-307) and param_sp3s_2_sp3d5s
 * (ham/mb_ham_spds_micro.c:2984-3026) for one material set. */
int orc_prepare_params(int sp3s_family, int include_strain, const double *pv,
                       const double *strain, double ev_offset, double a0,
                       double *out) {
  double *p = out;
  double shift_c = 0.0, shift_a = 0.0;
  int i;
  memset(out, 0, sizeof(double) * ORC_NPAR);
  if (sp3s_family) {
    const double r3 = sqrt(3.0);
    for (i = 0; i < 6; i++) p[i] = pv[i];
    p[8] = pv[13] / 3;
    p[9] = pv[14] / 3;
    p[10] = pv[6] / 4;
    p[14] = pv[9] * r3 / 4;
    p[15] = pv[10] * r3 / 4;
    p[16] = pv[11] * r3 / 4;
    p[17] = pv[12] * r3 / 4;
    p[22] = (pv[7] + 2 * pv[8]) / 4;
    p[23] = (pv[7] - pv[8]) / 4;
    p[31] = a0;
    p[32] = p[33] = p[34] = 1.0;
  } else {
    for (i = 0; i < ORC_NPV; i++) p[i] = pv[i];
  }
  for (i = 0; i < ORC_NSTR; i++) out[STR(i)] = strain[i];
  if (include_strain) { /* STRAIN_SHIFT_ENABLE, mat3d.c:153-165 */
    shift_c = strain[eta_cat_shift];
    shift_a = strain[eta_an_shift];
  }
  p[pE_sa] += ev_offset - shift_a;
  p[pE_pa] += ev_offset - shift_a;
  p[pE_sta] += ev_offset - shift_a;
  p[pE_sc] += ev_offset - shift_c;
  p[pE_pc] += ev_offset - shift_c;
  p[pE_stc] += ev_offset - shift_c;
  if (!sp3s_family) {
    p[pE_da] += ev_offset - shift_a;
    p[pE_dc] += ev_offset - shift_c;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Zincblende cell (base/Cell.c:185-210) and neighbour map (Cell.c:599-715). */
static const double pin[8][3] = {
    {0, 0, 0},          {0, -0.5, -0.5},      {-0.5, -0.5, 0},
    {-0.5, 0, -0.5},    {-0.25, -0.25, -0.25}, {-0.25, -0.75, -0.75},
    {-0.75, -0.75, -0.25}, {-0.75, -0.25, -0.75}};
static const int nnmap[8][4][4] = {
    {{0, 0, 0, 4}, {1, 0, 1, 7}, {1, 1, 0, 6}, {0, 1, 1, 5}},
    {{0, 0, 0, 5}, {0, 0, 0, 4}, {1, 0, 0, 6}, {1, 0, 0, 7}},
    {{0, 0, 0, 4}, {0, 0, 0, 6}, {0, 0, 1, 5}, {0, 0, 1, 7}},
    {{0, 0, 0, 4}, {0, 0, 0, 7}, {0, 1, 0, 5}, {0, 1, 0, 6}},
    {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 0, 2}, {0, 0, 0, 3}},
    {{0, 0, 0, 1}, {0, -1, 0, 3}, {0, 0, -1, 2}, {0, -1, -1, 0}},
    {{0, 0, 0, 2}, {0, -1, 0, 3}, {-1, 0, 0, 1}, {-1, -1, 0, 0}},
    {{0, 0, 0, 3}, {0, 0, -1, 2}, {-1, 0, 0, 1}, {-1, 0, -1, 0}}};

/* site index of (cell i,j,k ; in-cell atom m) */
static long site_of(const orc_geom *g, int i, int j, int k, int m) {
  return (((long)i * g->ny + j) * g->nz + k) * 8 + m;
}

/* Neighbour site of (i,j,k,m) along n; -1 if outside a closed boundary.
 * w receives the periodic image crossed per axis. */
static long nbr_site(const orc_geom *g, int i, int j, int k, int m, int n,
                     signed char w[3]) {
  int c[3] = {i + nnmap[m][n][0], j + nnmap[m][n][1], k + nnmap[m][n][2]};
  int dim[3] = {g->nx, g->ny, g->nz};
  int d;
  for (d = 0; d < 3; d++) {
    w[d] = 0;
    if (c[d] < 0 || c[d] >= dim[d]) {
      if (!g->periodic[d]) return -1;
      w[d] = (signed char)(c[d] < 0 ? -1 : 1);
      c[d] = (c[d] + dim[d]) % dim[d];
    }
  }
  return site_of(g, c[0], c[1], c[2], nnmap[m][n][3]);
}

/* get_total_hamiltonian_dimension_and_offsets (ham3d_final.c:547-568) after
 * remove_few_bonded_atoms(0) (geo_struct.c:1527-1579) and FindSurfaceAtoms
 * (geo_struct.c:1374-1463). */
long orc_topology(const orc_geom *g, long max_atoms, int *atom_slot, int *nbr,
                  signed char *wrap, unsigned char *surface) {
  long nsite = (long)g->nx * g->ny * g->nz * 8;
  long *index = (long *)malloc(sizeof(long) * nsite);
  long natoms = 0, s;
  int i, j, k, m, n;
  signed char w[3];
  /* pass 1: keep sites that hold an atom bonded to at least one in-domain
   * atom (the reference counts only non-wrapped neighbours here). */
  for (i = 0; i < g->nx; i++)
    for (j = 0; j < g->ny; j++)
      for (k = 0; k < g->nz; k++)
        for (m = 0; m < 8; m++) {
          s = site_of(g, i, j, k, m);
          index[s] = -1;
          if (!g->type[s]) continue;
          int bonds = 0;
          for (n = 0; n < 4; n++) {
            long t = nbr_site(g, i, j, k, m, n, w);
            if (t >= 0 && !w[0] && !w[1] && !w[2] && g->type[t]) bonds++;
          }
          if (bonds == 0) continue; /* zincblende: 8 atoms per cell */
          index[s] = natoms++;
        }
  if (natoms > max_atoms) {
    free(index);
    return -1;
  }
  /* pass 2: neighbour table in nnmap order */
  for (i = 0; i < g->nx; i++)
    for (j = 0; j < g->ny; j++)
      for (k = 0; k < g->nz; k++)
        for (m = 0; m < 8; m++) {
          s = site_of(g, i, j, k, m);
          long a = index[s];
          if (a < 0) continue;
          atom_slot[a] = (int)s;
          int cnt = 0;
          for (n = 0; n < 4; n++) {
            long t = nbr_site(g, i, j, k, m, n, w);
            long b = (t >= 0) ? index[t] : -1;
            nbr[a * 4 + n] = (int)b;
            wrap[(a * 4 + n) * 3 + 0] = b >= 0 ? w[0] : 0;
            wrap[(a * 4 + n) * 3 + 1] = b >= 0 ? w[1] : 0;
            wrap[(a * 4 + n) * 3 + 2] = b >= 0 ? w[2] : 0;
            if (b >= 0) cnt++;
          }
          surface[a] = (unsigned char)(cnt != 4);
        }
  free(index);
  return natoms;
}

/* ------------------------------------------------------------------------ */
/* Slater-Koster two-centre elements (Slater & Koster, Phys. Rev. 94, 1498
 * (1954), Table I) for an orbital "a" on the first atom and "b" on the second,
 * direction cosines (l,m,n) from the first atom to the second, with the
 * angular momentum of a not above that of b.  V = {sigma, pi, delta}. */
static double sk_std(int a, int b, double l, double m, double n, const double *V) {
  const double l2 = l * l, m2 = m * m, n2 = n * n;
  const double s3 = SQR3;
  int ta = orb_type[a], tb = orb_type[b];
  if (ta != T_P && ta != T_D && tb != T_P && tb != T_D) return V[0]; /* s,s* */
  if (ta != T_P && ta != T_D && tb == T_P) {                           /* s-p  */
    return (b == 2 ? l : b == 3 ? m : n) * V[0];
  }
  if (ta != T_P && ta != T_D && tb == T_D) { /* s-d */
    switch (b) {
    case 5: return s3 * l * m * V[0];
    case 6: return s3 * m * n * V[0];
    case 7: return s3 * n * l * V[0];
    case 8: return 0.5 * s3 * (l2 - m2) * V[0];
    default: return (n2 - 0.5 * (l2 + m2)) * V[0];
    }
  }
  if (ta == T_P && tb == T_P) { /* p-p */
    double da = a == 2 ? l : a == 3 ? m : n;
    double db = b == 2 ? l : b == 3 ? m : n;
    if (a == b) return da * da * V[0] + (1 - da * da) * V[1];
    return da * db * V[0] - da * db * V[1];
  }
  if (ta == T_P && tb == T_D) { /* p-d */
    const double Vs = V[0], Vp = V[1];
    switch (a * 16 + b) {
    case 2 * 16 + 5: return s3 * l2 * m * Vs + m * (1 - 2 * l2) * Vp;
    case 2 * 16 + 6: return s3 * l * m * n * Vs - 2 * l * m * n * Vp;
    case 2 * 16 + 7: return s3 * l2 * n * Vs + n * (1 - 2 * l2) * Vp;
    case 2 * 16 + 8: return 0.5 * s3 * l * (l2 - m2) * Vs + l * (1 - l2 + m2) * Vp;
    case 2 * 16 + 9: return l * (n2 - 0.5 * (l2 + m2)) * Vs - s3 * l * n2 * Vp;
    case 3 * 16 + 5: return s3 * l * m2 * Vs + l * (1 - 2 * m2) * Vp;
    case 3 * 16 + 6: return s3 * n * m2 * Vs + n * (1 - 2 * m2) * Vp;
    case 3 * 16 + 7: return s3 * l * m * n * Vs - 2 * l * m * n * Vp;
    case 3 * 16 + 8: return 0.5 * s3 * m * (l2 - m2) * Vs - m * (1 + l2 - m2) * Vp;
    case 3 * 16 + 9: return m * (n2 - 0.5 * (l2 + m2)) * Vs - s3 * m * n2 * Vp;
    case 4 * 16 + 5: return s3 * l * m * n * Vs - 2 * l * m * n * Vp;
    case 4 * 16 + 6: return s3 * m * n2 * Vs + m * (1 - 2 * n2) * Vp;
    case 4 * 16 + 7: return s3 * l * n2 * Vs + l * (1 - 2 * n2) * Vp;
    case 4 * 16 + 8: return 0.5 * s3 * n * (l2 - m2) * Vs - n * (l2 - m2) * Vp;
    default: return n * (n2 - 0.5 * (l2 + m2)) * Vs + s3 * n * (l2 + m2) * Vp;
    }
  }
  { /* d-d, symmetric in (a,b) */
    const double Vs = V[0], Vp = V[1], Vd = V[2];
    int x = a < b ? a : b, y = a < b ? b : a;
    const double q = n2 - 0.5 * (l2 + m2), lm = l2 - m2;
    switch (x * 16 + y) {
    case 5 * 16 + 5: return 3 * l2 * m2 * Vs + (l2 + m2 - 4 * l2 * m2) * Vp + (n2 + l2 * m2) * Vd;
    case 6 * 16 + 6: return 3 * m2 * n2 * Vs + (m2 + n2 - 4 * m2 * n2) * Vp + (l2 + m2 * n2) * Vd;
    case 7 * 16 + 7: return 3 * n2 * l2 * Vs + (n2 + l2 - 4 * n2 * l2) * Vp + (m2 + n2 * l2) * Vd;
    case 5 * 16 + 6: return 3 * l * m2 * n * Vs + l * n * (1 - 4 * m2) * Vp + l * n * (m2 - 1) * Vd;
    case 6 * 16 + 7: return 3 * m * n2 * l * Vs + m * l * (1 - 4 * n2) * Vp + m * l * (n2 - 1) * Vd;
    case 5 * 16 + 7: return 3 * l2 * m * n * Vs + m * n * (1 - 4 * l2) * Vp + m * n * (l2 - 1) * Vd;
    case 5 * 16 + 8: return 1.5 * l * m * lm * Vs - 2 * l * m * lm * Vp + 0.5 * l * m * lm * Vd;
    case 6 * 16 + 8: return 1.5 * m * n * lm * Vs - m * n * (1 + 2 * lm) * Vp + m * n * (1 + 0.5 * lm) * Vd;
    case 7 * 16 + 8: return 1.5 * n * l * lm * Vs + n * l * (1 - 2 * lm) * Vp - n * l * (1 - 0.5 * lm) * Vd;
    case 5 * 16 + 9: return s3 * l * m * q * Vs - s3 * 2 * l * m * n2 * Vp + 0.5 * s3 * l * m * (1 + n2) * Vd;
    case 6 * 16 + 9: return s3 * m * n * q * Vs + s3 * m * n * (l2 + m2 - n2) * Vp - 0.5 * s3 * m * n * (l2 + m2) * Vd;
    case 7 * 16 + 9: return s3 * l * n * q * Vs + s3 * l * n * (l2 + m2 - n2) * Vp - 0.5 * s3 * l * n * (l2 + m2) * Vd;
    case 8 * 16 + 8: return 0.75 * lm * lm * Vs + (l2 + m2 - lm * lm) * Vp + (n2 + 0.25 * lm * lm) * Vd;
    case 8 * 16 + 9: return 0.5 * s3 * lm * q * Vs - s3 * n2 * lm * Vp + 0.25 * s3 * (1 + n2) * lm * Vd;
    default: return q * q * Vs + 3 * n2 * (l2 + m2) * Vp + 0.75 * (l2 + m2) * (l2 + m2) * Vd;
    }
  }
}

/* Index of the two-centre integrals of an (anion type, cation type) pair in
 * the parameter vector (mb_ham_spds_micro.c:58-78), its strain exponent
 * (E_const_prep, mb_ham_spds_micro.c:2772-2845) and its strain-correction
 * coefficient (mb_ham_spds_micro.c:95-146). */
typedef struct {
  int v[3];   /* sigma, pi, delta parameter indices (-1 = unused) */
  int eta[3]; /* strain exponent indices */
  int c;      /* c_ind_* coefficient index within the strain vector */
  int par;    /* parity sign applied when the anion orbital has the higher l */
} pair_info;

static pair_info pair_of(int ta, int tc) {
  pair_info r = {{-1, -1, -1}, {0, 0, 0}, 0, 1};
#define SETP(V0, E0, C) do { r.v[0] = V0; r.eta[0] = E0; r.c = C; } while (0)
  if (ta == T_S && tc == T_S) SETP(10, eta_sss, 17);
  else if (ta == T_SST && tc == T_SST) SETP(11, eta_ststs, 18);
  else if (ta == T_SST && tc == T_S) SETP(12, eta_ssts, 19);
  else if (ta == T_S && tc == T_SST) SETP(13, eta_ssts, 20);
  else if (ta == T_S && tc == T_P) SETP(14, eta_sps, 21);
  else if (ta == T_P && tc == T_S) { SETP(15, eta_sps, 22); r.par = -1; }
  else if (ta == T_SST && tc == T_P) SETP(16, eta_stps, 23);
  else if (ta == T_P && tc == T_SST) { SETP(17, eta_stps, 24); r.par = -1; }
  else if (ta == T_S && tc == T_D) SETP(18, eta_sds, 25);
  else if (ta == T_D && tc == T_S) SETP(19, eta_sds, 26);
  else if (ta == T_SST && tc == T_D) SETP(20, eta_stds, 27);
  else if (ta == T_D && tc == T_SST) SETP(21, eta_stds, 28);
  else if (ta == T_P && tc == T_P) {
    SETP(22, eta_pps, 29); r.v[1] = 23; r.eta[1] = eta_ppp;
  } else if (ta == T_P && tc == T_D) {
    SETP(24, eta_pds, 30); r.v[1] = 26; r.eta[1] = eta_pdp;
  } else if (ta == T_D && tc == T_P) {
    SETP(25, eta_pds, 31); r.v[1] = 27; r.eta[1] = eta_pdp; r.par = -1;
  } else { /* d-d */
    SETP(28, eta_dds, 32); r.v[1] = 29; r.eta[1] = eta_ddp;
    r.v[2] = 30; r.eta[2] = eta_ddd;
  }
#undef SETP
  return r;
}

/* on-site energy index of an orbital type on the anion / cation
 * (diag_map_set, mb_ham_spds_micro.c:199-227) */
static int onsite_index(int type, int cation) {
  static const int an[4] = {pE_sta, pE_sa, pE_pa, pE_da};
  static const int ca[4] = {pE_stc, pE_sc, pE_pc, pE_dc};
  return cation ? ca[type] : an[type];
}

/* <anion orbital a | H | cation orbital c> for a bond with direction cosines
 * (l,m,n) from anion to cation, integrals taken from vector V. */
static double sk_pair(int a, int c, double l, double m, double n,
                      const double *V, const pair_info *pi) {
  double v[3] = {0, 0, 0};
  int k;
  for (k = 0; k < 3; k++) v[k] = pi->v[k] >= 0 ? V[pi->v[k]] : 0.0;
  int la = orb_type[a] == T_P ? 1 : orb_type[a] == T_D ? 2 : 0;
  int lc = orb_type[c] == T_P ? 1 : orb_type[c] == T_D ? 2 : 0;
  if (la <= lc) return sk_std(a, c, l, m, n, v);
  /* E_{a,c}(d) = (-1)^(la+lc) E_{c,a}(d) */
  return ((la + lc) % 2 ? -1.0 : 1.0) * sk_std(c, a, l, m, n, v);
}

/* One bond from the point of view of "this" atom: the norb x norb block
 * blk[c][a] = <anion a|H|cation c> and the strain-induced correction to this
 * atom's on-site energies accumulated into ediag[norb] in the reference's
 * order.  Restates h3d_offdiag_diag_corr (mb_ham_spds_micro.c:597-1451) with
 * strain_corr_prep (mb_ham_spds_micro.c:2848-2982) and the get_X_Y macros of
 * mb_ham_spds_VoffdEdiag_constructors.h.  nnv, nnv0 point anion -> cation. */
static void bond_block(int norb, int this_cation, const double *nnv,
                       const double *nnv0, const double *par, int use_strain,
                       double a0, double *blk, double *ediag) {
  const double *pv = par, *st = par + ORC_NPV;
  double scaled[ORC_NPV];
  double den0 = sqrt(nnv0[0] * nnv0[0] + nnv0[1] * nnv0[1] + nnv0[2] * nnv0[2]);
  double den = sqrt(nnv[0] * nnv[0] + nnv[1] * nnv[1] + nnv[2] * nnv[2]);
  double l0 = nnv0[0] / den0, m0 = nnv0[1] / den0, n0 = nnv0[2] / den0;
  double l = nnv[0] / den, m = nnv[1] / den, n = nnv[2] / den;
  double cstrain = use_strain ? st[eta_const] : 0.0;
  int i, a, c, k;
  memcpy(scaled, pv, sizeof(scaled));
  if (use_strain) {
    double brat = (0.25 * SQR3 * a0) / den;
    static const int vidx[21] = {10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20,
                                 21, 22, 23, 24, 25, 26, 27, 28, 29, 30};
    static const int eidx[21] = {eta_sss, eta_ststs, eta_ssts, eta_ssts,
                                 eta_sps, eta_sps, eta_stps, eta_stps,
                                 eta_sds, eta_sds, eta_stds, eta_stds,
                                 eta_pps, eta_ppp, eta_pds, eta_pds,
                                 eta_pdp, eta_pdp, eta_dds, eta_ddp, eta_ddd};
    for (i = 0; i < 21; i++)
      scaled[vidx[i]] = pv[vidx[i]] * pow(brat, st[eidx[i]]);
  }
  for (c = 0; c < norb; c++)
    for (a = 0; a < norb; a++) {
      pair_info pi = pair_of(orb_type[a], orb_type[c]);
      double r1 = sk_pair(a, c, l, m, n, scaled, &pi);
      blk[c * norb + a] = r1;
      (void)k;
    }
  /* strain correction: r3 = (r2^2 - r1^2) * cstrain / (E_a + E_c) * c_pair,
   * accumulated per row of this atom in the order of the neighbour's
   * orbitals (the macro denominators expand without outer parentheses). */
  for (i = 0; i < norb; i++) {
    double E = ediag[i];
    for (k = 0; k < norb; k++) {
      int a_ = this_cation ? k : i, c_ = this_cation ? i : k;
      pair_info pi = pair_of(orb_type[a_], orb_type[c_]);
      double r1 = blk[c_ * norb + a_];
      double r2 = sk_pair(a_, c_, l0, m0, n0, pv, &pi);
      double esum = pv[onsite_index(orb_type[a_], 0)] +
                    pv[onsite_index(orb_type[c_], 1)];
      E += (r2 * r2 - r1 * r1) * cstrain / esum * st[pi.c];
    }
    ediag[i] = E;
  }
}

/* spin-orbit element (mb_ham_spds_so.h) between p orbitals b1 (spin s1) and
 * b2 (spin s2) of one atom; spin 1 = up (first half), 0 = down. */
static void so_elem(int b1, int b2, int s1, int s2, double d, double *re,
                    double *im) {
  *re = *im = 0.0;
  if (s1 == 1 && s2 == 0) {
    if (b1 == 2 && b2 == 4) *re = d;
    if (b1 == 3 && b2 == 4) *im = -d;
    if (b1 == 4 && b2 == 2) *re = -d;
    if (b1 == 4 && b2 == 3) *im = d;
  } else if (s1 == 0 && s2 == 1) {
    if (b1 == 2 && b2 == 4) *re = -d;
    if (b1 == 3 && b2 == 4) *im = -d;
    if (b1 == 4 && b2 == 2) *re = d;
    if (b1 == 4 && b2 == 3) *im = d;
  } else if (s1 == 1 && s2 == 1) {
    if (b1 == 2 && b2 == 3) *im = -d;
    if (b1 == 3 && b2 == 2) *im = d;
  } else {
    if (b1 == 2 && b2 == 3) *im = d;
    if (b1 == 3 && b2 == 2) *im = -d;
  }
}

/* On-site block of one atom from its (bond-averaged) parameter vector p:
 * on-site energies on the diagonal and, for nspin = 2, the spin-orbit
 * couplings.  Restates h3d_diag (mb_ham_spds_micro.c:1453-1505) with the
 * spin-orbit table of mb_ham_spds_so.h.  h: [nb][nb] complex, overwritten. */
void orc_onsite_block(int norb, int nspin, int cation, const double *p, double *h) {
  const int nb = norb * nspin;
  int i, j;
  memset(h, 0, sizeof(double) * nb * nb * 2);
  for (i = 0; i < nb; i++) {
    int oi = i % norb, si = nspin == 2 ? (i < norb ? 1 : 0) : -1;
    h[(i * nb + i) * 2] = p[onsite_index(orb_type[oi], cation)];
    if (nspin == 2)
      for (j = 0; j < nb; j++) {
        int oj = j % norb, sj = j < norb ? 1 : 0;
        double re, im;
        so_elem(oi, oj, si, sj, cation ? p[pE_Lc] : p[pE_La], &re, &im);
        h[(i * nb + j) * 2] += re;
        h[(i * nb + j) * 2 + 1] += im;
      }
  }
}

/* One bond seen from "this" atom (public form of bond_block, for tests). */
void orc_bond(int norb, int this_cation, const double *nnv, const double *nnv0,
              const double *par, int use_strain, double a0, double *blk,
              double *ediag) {
  bond_block(norb, this_cation, nnv, nnv0, par, use_strain, a0, blk, ediag);
}

/* bond vectors anion->cation of atom (site) "this" to its neighbour n
 * (geo_struct::getRelativePosVec, geo_struct.c:2224-2297, with the sign flip
 * for a cation in H_DiagStrainCorr_OffDiag_Wrapper, h_cvectr_mult.c:1077-1100) */
static void bond_vectors(const orc_geom *g, long s_this, long s_nbr, int n,
                         double a0, double *nnv, double *nnv0) {
  int m = (int)(s_this % 8), mn = nnmap[m][n][3];
  int d;
  for (d = 0; d < 3; d++) {
    double norm = nnmap[m][n][d] + pin[mn][d] - pin[m][d];
    nnv0[d] = a0 * norm;
    nnv[d] = g->lattice[d] * norm;
    if (g->dsp) nnv[d] = nnv[d] + g->dsp[s_nbr * 3 + d] - g->dsp[s_this * 3 + d];
    if (m < 4) {
      nnv[d] = -nnv[d];
      nnv0[d] = -nnv0[d];
    }
  }
}

/* Assembly loop of Hmult_spds_col (h_cvectr_mult.c:1134-1886): on-site
 * block by H_Diag_Wrapper (h_cvectr_mult.c:841-1005) and h3d_diag
 * (mb_ham_spds_micro.c:1453-1505), dangling-bond passivation
 * (mb_ham_spds_micro.c:1910-2150), strain shift, and per-bond blocks with
 * their diagonal corrections. */
int orc_build(const orc_geom *g, const orc_model *md, long natoms,
              const int *atom_slot, const int *nbr, const signed char *wrap,
              const unsigned char *surface, double *onsite, double *blocks) {
  const int norb = md->norb, nspin = md->nspin, nb = norb * nspin;
  const int NS = md->nspecies;
  long a;
  int rc = 0;
  (void)wrap;
  memset(blocks, 0, sizeof(double) * natoms * 4 * norb * norb);
#pragma omp parallel for schedule(static) reduction(min : rc)
  for (a = 0; a < natoms; a++) {
    long s = atom_slot[a];
    int m = (int)(s % 8), cat = m < 4, n, i, j, d;
    int tthis = g->type[s];
    double p[ORC_NPAR], shiftsum = 0.0;
    double *h = onsite + (size_t)a * nb * nb * 2;
    int cnt = 0;
    memset(p, 0, sizeof(p));
    memset(h, 0, sizeof(double) * nb * nb * 2);
    /* bond-averaged parameters (h_cvectr_mult.c:855-916) */
    for (n = 0; n < 4; n++) {
      int b = nbr[a * 4 + n];
      if (b < 0) continue;
      int tn = g->type[atom_slot[b]];
      int c_ = cat ? tthis : tn, a_ = cat ? tn : tthis;
      if (!md->par_ok[c_ * NS + a_]) { rc = -1; continue; }
      const double *pp = md->par + ((size_t)c_ * NS + a_) * ORC_NPAR;
      for (i = 0; i < ORC_NPV; i++) p[i] += pp[i];
      if (md->include_strain)
        shiftsum += pp[ORC_NPV + (cat ? eta_cat_shift : eta_an_shift)];
      cnt++;
    }
    if (cnt == 0) continue;
    shiftsum /= cnt;
    for (i = 0; i < ORC_NPV; i++) p[i] /= cnt;
    orc_onsite_block(norb, nspin, cat, p, h); /* h3d_diag */
    /* dangling-bond passivation of surface atoms */
    if (md->passivate && surface[a]) {
      static const double bond[4][3] = {{0.25, 0.25, 0.25},
                                        {-0.25, -0.25, 0.25},
                                        {0.25, -0.25, -0.25},
                                        {-0.25, 0.25, -0.25}};
      double v[4], cosv = 0.0;
      double sh = md->dangling_shift * 0.25;
      int sp;
      for (n = 0; n < 4; n++) v[n] = sh;
      for (n = 0; n < 4; n++) {
        int mn = nnmap[m][n][3], ib = 0;
        double nn[3];
        for (d = 0; d < 3; d++) nn[d] = nnmap[m][n][d] + (pin[mn][d] - pin[m][d]);
        cosv = nn[0] * bond[0][0] + nn[1] * bond[0][1] + nn[2] * bond[0][2];
        while (fabs(cosv) < 0.15 && ib < 3) {
          ib++;
          cosv = nn[0] * bond[ib][0] + nn[1] * bond[ib][1] + nn[2] * bond[ib][2];
        }
        if (nbr[a * 4 + n] >= 0) v[ib] = 0.0;
      }
      double sgn = cosv > 0 ? 1.0 : -1.0;
      double vs0 = v[0] + v[1] + v[2] + v[3];
      double vs1 = v[0] - v[1] + v[2] - v[3];
      double vs2 = v[0] - v[1] - v[2] + v[3];
      double vs3 = v[0] + v[1] - v[2] - v[3];
      for (sp = 0; sp < nspin; sp++) {
        int o = sp * norb, S = o + 1, X = o + 2, Y = o + 3, Z = o + 4;
#define HR(r, c) h[((r) * nb + (c)) * 2]
        HR(S, S) += vs0; HR(X, X) += vs0; HR(Y, Y) += vs0; HR(Z, Z) += vs0;
        HR(S, X) += sgn * vs1; HR(X, S) += sgn * vs1; HR(Y, Z) += vs1; HR(Z, Y) += vs1;
        HR(S, Y) += sgn * vs2; HR(Y, S) += sgn * vs2; HR(X, Z) += vs2; HR(Z, X) += vs2;
        HR(S, Z) += sgn * vs3; HR(Z, S) += sgn * vs3; HR(X, Y) += vs3; HR(Y, X) += vs3;
#undef HR
      }
    }
    if (md->include_strain)
      for (i = 0; i < nb; i++) h[(i * nb + i) * 2] += shiftsum;
    /* bonds: blocks (stored by the cation) and diagonal corrections */
    for (n = 0; n < 4; n++) {
      int b = nbr[a * 4 + n];
      if (b < 0) continue;
      long sn = atom_slot[b];
      int tn = g->type[sn];
      int c_ = cat ? tthis : tn, a_ = cat ? tn : tthis;
      if (!md->par_ok[c_ * NS + a_]) continue;
      const double *pp = md->par + ((size_t)c_ * NS + a_) * ORC_NPAR;
      /* a0 of the pair: parmat[this][nbr] (h_cvectr_mult.c:1026) */
      /* (parmat is symmetrised in param_init, mat3d.c:287-306) */
      double a0 = pp[31];
      double nnv[3], nnv0[3], blk[100], ediag[10];
      for (i = 0; i < norb; i++) ediag[i] = h[(i * nb + i) * 2];
      bond_vectors(g, s, sn, n, a0, nnv, nnv0);
      bond_block(norb, cat, nnv, nnv0, pp, md->include_strain, a0, blk, ediag);
      for (i = 0; i < nb; i++) h[(i * nb + i) * 2] = ediag[i % norb];
      if (cat) memcpy(blocks + ((size_t)a * 4 + n) * norb * norb, blk,
                      sizeof(double) * norb * norb);
    }
  }
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Bloch phase of a bond that crosses the periodic boundary
 * (geo_struct::phasePeriodic, geo_struct.h:811-826). */
static void bloch(const signed char *w, const double *k, double *cr, double *ci) {
  double ph = 0.0;
  if (!k || (!w[0] && !w[1] && !w[2])) { *cr = 1.0; *ci = 0.0; return; }
  ph = w[0] * k[0] + w[1] * k[1] + w[2] * k[2];
  ph = -M_PI * (ph - 2 * (int)(0.5 * ph));
  *cr = cos(ph);
  *ci = sin(ph);
}

/* reverse slot: the n' of atom b whose neighbour is a across the opposite
 * periodic image */
static int reverse_slot(const int *nbr, const signed char *wrap, long a, int n,
                        long b) {
  int q;
  for (q = 0; q < 4; q++) {
    if (nbr[b * 4 + q] != a) continue;
    if (!wrap) return q;
    const signed char *w1 = wrap + (a * 4 + n) * 3, *w2 = wrap + (b * 4 + q) * 3;
    if (w1[0] == -w2[0] && w1[1] == -w2[1] && w1[2] == -w2[2]) return q;
  }
  return -1;
}

/* y = (H - shift) x over the stored form (Hmult_spds_col_stored,
 * Hmult_stored.c:73-172, Hv_stored_20_Hzb Hmult_stored.c:176-607): on-site
 * block, then every bond applied in both directions. */
void orc_hx(int norb, int nspin, long natoms, const int *atom_slot,
            const int *nbr, const signed char *wrap, const double *kvec, const double *onsite,
            const double *blocks, double shift, const double *x, double *y) {
  const int nb = norb * nspin;
  long a;
#pragma omp parallel for schedule(static)
  for (a = 0; a < natoms; a++) {
    const double *h = onsite + (size_t)a * nb * nb * 2;
    const double *xa = x + (size_t)a * nb * 2;
    double *ya = y + (size_t)a * nb * 2;
    int i, j, n, sp, cat;
    for (i = 0; i < nb; i++) {
      double re = 0.0, im = 0.0;
      for (j = 0; j < nb; j++) {
        double hr = h[(i * nb + j) * 2], hi = h[(i * nb + j) * 2 + 1];
        re += hr * xa[j * 2] - hi * xa[j * 2 + 1];
        im += hr * xa[j * 2 + 1] + hi * xa[j * 2];
      }
      ya[i * 2] = re - shift * xa[i * 2];
      ya[i * 2 + 1] = im - shift * xa[i * 2 + 1];
    }
    cat = (atom_slot[a] % 8) < 4; /* cation sites hold the bond blocks */
    for (n = 0; n < 4; n++) {
      long b = nbr[a * 4 + n];
      if (b < 0) continue;
      const double *xb = x + (size_t)b * nb * 2;
      double cr, ci;
      bloch(wrap ? wrap + (a * 4 + n) * 3 : NULL, kvec, &cr, &ci);
      /* H[a][b] = phase(b -> a) * block, with phase(b->a) = conj(phase(a->b)) */
      ci = -ci;
      const double *M;
      int q = -1;
      if (cat == 1) M = blocks + ((size_t)a * 4 + n) * norb * norb;
      else {
        q = reverse_slot(nbr, wrap, a, n, b);
        M = blocks + ((size_t)b * 4 + q) * norb * norb;
      }
      for (sp = 0; sp < nspin; sp++)
        for (i = 0; i < norb; i++) {
          double re = 0.0, im = 0.0;
          for (j = 0; j < norb; j++) {
            double v = (cat == 1) ? M[i * norb + j] : M[j * norb + i];
            re += v * xb[(sp * norb + j) * 2];
            im += v * xb[(sp * norb + j) * 2 + 1];
          }
          ya[(sp * norb + i) * 2] += cr * re - ci * im;
          ya[(sp * norb + i) * 2 + 1] += cr * im + ci * re;
        }
    }
  }
}

void orc_dense(int norb, int nspin, long natoms, const int *atom_slot,
               const int *nbr, const signed char *wrap, const double *kvec, const double *onsite,
               const double *blocks, double *h) {
  const long nb = norb * nspin, N = natoms * nb;
  double *x = (double *)calloc((size_t)N * 2, sizeof(double));
  double *y = (double *)malloc(sizeof(double) * N * 2);
  long col, r;
  for (col = 0; col < N; col++) {
    x[col * 2] = 1.0;
    orc_hx(norb, nspin, natoms, atom_slot, nbr, wrap, kvec, onsite, blocks, 0.0,
           x, y);
    for (r = 0; r < N; r++) {
      h[(r * N + col) * 2] = y[r * 2];
      h[(r * N + col) * 2 + 1] = y[r * 2 + 1];
    }
    x[col * 2] = 0.0;
  }
  free(x);
  free(y);
}

void orc_ham_matvec(void *ham, const double *x, double *y) {
  const orc_ham *H = (const orc_ham *)ham;
  orc_hx(H->norb, H->nspin, H->natoms, H->atom_slot, H->nbr, H->wrap, H->kvec, H->onsite,
         H->blocks, H->shift, x, y);
}

/* ------------------------------------------------------------------------ */
/* Tridiagonal eigenvalues by Sturm-sequence bisection.  The reference calls
 * LAPACK dstebz (RANGE='V', ORDER='E', abstol=1e-13; lanczos.c:793-811); this
 * restates its result: every eigenvalue in (vl, vu], ascending. */
static int sturm_count(int n, const double *d, const double *e2, double x) {
  /* number of eigenvalues < x */
  int cnt = 0, i;
  double q = d[0] - x;
  const double tiny = 1e-300;
  if (q < 0) cnt++;
  for (i = 1; i < n; i++) {
    if (fabs(q) < tiny) q = q < 0 ? -tiny : tiny;
    q = d[i] - x - e2[i - 1] / q;
    if (q < 0) cnt++;
  }
  return cnt;
}

int orc_tridiag_eigs(int n, const double *d, const double *e, double vl,
                     double vu, double abstol, double *w) {
  double *e2 = (double *)malloc(sizeof(double) * (n > 1 ? n - 1 : 1));
  double lo = d[0], hi = d[0];
  int i, k;
  for (i = 0; i < n - 1; i++) e2[i] = e[i] * e[i];
  for (i = 0; i < n; i++) { /* Gershgorin bounds */
    double r = (i > 0 ? fabs(e[i - 1]) : 0) + (i < n - 1 ? fabs(e[i]) : 0);
    if (d[i] - r < lo) lo = d[i] - r;
    if (d[i] + r > hi) hi = d[i] + r;
  }
  /* (vl, vu]: eigenvalues with count(<=vu) - count(<=vl) */
  int c_lo = sturm_count(n, d, e2, vl), c_hi = sturm_count(n, d, e2, vu);
  /* sturm_count counts < x; treat x exactly at an eigenvalue as negligible */
  int nf = c_hi - c_lo;
  for (k = 0; k < nf; k++) {
    int idx = c_lo + k; /* find the idx-th eigenvalue (0-based) */
    double a = vl > lo ? vl : lo, b = vu < hi ? vu : hi;
    int it;
    for (it = 0; it < 200; it++) {
      double mid = 0.5 * (a + b);
      double tol = abstol + 2.2e-16 * (fabs(a) > fabs(b) ? fabs(a) : fabs(b));
      if (b - a <= tol) break;
      if (sturm_count(n, d, e2, mid) > idx) b = mid;
      else a = mid;
    }
    w[k] = 0.5 * (a + b);
  }
  free(e2);
  return nf;
}

/* solve_rtridiag_ii (lanczos.c:249-308): T x = y, T symmetric tridiagonal
 * with diagonal d and off-diagonal e (e[j-1] couples j-1 and j). */
static void solve_tri(int m, const double *d, const double *e, const double *y,
                      double *x, double *g) {
  double piv = d[0];
  int j;
  x[0] = y[0] / piv;
  for (j = 1; j < m; j++) {
    g[j] = e[j - 1] / piv;
    piv = d[j] - e[j - 1] * g[j];
    x[j] = (y[j] - e[j - 1] * x[j - 1]) / piv;
  }
  for (j = m - 1; 0 < j; --j) x[j - 1] -= g[j] * x[j];
}

/* originalInverseIteration (lanczos.c:378-418) on the leading m x m block:
 * 20 solves with T - (lambda + 1e-8), normalising each time.  x: out. */
static void inverse_iteration(int m, const double *d, const double *e,
                              double lambda, double *y, double *x) {
  double *ds = (double *)malloc(sizeof(double) * m);
  double *g = (double *)malloc(sizeof(double) * m);
  double nrm = 0.0;
  int i, it;
  for (i = 0; i < m; i++) ds[i] = d[i] - (lambda + 1e-8);
  for (i = 0; i < m; i++) nrm += y[i] * y[i];
  for (i = 0; i < m; i++) y[i] /= sqrt(nrm);
  for (it = 0; it < 20; it++) {
    solve_tri(m, ds, e, y, x, g);
    nrm = 0.0;
    for (i = 0; i < m; i++) nrm += x[i] * x[i];
    for (i = 0; i < m; i++) y[i] = x[i] / sqrt(nrm);
  }
  for (i = 0; i < m; i++) x[i] = y[i];
  free(ds);
  free(g);
}

/* uniform [0,1] start for inverse iteration (the reference draws
 * rand()/RAND_MAX; the converged vector does not depend on it) */
static double urand(unsigned long long *s) {
  *s = *s * 6364136223846793005ULL + 1442695040888963407ULL;
  return (double)(*s >> 11) / 9007199254740992.0;
}

/* find_converged_eigval, method 2 (lanczos.c:764-996) */
static void find_converged(int it, const double *al, const double *be,
                           double emin, double emax, double tol, double res,
                           double *conv, int *conv_it, int *nconv,
                           unsigned long long *rng) {
  double *ev = (double *)malloc(sizeof(double) * it);
  double *yy = (double *)malloc(sizeof(double) * it);
  double *xx = (double *)malloc(sizeof(double) * it);
  int ne = orc_tridiag_eigs(it, al, be, emin, emax, 1e-13, ev);
  int i, j, k;
  for (i = 0; i < ne; i++) {
    if (i > 0 && fabs(ev[i - 1] - ev[i]) < fabs(1e-80 + ev[i]) * res) continue;
    int done = 0;
    for (j = 0; j < *nconv; j++)
      if (fabs(conv[j] - ev[i]) < res) done = 1;
    if (done) continue;
    for (k = 0; k < it; k++) yy[k] = urand(rng);
    inverse_iteration(it, al, be, ev[i], yy, xx);
    int flag = 1;
    for (k = it - 2; k < it; k++)
      if (k >= 0 && fabs(xx[k]) > tol) flag = 0;
    if (flag) {
      conv[*nconv] = ev[i];
      conv_it[*nconv] = it;
      (*nconv)++;
    }
  }
  free(ev);
  free(yy);
  free(xx);
}

/* single_lanczos_iteration (lanczos.c:421-757), default variant */
static void lanczos_step(orc_matvec_fn mv, void *ctx, long n, double *r,
                         double *q, double *qp, double beta_prev, double *alpha,
                         double *beta) {
  long j;
  double inv = 1.0 / beta_prev, al = 0.0, bsq = 0.0;
  for (j = 0; j < 2 * n; j++) q[j] = r[j] * inv;
  mv(ctx, q, r);
  for (j = 0; j < n; j++) al += r[2 * j] * q[2 * j] + r[2 * j + 1] * q[2 * j + 1];
  for (j = 0; j < 2 * n; j++) {
    r[j] -= al * q[j] + beta_prev * qp[j];
    bsq += r[j] * r[j];
    qp[j] = q[j];
  }
  *alpha = al;
  *beta = sqrt(bsq);
}

static void sort2(double *v, int *w, int n) {
  int i, j;
  for (i = 1; i < n; i++)
    for (j = i; j > 0 && v[j] < v[j - 1]; j--) {
      double t = v[j]; v[j] = v[j - 1]; v[j - 1] = t;
      int u = w[j]; w[j] = w[j - 1]; w[j - 1] = u;
    }
}

int orc_eigensolve_lanczos(orc_matvec_fn mv, void *ctx, long n, const double *r0,
                           const orc_lanczos_opts *o, double *evals,
                           int *conv_it, int *iterations, double *evecs,
                           double *alpha, double *beta) {
  double *r = (double *)malloc(sizeof(double) * 2 * n);
  double *q = (double *)malloc(sizeof(double) * 2 * n);
  double *qp = (double *)calloc(2 * n, sizeof(double));
  double *c1 = (double *)malloc(sizeof(double) * o->imax);
  double *c2 = (double *)malloc(sizeof(double) * o->imax);
  int *i1 = (int *)malloc(sizeof(int) * o->imax);
  int *i2 = (int *)malloc(sizeof(int) * o->imax);
  int n1 = 0, n2 = 0, it = 0, skip = 0, k;
  long j;
  const double res = 100.0 * o->tolerance;
  unsigned long long rng = o->seed * 2654435761ULL + 12345ULL;
  double nrm = 0.0, bprev;
  /* lanczos_initialize (eigsys3d_par.c:113-215): normalised start */
  for (j = 0; j < 2 * n; j++) nrm += r0[j] * r0[j];
  nrm = sqrt(nrm);
  for (j = 0; j < 2 * n; j++) r[j] = r0[j] / nrm;
  /* lanczos_tridiagonal (lanczos.c:1000-1278) */
  nrm = 0.0;
  for (j = 0; j < 2 * n; j++) nrm += r[j] * r[j];
  bprev = sqrt(nrm);
  for (;;) {
    double al, be;
    lanczos_step(mv, ctx, n, r, q, qp, bprev, &al, &be);
    alpha[it] = al;
    beta[it] = be;
    bprev = be;
    it++;
    skip++;
    if (o->conv_start < it && o->conv_skip <= skip) {
      skip = 0;
      if (o->req1 > 0 && n1 <= o->req1)
        find_converged(it, alpha, beta, o->emin1, o->emax1, o->tolerance, res,
                       c1, i1, &n1, &rng);
      if (o->req2 > 0 && n2 <= o->req2)
        find_converged(it, alpha, beta, o->emin2, o->emax2, o->tolerance, res,
                       c2, i2, &n2, &rng);
    }
    if (!((it + 1 < o->imax) && (n1 < o->req1 || n2 < o->req2))) break;
  }
  int ne = n1 + n2;
  for (k = 0; k < n1; k++) { evals[k] = c1[k]; conv_it[k] = i1[k]; }
  for (k = 0; k < n2; k++) { evals[n1 + k] = c2[k]; conv_it[n1 + k] = i2[k]; }
  sort2(evals, conv_it, ne);
  *iterations = it;
  if (evecs && ne > 0) { /* eigenvectorsLanczos, method 3 (lanczos.c:1364-1689) */
    int maxit = 0;
    double *xm = (double *)calloc((size_t)ne * it, sizeof(double));
    double *yy = (double *)malloc(sizeof(double) * it);
    for (k = 0; k < ne; k++) {
      int req = conv_it[k], t;
      if (req > maxit) maxit = req;
      for (t = 0; t < req; t++) yy[t] = urand(&rng);
      inverse_iteration(req, alpha, beta, evals[k], yy, xm + (size_t)k * it);
    }
    memset(evecs, 0, sizeof(double) * 2 * n * ne);
    nrm = 0.0;
    for (j = 0; j < 2 * n; j++) r[j] = r0[j];
    for (j = 0; j < 2 * n; j++) nrm += r[j] * r[j];
    nrm = sqrt(nrm);
    for (j = 0; j < 2 * n; j++) r[j] /= nrm;
    memset(qp, 0, sizeof(double) * 2 * n);
    nrm = 0.0;
    for (j = 0; j < 2 * n; j++) nrm += r[j] * r[j];
    bprev = sqrt(nrm);
    for (int t = 0; t < maxit; t++) {
      double al, be;
      lanczos_step(mv, ctx, n, r, q, qp, bprev, &al, &be);
      bprev = be;
      for (k = 0; k < ne; k++) {
        if (t >= conv_it[k]) continue;
        double c = xm[(size_t)k * it + t];
        double *v = evecs + (size_t)k * 2 * n;
        for (j = 0; j < 2 * n; j++) v[j] += c * q[j];
      }
    }
    free(xm);
    free(yy);
  }
  free(r); free(q); free(qp); free(c1); free(c2); free(i1); free(i2);
  return ne;
}

/* ------------------------------------------------------------------------ */
/* Keating valence force field, StrainModel = VFF_keating (no anharmonic
 * corrections, no lattice-constant minimisation).
 *
 * calc_estrain (base/strain3d.c:1361-2080): for every atom m and its
 * neighbours n, p (all present), nnv = a_latt*eta + (u_nbr - u_m) with eta
 * the neighbour's cell offset plus the in-cell position difference, nnv0 =
 * alat(m, n)*eta.  Bond stretching 0.5*alpha/d0^2*(d^2 - d0^2)^2 per atom and
 * bond (each bond thus counted from both ends), bond bending
 * sqrt(beta_n beta_p)/sqrt(d0_p^2 d0_n^2)*(nnv_n.nnv_p - nnv0_n.nnv0_p)^2 per
 * atom and neighbour pair; the gradient as the reference accumulates it. */
double orc_vff_energy(const orc_geom *g, long natoms, const int *atom_slot, const int *nbr,
                      int ns, const double *vff, const double *u, double *grad) {
  double bld = 0.0, bbd = 0.0;
  long a;
  int n, p, q;
  memset(grad, 0, sizeof(double) * 3 * natoms);
  for (a = 0; a < natoms; a++) {
    const long s = atom_slot[a];
    const int m = (int)(s % 8);
    const int tm = g->type[s];
    double nnv[4][3], nnv0[4][3], alpha[4], beta[4];
    int stat[4], nb[4];
    for (n = 0; n < 4; n++) {
      nb[n] = nbr[a * 4 + n];
      stat[n] = nb[n] >= 0;
      if (!stat[n]) continue;
      const long sn = atom_slot[nb[n]];
      const int tn = g->type[sn];
      const int mn = nnmap[m][n][3];
      const double *vp = vff + ((long)tm * ns + tn) * 3;
      const double alat = vp[0];
      for (q = 0; q < 3; q++) {
        const double disp = u[nb[n] * 3 + q] - u[a * 3 + q];
        const double r1 = (double)nnmap[m][n][q] + (pin[mn][q] - pin[m][q]);
        nnv[n][q] = g->lattice[q] * r1 + disp;
        nnv0[n][q] = alat * r1;
      }
      alpha[n] = vp[1];
      beta[n] = vp[2];
    }
    for (n = 0; n < 4; n++) {
      if (!stat[n]) continue;
      const double dssq = nnv[n][0] * nnv[n][0] + nnv[n][1] * nnv[n][1] + nnv[n][2] * nnv[n][2];
      const double d0sq =
          nnv0[n][0] * nnv0[n][0] + nnv0[n][1] * nnv0[n][1] + nnv0[n][2] * nnv0[n][2];
      const double bldc = 0.5 * alpha[n] / d0sq;
      const double bldl = dssq - d0sq;
      bld += bldc * bldl * bldl;
      const double r1 = 4 * bldc * bldl;
      for (q = 0; q < 3; q++) grad[a * 3 + q] -= r1 * nnv[n][q];
      for (p = n + 1; p < 4; p++) {
        if (!stat[p]) continue;
        const double d0dot =
            nnv0[n][0] * nnv0[p][0] + nnv0[n][1] * nnv0[p][1] + nnv0[n][2] * nnv0[p][2];
        const double dsdot = nnv[n][0] * nnv[p][0] + nnv[n][1] * nnv[p][1] + nnv[n][2] * nnv[p][2];
        const double den =
            nnv0[p][0] * nnv0[p][0] + nnv0[p][1] * nnv0[p][1] + nnv0[p][2] * nnv0[p][2];
        const double Beta = sqrt(beta[n] * beta[p]);
        const double bbdc = Beta / sqrt(den * d0sq);
        const double bbdl = dsdot - d0dot;
        const double bb_mul = bbdc * bbdl;
        bbd += bb_mul * bbdl;
        const double bb2 = 2 * bb_mul;
        for (q = 0; q < 3; q++) {
          grad[nb[n] * 3 + q] += nnv[p][q] * bb2;
          grad[a * 3 + q] -= nnv[p][q] * bb2;
        }
        for (q = 0; q < 3; q++) {
          grad[nb[p] * 3 + q] += nnv[n][q] * bb2;
          grad[a * 3 + q] -= nnv[n][q] * bb2;
        }
      }
    }
  }
  return bld + bbd;
}

/* Which atoms move under the reference's Keating boundary conditions
 * (calc_estrain_macopt, base/strain3d.c:846-1000, 1242-1340): 0 AllFree,
 * 1 FixOne (the first atom fixed), 2 FixSurfaceAll (surface atoms fixed),
 * 3 FixZmin (atoms of the two lowest cell layers fixed, isInZ_min: bit 64 of
 * FindSurfaceAtoms, geo_struct.c:1374-1410), 4 FixInterior (only surface
 * atoms move). */
void orc_vff_free_mask(const orc_geom *g, long natoms, const int *atom_slot,
                       const unsigned char *surface, int bc, unsigned char *free_mask) {
  long a;
  for (a = 0; a < natoms; a++) {
    const long cell = atom_slot[a] / 8;
    const int k = (int)(cell % g->nz);
    int f = 1;
    if (bc == 1) f = a != 0;
    else if (bc == 2) f = !surface[a];
    else if (bc == 3) f = k > 1;
    else if (bc == 4) f = surface[a] != 0;
    free_mask[a] = (unsigned char)f;
  }
}

/* macoptII_par / maclinminII_par / macprodII_par / macopt_restart
 * (NEMO_3D/eigen/src/macopt_par.c:121-475, macopt.c:418-520) with the
 * defaults of macopt_defaults (rich = 1, linmin g1 2.0, g2 1.25, g3 0.5,
 * 20 line-search steps, lastx 0.01, grad_tol_tiny 1e-28, step_tol_tiny 0)
 * driving the Keating gradient of the free atoms (calc_estrain_macopt).
 * u: [natoms*3] displacements, updated in place.  Returns the iteration at
 * which it stopped; *energy is the energy at the final u. */
typedef struct {
  const orc_geom *g;
  long natoms;
  const int *atom_slot, *nbr;
  int ns;
  const double *vff;
  const unsigned char *free_mask;
  double *tmp;
  double value;
} vff_ctx;

static void vff_dfunc(vff_ctx *c, const double *u, double *xi) {
  long i;
  c->value = orc_vff_energy(c->g, c->natoms, c->atom_slot, c->nbr, c->ns, c->vff, u, c->tmp);
  for (i = 0; i < 3 * c->natoms; i++) xi[i] = c->free_mask[i / 3] ? c->tmp[i] : 0.0;
}

int orc_vff_relax(const orc_geom *g, long natoms, const int *atom_slot, const int *nbr,
                  const unsigned char *surface, int ns, const double *vff, int bc, int itmax,
                  double tol, int end_if_small_step, double *u, double *energy) {
  const long n = 3 * natoms;
  double *gv = (double *)calloc(n, sizeof(double)), *h = (double *)calloc(n, sizeof(double));
  double *xi = (double *)calloc(n, sizeof(double)), *pt = (double *)calloc(n, sizeof(double));
  double *gx = (double *)calloc(n, sizeof(double)), *gy = (double *)calloc(n, sizeof(double));
  unsigned char *fm = (unsigned char *)malloc(natoms);
  vff_ctx c = {g, natoms, atom_slot, nbr, ns, vff, fm, (double *)calloc(n, sizeof(double)), 0.0};
  const int end_if_small_grad = 1 - end_if_small_step;
  int rich = 1, restart = 0, its;
  double lastx = 0.01, gtyp = 0.0;
  long j;
  orc_vff_free_mask(g, natoms, atom_slot, surface, bc, fm);
  vff_dfunc(&c, u, xi);
  for (j = 0; j < n; j++) { /* macopt_restart(a, 1) */
    gv[j] = -xi[j];
    xi[j] = h[j] = gv[j];
  }
  for (its = 1; its <= itmax; ++its) {
    double gg = 0.0;
    for (j = 0; j < n; j++) gg += gv[j] * gv[j];
    gtyp = sqrt(gg / (double)n);
    if ((end_if_small_grad && gg <= tol) || gg <= 1e-28) break;
    /* maclinmin */
    double x = lastx / gtyp, y = 0.0, s, t, m, step = 0.0, *ga = gx, *gb = gy, *sw;
    int lits = 1;
#define MACPROD(yy, gout, res)                                   \
    do {                                                         \
      for (j = 0; j < n; j++) pt[j] = u[j] + (yy) * xi[j];       \
      vff_dfunc(&c, pt, gout);                                   \
      res = 0.0;                                                 \
      for (j = 0; j < n; j++) res += gout[j] * xi[j];            \
    } while (0)
    MACPROD(x, ga, s);
    if (s < 0) {
      do {
        y = x * 2.0;
        MACPROD(y, gb, t);
        if (t >= 0.0) break;
        x = y; s = t; sw = ga; ga = gb; gb = sw;
        ++lits;
      } while (lits <= 20);
    } else if (s > 0) {
      do {
        y = x * 0.5;
        MACPROD(y, gb, t);
        if (t <= 0.0) break;
        x = y; s = t; sw = ga; ga = gb; gb = sw;
        ++lits;
      } while (lits <= 20);
    } else {
      t = 1.0;
      y = x;
    }
    if (lits > 20) {
      double tmpd;
      MACPROD(0.0, gb, tmpd);
      if (tmpd > 0 && rich == 0) rich = 1;
      if (tmpd > 0) restart = 1;
    }
#undef MACPROD
    if (s < 0.0) s = -s;
    if (t < 0.0) t = -t;
    m = s + t;
    s /= m;
    t /= m;
    m = s * y + t * x;
    for (j = 0; j < n; j++) {
      const double tmpd = m * xi[j];
      u[j] += tmpd;
      step += fabs(tmpd);
      xi[j] = s * gb[j] + t * ga[j];
    }
    lastx = m * 1.25 * gtyp;
    step /= (double)n;
    if (((end_if_small_step && step <= tol) || step <= 0.0) && restart == 0) break;
    if (rich || restart) vff_dfunc(&c, u, xi);
    if (restart) { /* macopt_restart(a, 0) */
      lastx = 0.01;
      for (j = 0; j < n; j++) {
        if (restart != 2) gv[j] = -xi[j];
        xi[j] = h[j] = gv[j];
      }
      restart = 0;
    } else {
      double dgg = 0.0, gam, tmpd = 0.0;
      for (j = 0; j < n; j++) dgg += (xi[j] + gv[j]) * xi[j];
      gam = dgg / gg;
      for (j = 0; j < n; j++) {
        gv[j] = -xi[j];
        xi[j] = h[j] = gv[j] + gam * h[j];
        tmpd -= xi[j] * gv[j];
      }
      if (tmpd > 0.0) {
        rich = 1;
        restart = 2;
        lastx = 0.01;
        for (j = 0; j < n; j++) xi[j] = h[j] = gv[j];
        restart = 0;
      }
    }
  }
  *energy = orc_vff_energy(g, natoms, atom_slot, nbr, ns, vff, u, c.tmp);
  free(gv); free(h); free(xi); free(pt); free(gx); free(gy); free(fm); free(c.tmp);
  return its > itmax ? itmax : its;
}
