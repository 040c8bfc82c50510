// Hamiltonian assembly on the GPU.
//
// k_bonds: one thread per (atom, neighbour slot).  Restates
//   H_DiagStrainCorr_OffDiag_Wrapper  nemo3d/src/base/h_cvectr_mult.c:1007-1126
//   getRelativePosVec                 nemo3d/src/base/geo_struct.c:2224-2297
//   strain_corr_prep                  nemo3d/src/ham/mb_ham_spds_micro.c:2848-2982
//   h3d_offdiag_diag_corr + get_X_Y   nemo3d/src/ham/mb_ham_spds_micro.c:597-1451,
//                                     mb_ham_spds_VoffdEdiag_constructors.h
// writing the bond block (stored once, by the cation) and this atom's
// strain-induced diagonal correction for the bond.
// k_onsite: one thread per atom.  Restates
//   H_Diag_Wrapper (bond-averaged parameters, strain shift)
//                                     nemo3d/src/base/h_cvectr_mult.c:841-1005
//   h3d_diag + spin-orbit table       nemo3d/src/ham/mb_ham_spds_micro.c:1453-1505,
//                                     mb_ham_spds_so.h
//   h3d_diag_dangling_bond_shift_zincblende
//                                     nemo3d/src/ham/mb_ham_spds_micro.c:1910-2150
//   HamZincBlende::setDiag            nemo3d/src/base/HamZincBlende.c:161-230
#include <cmath>

#include "reduce.cuh"
#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

// orbital order s*, s, px, py, pz, dxy, dyz, dzx, dx2-y2, dz2
// (mb_ham_spds_micro.h:97-116); orbital kinds: 0 s*, 1 s, 2 p, 3 d
__device__ __forceinline__ int kind_of(int o) { return o == 0 ? 0 : o == 1 ? 1 : o < 5 ? 2 : 3; }
__device__ __forceinline__ int ang_of(int o) { return o < 2 ? 0 : o < 5 ? 1 : 2; }

// Integral parameter indices (sigma, pi, delta) of an (anion kind, cation
// kind) pair and its strain-correction coefficient index
// (mb_ham_spds_micro.c:58-146).
static __constant__ int8_t c_vidx[4][4][3] = {
    // anion s*      with cation s*, s, p, d
    {{11, -1, -1}, {12, -1, -1}, {16, -1, -1}, {20, -1, -1}},
    // anion s
    {{13, -1, -1}, {10, -1, -1}, {14, -1, -1}, {18, -1, -1}},
    // anion p
    {{17, -1, -1}, {15, -1, -1}, {22, 23, -1}, {24, 26, -1}},
    // anion d
    {{21, -1, -1}, {19, -1, -1}, {25, 27, -1}, {28, 29, 30}}};
static __constant__ int8_t c_cidx[4][4] = {
    {18, 19, 23, 27}, {20, 17, 21, 25}, {24, 22, 29, 30}, {28, 26, 31, 32}};
// on-site energy index by kind for anion / cation (diag_map_set)
static __constant__ int8_t c_eidx[2][4] = {{4, 0, 1, 6}, {5, 2, 3, 7}};
// two-centre integral index -> strain exponent index (E_const_prep)
static __constant__ int8_t c_eta_of[21] = {
    eta_sss, eta_ststs, eta_ssts, eta_ssts, eta_sps, eta_sps, eta_stps,
    eta_stps, eta_sds, eta_sds, eta_stds, eta_stds, eta_pps, eta_ppp,
    eta_pds, eta_pds, eta_pdp, eta_pdp, eta_dds, eta_ddp, eta_ddd};

// Slater-Koster element for orbital a on the first atom, b on the second,
// ang(a) <= ang(b), cosines d[] from first to second (Slater & Koster 1954,
// Table I, written with index permutations).
__device__ double sk_ordered(int a, int b, const double d[3], double Vs, double Vp,
                             double Vd) {
  const int la = ang_of(a), lb = ang_of(b);
  const double s3 = kSqr3;
  if (lb == 0) return Vs;                          // s/s* - s/s*
  if (la == 0 && lb == 1) return d[b - 2] * Vs;    // s - p
  const double l2 = d[0] * d[0], m2 = d[1] * d[1], n2 = d[2] * d[2];
  const double q = n2 - 0.5 * (l2 + m2);           // 3z2-r2 angular factor
  const double lm2 = l2 - m2;
  // t2g orbitals dxy, dyz, dzx as index pairs (u, v)
  const int tu[3] = {0, 1, 2}, tv[3] = {1, 2, 0};
  if (la == 0) {                                    // s - d
    if (b < 8) return s3 * d[tu[b - 5]] * d[tv[b - 5]] * Vs;
    return (b == 8 ? 0.5 * s3 * lm2 : q) * Vs;
  }
  if (la == 1 && lb == 1) {                         // p - p
    const double di = d[a - 2], dj = d[b - 2];
    return a == b ? di * di * Vs + (1.0 - di * di) * Vp : di * dj * Vs - di * dj * Vp;
  }
  if (la == 1) {                                    // p - d
    const int i = a - 2;
    const double di = d[i];
    if (b < 8) {
      const int u = tu[b - 5], v = tv[b - 5];
      if (i == u) return s3 * d[u] * d[u] * d[v] * Vs + d[v] * (1.0 - 2.0 * d[u] * d[u]) * Vp;
      if (i == v) return s3 * d[v] * d[v] * d[u] * Vs + d[u] * (1.0 - 2.0 * d[v] * d[v]) * Vp;
      const double p3 = d[0] * d[1] * d[2];
      return s3 * p3 * Vs - 2.0 * p3 * Vp;
    }
    if (b == 8) {
      if (i == 0) return 0.5 * s3 * di * lm2 * Vs + di * (1.0 - lm2) * Vp;
      if (i == 1) return 0.5 * s3 * di * lm2 * Vs - di * (1.0 + lm2) * Vp;
      return 0.5 * s3 * di * lm2 * Vs - di * lm2 * Vp;
    }
    if (i < 2) return di * q * Vs - s3 * di * n2 * Vp;
    return di * q * Vs + s3 * di * (l2 + m2) * Vp;
  }
  // d - d (symmetric in a, b)
  int x = a < b ? a : b, y = a < b ? b : a;
  if (y < 8) {                                      // t2g - t2g
    const int u1 = tu[x - 5], v1 = tv[x - 5];
    if (x == y) {
      const int w = 3 - u1 - v1;
      const double pu = d[u1] * d[u1], pv = d[v1] * d[v1];
      return 3.0 * pu * pv * Vs + (pu + pv - 4.0 * pu * pv) * Vp + (d[w] * d[w] + pu * pv) * Vd;
    }
    const int u2 = tu[y - 5], v2 = tv[y - 5];
    const int sh = (u1 == u2 || u1 == v2) ? u1 : v1;  // shared index
    const int p = (u1 == sh) ? v1 : u1, r = (u2 == sh) ? v2 : u2;
    const double ds2 = d[sh] * d[sh], pr = d[p] * d[r];
    return 3.0 * pr * ds2 * Vs + pr * (1.0 - 4.0 * ds2) * Vp + pr * (ds2 - 1.0) * Vd;
  }
  if (x < 8) {                                      // t2g - eg
    const double l = d[0], m = d[1], n = d[2];
    if (y == 8) {
      if (x == 5) return 1.5 * l * m * lm2 * Vs - 2.0 * l * m * lm2 * Vp + 0.5 * l * m * lm2 * Vd;
      if (x == 6) return 1.5 * m * n * lm2 * Vs - m * n * (1.0 + 2.0 * lm2) * Vp + m * n * (1.0 + 0.5 * lm2) * Vd;
      return 1.5 * n * l * lm2 * Vs + n * l * (1.0 - 2.0 * lm2) * Vp - n * l * (1.0 - 0.5 * lm2) * Vd;
    }
    if (x == 5) return s3 * l * m * q * Vs - 2.0 * s3 * l * m * n2 * Vp + 0.5 * s3 * l * m * (1.0 + n2) * Vd;
    const double uv = (x == 6) ? m * n : l * n;
    return s3 * uv * q * Vs + s3 * uv * (l2 + m2 - n2) * Vp - 0.5 * s3 * uv * (l2 + m2) * Vd;
  }
  if (x == 8 && y == 8) return 0.75 * lm2 * lm2 * Vs + (l2 + m2 - lm2 * lm2) * Vp + (n2 + 0.25 * lm2 * lm2) * Vd;
  if (x == 8) return 0.5 * s3 * lm2 * q * Vs - s3 * n2 * lm2 * Vp + 0.25 * s3 * (1.0 + n2) * lm2 * Vd;
  return q * q * Vs + 3.0 * n2 * (l2 + m2) * Vp + 0.75 * (l2 + m2) * (l2 + m2) * Vd;
}

// <anion orbital a | H | cation orbital c>, cosines from anion to cation,
// integrals from V (parity (-1)^(la+lc) when the anion orbital has higher l)
__device__ __forceinline__ double sk_bond(int a, int c, const double d[3], const double *V) {
  const int ka = kind_of(a), kc = kind_of(c);
  const int i0 = c_vidx[ka][kc][0], i1 = c_vidx[ka][kc][1], i2 = c_vidx[ka][kc][2];
  const double Vs = V[i0], Vp = i1 >= 0 ? V[i1] : 0.0, Vd = i2 >= 0 ? V[i2] : 0.0;
  const int la = ang_of(a), lc = ang_of(c);
  if (la <= lc) return sk_ordered(a, c, d, Vs, Vp, Vd);
  const double e = sk_ordered(c, a, d, Vs, Vp, Vd);
  return ((la + lc) & 1) ? -e : e;
}

// One bond seen from its cation (site s, neighbour slot n) to the anion at
// site sn: direction cosines of the strained (d) and unstrained (d0) bond,
// anion -> cation, and the two-centre integrals with Harrison's scaling
// (d0/d)^eta in Vsc[10..30].  Shared by the stored assembly and the
// recompute H*x, so both produce the same numbers.
__device__ __forceinline__ void bond_frame(long s, int n, long sn, const double *P,
                                           const double *dsp, double lx, double ly,
                                           double lz, int include_strain, double d[3],
                                           double d0[3], double *Vsc) {
  const double *S = P + kNPV;
  const int m = int(s & 7), mn = c_nnmap[m][n][3];
  const double a0 = P[pA0];
  const double lat[3] = {lx, ly, lz};
  double v[3], v0[3];
  for (int k = 0; k < 3; k++) {
    const double norm = c_nnmap[m][n][k] + c_site_pos[mn][k] - c_site_pos[m][k];
    v0[k] = a0 * norm;
    v[k] = lat[k] * norm;
    if (dsp) v[k] = v[k] + dsp[sn * 3 + k] - dsp[s * 3 + k];
    v[k] = -v[k];  // seen from the cation: flip to anion -> cation
    v0[k] = -v0[k];
  }
  const double r0 = sqrt(v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2]);
  const double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int k = 0; k < 3; k++) {
    d0[k] = v0[k] / r0;
    d[k] = v[k] / r;
  }
  for (int k = 0; k < kNPV; k++) Vsc[k] = P[k];
  if (include_strain) {
    const double brat = (0.25 * kSqr3 * a0) / r;
    for (int k = 0; k < 21; k++) Vsc[10 + k] = P[10 + k] * pow(brat, S[c_eta_of[k]]);
  }
}

template <int NORB>
__global__ void k_bonds(long natoms, const int *atom_site, const int4 *nbr,
                        const unsigned char *type, const double *dsp, const double *par,
                        const unsigned char *par_ok, int ns, double lx, double ly,
                        double lz, int include_strain, double *blocks, double *ecorr,
                        int *status) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= natoms * 4) return;
  const long a = t >> 2;
  const int n = int(t & 3);
  double *ec = ecorr + t * NORB;
  const int4 nb4 = nbr[a];
  const int b = n == 0 ? nb4.x : n == 1 ? nb4.y : n == 2 ? nb4.z : nb4.w;
  if (b < 0) {
    for (int i = 0; i < NORB; i++) ec[i] = 0.0;
    return;
  }
  const long s = atom_site[a], sn = atom_site[b];
  const int m = int(s & 7), mn = c_nnmap[m][n][3];
  const bool cat = m < 4;
  const int tt = type[s], tn = type[sn];
  const int cs = cat ? tt : tn, as = cat ? tn : tt;
  if (cs >= ns || as >= ns || !par_ok[cs * ns + as]) {
    atomicExch(status, TBGPU_E_MATERIAL);
    for (int i = 0; i < NORB; i++) ec[i] = 0.0;
    return;
  }
  const double *P = par + (long(cs) * ns + as) * kNPAR;
  const double *S = P + kNPV;
  // the bond from its cation's side (an anion takes the cation's view of it,
  // so that both ends use the same numbers)
  double d[3], d0[3], Vsc[kNPV];
  if (cat)
    bond_frame(s, n, sn, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
  else
    bond_frame(sn, c_rev_slot[m][n], s, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
  (void)mn;
  const double cstrain = include_strain ? S[eta_const] : 0.0;
  double *blk = blocks ? blocks + (a * 4 + n) * NORB * NORB : nullptr;
  for (int i = 0; i < NORB; i++) {  // orbital of this atom
    double E = 0.0;
    for (int k = 0; k < NORB; k++) {  // orbital of the neighbour
      const int oa = cat ? k : i, oc = cat ? i : k;
      const double r1 = sk_bond(oa, oc, d, Vsc);
      if (cat && blk) blk[i * NORB + k] = r1;  // row: cation orbital
      const double r2 = sk_bond(oa, oc, d0, P);
      const int ka = kind_of(oa), kc = kind_of(oc);
      const double esum = P[c_eidx[0][ka]] + P[c_eidx[1][kc]];
      E += (r2 * r2 - r1 * r1) * cstrain / esum * S[c_cidx[ka][kc]];
    }
    ec[i] = E;
  }
}

template <int NORB, int NSPIN>
__global__ void k_onsite(long natoms, const int *atom_site, const int4 *nbr,
                         const unsigned char *surface, const unsigned char *type,
                         const double *par, const unsigned char *par_ok, int ns,
                         int include_strain, int passivate, double dangling_shift,
                         const double *ecorr, double *onsite) {
  constexpr int NB = NORB * NSPIN;
  constexpr int ONS = onsite_len(NB);
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const long s = atom_site[a];
  const int m = int(s & 7);
  const bool cat = m < 4;
  const int tt = type[s];
  const int4 nb4 = nbr[a];
  const int nbv[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
  // bond-averaged on-site parameters and strain shift
  double E[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double shift = 0.0;
  int cnt = 0;
  for (int n = 0; n < 4; n++) {
    if (nbv[n] < 0) continue;
    const int tn = type[atom_site[nbv[n]]];
    const int cs = cat ? tt : tn, as = cat ? tn : tt;
    if (cs >= ns || as >= ns || !par_ok[cs * ns + as]) continue;
    const double *P = par + (long(cs) * ns + as) * kNPAR;
    for (int k = 0; k < 10; k++) E[k] += P[k];
    if (include_strain) shift += P[kNPV + (cat ? eta_cat_shift : eta_an_shift)];
    cnt++;
  }
  double *rec = onsite + a * ONS;
  for (int k = 0; k < ONS; k++) rec[k] = 0.0;
  if (cnt == 0) return;
  shift /= cnt;
  for (int k = 0; k < 10; k++) E[k] /= cnt;
  double diag[NORB];
  for (int o = 0; o < NORB; o++) diag[o] = E[c_eidx[cat ? 1 : 0][kind_of(o)]];
  const double lambda = (NSPIN == 2) ? (cat ? E[pE_Lc] : E[pE_La]) : 0.0;
  // dangling-bond passivation: sp3 hybrids along the ideal bond directions
  double sx = 0, sy = 0, sz = 0, xy = 0, xz = 0, yz = 0, flag = 0;
  if (passivate && surface[a]) {
    const double bdir[4][3] = {{0.25, 0.25, 0.25}, {-0.25, -0.25, 0.25},
                               {0.25, -0.25, -0.25}, {-0.25, 0.25, -0.25}};
    double v[4];
    const double sh = dangling_shift * 0.25;
    for (int q = 0; q < 4; q++) v[q] = sh;
    double cosv = 0.0;
    for (int n = 0; n < 4; n++) {
      const int mn = c_nnmap[m][n][3];
      double w[3];
      for (int k = 0; k < 3; k++) w[k] = c_nnmap[m][n][k] + (c_site_pos[mn][k] - c_site_pos[m][k]);
      int ib = 0;
      cosv = w[0] * bdir[0][0] + w[1] * bdir[0][1] + w[2] * bdir[0][2];
      while (fabs(cosv) < 0.15 && ib < 3) {
        ++ib;
        cosv = w[0] * bdir[ib][0] + w[1] * bdir[ib][1] + w[2] * bdir[ib][2];
      }
      if (nbv[n] >= 0) v[ib] = 0.0;
    }
    const double sg = cosv > 0 ? 1.0 : -1.0;
    const double v0 = v[0] + v[1] + v[2] + v[3];
    const double v1 = v[0] - v[1] + v[2] - v[3];
    const double v2 = v[0] - v[1] - v[2] + v[3];
    const double v3 = v[0] + v[1] - v[2] - v[3];
    for (int o = 1; o <= 4; o++) diag[o] += v0;
    sx = sg * v1; sy = sg * v2; sz = sg * v3;
    yz = v1; xz = v2; xy = v3;
    flag = 1.0;
  }
  for (int o = 0; o < NORB; o++) diag[o] += shift;
  // strain-induced diagonal corrections, bond by bond
  for (int n = 0; n < 4; n++) {
    if (nbv[n] < 0) continue;
    const double *ec = ecorr + (a * 4 + n) * NORB;
    for (int o = 0; o < NORB; o++) diag[o] += ec[o];
  }
  for (int sp = 0; sp < NSPIN; sp++)
    for (int o = 0; o < NORB; o++) rec[sp * NORB + o] = diag[o];
  rec[NB] = lambda;
  rec[NB + 1] = flag;
  rec[NB + 2] = sx; rec[NB + 3] = sy; rec[NB + 4] = sz;
  rec[NB + 5] = xy; rec[NB + 6] = xz; rec[NB + 7] = yz;
}

// y = (H - shift) x with the bond blocks recomputed inside every product
// (the reference's HamCompute=Recompute, Hmult_spds_col multiplying on the
// fly, nemo3d/src/base/h_cvectr_mult.c:1134-1886): only the on-site records
// are stored.  Layout as k_spmv (spmv.cu): NORB lanes per atom, one lane per
// orbital row, neighbour segments staged per warp.  The first four lanes of
// each atom set up its four bonds (cosines and Harrison-scaled integrals,
// from the cation's side, bond_frame) in shared memory; every lane then
// evaluates its row (cation) or column (anion) of each block.
template <int NORB, int NSPIN, int WPB, bool DOT, bool PHASE>
__global__ void __launch_bounds__(WPB * 32)
    k_spmv_recompute(long natoms, const int4 *__restrict__ nbr,
                     const unsigned char *__restrict__ site_m, const int *__restrict__ atom_site,
                     const unsigned char *__restrict__ type, const double *__restrict__ dsp,
                     const double *__restrict__ par, int ns, double lx, double ly, double lz,
                     int include_strain, const double *__restrict__ onsite,
                     const double2 *__restrict__ x, double2 *__restrict__ y, double shift,
                     const double *__restrict__ xnorm, int xnorm_idx, double *partial,
                     unsigned int *counter, double *alpha_out, int alpha_idx,
                     const double2 *__restrict__ phase) {
  constexpr int NB = NORB * NSPIN;
  constexpr int APW = 32 / NORB;
  constexpr int ONS = onsite_len(NB);
  // per bond, laid out as the parameter vector: scaled integrals at 10..30,
  // cosines at 31..33 (sk_bond reads the integrals in place)
  constexpr int BF = 34;
  __shared__ double2 xs[WPB][APW][5][NB];
  __shared__ double bf[WPB][APW][4][BF];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ai = lane / NORB, o = lane - ai * NORB;
  const long a = (long(blockIdx.x) * WPB + w) * APW + ai;
  const bool act = ai < APW && a < natoms;
  const double scale = xnorm ? 1.0 / xnorm[xnorm_idx] : 1.0;
  int nb[4] = {-1, -1, -1, -1};
  int m = 0;
  if (act) {
    const int4 v = nbr[a];
    nb[0] = v.x; nb[1] = v.y; nb[2] = v.z; nb[3] = v.w;
    m = site_m[a];
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const int e = sp * NORB + o;
      const double2 v0 = x[a * NB + e];
      xs[w][ai][4][e] = make_double2(scale * v0.x, scale * v0.y);
#pragma unroll
      for (int n = 0; n < 4; n++) {
        double2 t = make_double2(0.0, 0.0);
        if (nb[n] >= 0) {
          const double2 u = x[long(nb[n]) * NB + e];
          t = make_double2(scale * u.x, scale * u.y);
        }
        xs[w][ai][n][e] = t;
      }
    }
    if (o < 4 && nb[o] >= 0) {  // bond o of this atom, from its cation's side
      const long s = atom_site[a], sn = atom_site[nb[o]];
      const bool cat = m < 4;
      const int cs = cat ? type[s] : type[sn], as = cat ? type[sn] : type[s];
      const double *P = par + (long(cs < ns ? cs : 0) * ns + (as < ns ? as : 0)) * kNPAR;
      double d[3], d0[3], Vsc[kNPV];
      if (cat)
        bond_frame(s, o, sn, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
      else
        bond_frame(sn, c_rev_slot[m][o], s, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
      double *f = bf[w][ai][o];
      for (int k = 10; k < 31; k++) f[k] = Vsc[k];
      f[31] = d[0]; f[32] = d[1]; f[33] = d[2];
    }
  }
  __syncwarp();
  double dot = 0.0;
  if (act) {
    const double *rec = onsite + a * ONS;
    double2 acc[NSPIN];
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const double2 v0 = xs[w][ai][4][sp * NORB + o];
      const double dg = rec[sp * NORB + o];
      acc[sp] = make_double2(dg * v0.x, dg * v0.y);
    }
    if (o >= 1 && o <= 4 && rec[NB + 1] != 0.0) {  // dangling-bond sp3 couplings
      const double sx = rec[NB + 2], sy = rec[NB + 3], sz = rec[NB + 4];
      const double cxy = rec[NB + 5], cxz = rec[NB + 6], cyz = rec[NB + 7];
      double c1, c2, c3;
      int k1, k2, k3;
      if (o == 1) { c1 = sx; k1 = 2; c2 = sy; k2 = 3; c3 = sz; k3 = 4; }
      else if (o == 2) { c1 = sx; k1 = 1; c2 = cxy; k2 = 3; c3 = cxz; k3 = 4; }
      else if (o == 3) { c1 = sy; k1 = 1; c2 = cxy; k2 = 2; c3 = cyz; k3 = 4; }
      else { c1 = sz; k1 = 1; c2 = cxz; k2 = 2; c3 = cyz; k3 = 3; }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const double2 *X0 = xs[w][ai][4] + sp * NORB;
        acc[sp].x = fma(c1, X0[k1].x, acc[sp].x); acc[sp].y = fma(c1, X0[k1].y, acc[sp].y);
        acc[sp].x = fma(c2, X0[k2].x, acc[sp].x); acc[sp].y = fma(c2, X0[k2].y, acc[sp].y);
        acc[sp].x = fma(c3, X0[k3].x, acc[sp].x); acc[sp].y = fma(c3, X0[k3].y, acc[sp].y);
      }
    }
    if (NSPIN == 2 && o >= 2 && o <= 4) {  // on-site spin-orbit (mb_ham_spds_so.h)
      const double L = rec[NB];
      const double2 *U = xs[w][ai][4], *D = xs[w][ai][4] + NORB;
      double2 &a0 = acc[0], &a1 = acc[NSPIN - 1];
      if (o == 2) {
        a0.x += L * U[3].y; a0.y -= L * U[3].x;
        a0.x += L * D[4].x; a0.y += L * D[4].y;
        a1.x -= L * D[3].y; a1.y += L * D[3].x;
        a1.x -= L * U[4].x; a1.y -= L * U[4].y;
      } else if (o == 3) {
        a0.x -= L * U[2].y; a0.y += L * U[2].x;
        a0.x += L * D[4].y; a0.y -= L * D[4].x;
        a1.x += L * D[2].y; a1.y -= L * D[2].x;
        a1.x += L * U[4].y; a1.y -= L * U[4].x;
      } else {
        a0.x -= L * D[2].x; a0.y -= L * D[2].y;
        a0.x -= L * D[3].y; a0.y += L * D[3].x;
        a1.x += L * U[2].x; a1.y += L * U[2].y;
        a1.x -= L * U[3].y; a1.y += L * U[3].x;
      }
    }
    const bool cat = m < 4;
#pragma unroll 1
    for (int n = 0; n < 4; n++) {
      if (nb[n] < 0) continue;
      const double *V = bf[w][ai][n];
      const double d[3] = {V[31], V[32], V[33]};
      const double2 *xn = xs[w][ai][n];
      double2 part[NSPIN];
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) part[sp] = make_double2(0.0, 0.0);
      for (int k = 0; k < NORB; k++) {
        // element (cation orbital, anion orbital) of the block
        const double v = cat ? sk_bond(k, o, d, V) : sk_bond(o, k, d, V);
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          part[sp].x = fma(v, xn[sp * NORB + k].x, part[sp].x);
          part[sp].y = fma(v, xn[sp * NORB + k].y, part[sp].y);
        }
      }
      if (PHASE) {
        const double2 ph = __ldg(phase + a * 4 + n);
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          acc[sp].x += ph.x * part[sp].x - ph.y * part[sp].y;
          acc[sp].y += ph.x * part[sp].y + ph.y * part[sp].x;
        }
      } else {
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          acc[sp].x += part[sp].x;
          acc[sp].y += part[sp].y;
        }
      }
    }
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const double2 xo = xs[w][ai][4][sp * NORB + o];
      const double2 out = make_double2(acc[sp].x - shift * xo.x, acc[sp].y - shift * xo.y);
      y[a * NB + sp * NORB + o] = out;
      dot += xo.x * out.x + xo.y * out.y;
    }
  }
  if (DOT) grid_reduce<WPB * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

template <int NORB, int NSPIN>
static int launch_recompute_t(Ctx &c, const double *x, double *y, double shift,
                              const double *xnorm, int xidx, double *alpha_out, int aidx,
                              cudaStream_t s) {
  constexpr int WPB = 4;
  constexpr int APW = 32 / NORB;
  const unsigned grid = unsigned((c.natoms + WPB * APW - 1) / (WPB * APW));
  const double2 *X = reinterpret_cast<const double2 *>(x);
  double2 *Y = reinterpret_cast<double2 *>(y);
  if (alpha_out) {
    int rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
#define TBGPU_RECOMPUTE(DOT, PH)                                                              \
  k_spmv_recompute<NORB, NSPIN, WPB, DOT, PH><<<grid, WPB * 32, 0, s>>>(                     \
      c.natoms, c.d_nbr, c.d_site_m, c.d_atom_site, c.d_type, c.d_dsp, c.d_par, c.nspecies,   \
      c.lattice[0], c.lattice[1], c.lattice[2], c.include_strain, c.d_onsite, X, Y, shift,    \
      xnorm, xidx, DOT ? c.d_partial : nullptr, DOT ? c.d_counter : nullptr, alpha_out, aidx, \
      c.d_phase)
  if (alpha_out && c.bloch) TBGPU_RECOMPUTE(true, true);
  else if (alpha_out) TBGPU_RECOMPUTE(true, false);
  else if (c.bloch) TBGPU_RECOMPUTE(false, true);
  else TBGPU_RECOMPUTE(false, false);
#undef TBGPU_RECOMPUTE
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

int launch_spmv_recompute(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                          int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (c.norb == 10 && c.nspin == 2) return launch_recompute_t<10, 2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10 && c.nspin == 1) return launch_recompute_t<10, 1>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 5 && c.nspin == 2) return launch_recompute_t<5, 2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 5 && c.nspin == 1) return launch_recompute_t<5, 1>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  return set_error(TBGPU_E_UNSUPPORTED);
}

template <int NORB, int NSPIN>
static int assemble_t(Ctx &c) {
  const long na = c.natoms;
  double *ecorr = nullptr;
  TB_CUDA(cudaMallocAsync(&ecorr, sizeof(double) * na * 4 * NORB, c.stream));
  if (c.d_blocks)
    TB_CUDA(cudaMemsetAsync(c.d_blocks, 0, sizeof(double) * na * 4 * NORB * NORB, c.stream));
  const int th = 128;
  k_bonds<NORB><<<unsigned((na * 4 + th - 1) / th), th, 0, c.stream>>>(
      na, c.d_atom_site, c.d_nbr, c.d_type, c.d_dsp, c.d_par, c.d_par_ok, c.nspecies,
      c.lattice[0], c.lattice[1], c.lattice[2], c.include_strain, c.d_blocks, ecorr,
      c.d_status);
  TB_CUDA(cudaGetLastError());
  k_onsite<NORB, NSPIN><<<unsigned((na + th - 1) / th), th, 0, c.stream>>>(
      na, c.d_atom_site, c.d_nbr, c.d_surface, c.d_type, c.d_par, c.d_par_ok, c.nspecies,
      c.include_strain, c.passivate, c.dangling_shift, ecorr, c.d_onsite);
  TB_CUDA(cudaGetLastError());
  TB_CUDA(cudaFreeAsync(ecorr, c.stream));
  return TBGPU_OK;
}

// the bond blocks into `blocks` ([natoms*4*norb*norb], cation slots), for
// exporting a Hamiltonian that is recomputed rather than stored
int compute_blocks(Ctx &c, double *blocks) {
  const long na = c.natoms;
  const int norb = c.norb;
  double *ecorr = nullptr;
  TB_CUDA(cudaMallocAsync(&ecorr, sizeof(double) * na * 4 * norb, c.stream));
  TB_CUDA(cudaMemsetAsync(blocks, 0, sizeof(double) * na * 4 * norb * norb, c.stream));
  const int th = 128;
  const unsigned g = unsigned((na * 4 + th - 1) / th);
  if (norb == 10)
    k_bonds<10><<<g, th, 0, c.stream>>>(na, c.d_atom_site, c.d_nbr, c.d_type, c.d_dsp, c.d_par,
                                        c.d_par_ok, c.nspecies, c.lattice[0], c.lattice[1],
                                        c.lattice[2], c.include_strain, blocks, ecorr, c.d_status);
  else
    k_bonds<5><<<g, th, 0, c.stream>>>(na, c.d_atom_site, c.d_nbr, c.d_type, c.d_dsp, c.d_par,
                                       c.d_par_ok, c.nspecies, c.lattice[0], c.lattice[1],
                                       c.lattice[2], c.include_strain, blocks, ecorr, c.d_status);
  TB_CUDA(cudaGetLastError());
  TB_CUDA(cudaFreeAsync(ecorr, c.stream));
  return TBGPU_OK;
}

// round the assembled store to float (the reference's HamMemorySave build
// keeps Hdd, Hdu, Hds and Hu as float: HamZincBlende.h:51-66)
__global__ void k_to_float(long n, const double *__restrict__ in, float *__restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    out[i] = float(in[i]);
}

static int to_float(Ctx &c, long n, const double *in, float **out) {
  TB_CUDA(cudaMalloc(out, sizeof(float) * n));
  k_to_float<<<1184, 256, 0, c.stream>>>(n, in, *out);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

int assemble(Ctx &c) {
  const long na = c.natoms;
  if (c.recompute && c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  // recompute: the blocks are not stored; the assembly still runs the bond
  // kernel for the on-site strain corrections
  if (!c.recompute)
    TB_CUDA(cudaMalloc(&c.d_blocks, sizeof(double) * na * 4 * c.norb * c.norb));
  TB_CUDA(cudaMalloc(&c.d_onsite, sizeof(double) * na * c.ons));
  int rc = TBGPU_E_UNSUPPORTED;
  if (c.norb == 10 && c.nspin == 2) rc = assemble_t<10, 2>(c);
  else if (c.norb == 10 && c.nspin == 1) rc = assemble_t<10, 1>(c);
  else if (c.norb == 5 && c.nspin == 2) rc = assemble_t<5, 2>(c);
  else if (c.norb == 5 && c.nspin == 1) rc = assemble_t<5, 1>(c);
  else return set_error(rc);
  if (rc || !c.ham_fp32) return rc;
  if ((rc = to_float(c, na * 4 * c.norb * c.norb, c.d_blocks, &c.d_blocks32))) return rc;
  if ((rc = to_float(c, na * c.ons, c.d_onsite, &c.d_onsite32))) return rc;
  TB_CUDA(cudaStreamSynchronize(c.stream));
  cudaFree(c.d_blocks);
  cudaFree(c.d_onsite);
  c.d_blocks = nullptr;
  c.d_onsite = nullptr;
  return TBGPU_OK;
}

}  // namespace tbgpu

// param_init for one material set (nemo3d/src/base/mat3d.c:133-307) with
// param_sp3s_2_sp3d5s (nemo3d/src/ham/mb_ham_spds_micro.c:2984-3026).
extern "C" int tbgpu_prepare_params(int sp3s_family, int include_strain,
                                    const double *pv, const double *strain,
                                    double ev_offset, double a0, double *out) {
  using namespace tbgpu;
  if (!pv || !strain || !out) return set_error(TBGPU_E_ARG);
  double *p = out;
  for (int k = 0; k < kNPAR; k++) out[k] = 0.0;
  if (sp3s_family) {
    // sp3s* (Vogl notation) -> two-centre integrals of the sp3d5s* layout
    const double r3 = std::sqrt(3.0);
    for (int k = 0; k < 6; k++) p[k] = pv[k];
    p[pE_La] = pv[13] / 3;
    p[pE_Lc] = pv[14] / 3;
    p[10] = pv[6] / 4;
    p[14] = pv[9] * r3 / 4;
    p[15] = pv[10] * r3 / 4;
    p[16] = pv[11] * r3 / 4;
    p[17] = pv[12] * r3 / 4;
    p[22] = (pv[7] + 2 * pv[8]) / 4;
    p[23] = (pv[7] - pv[8]) / 4;
    p[pA0] = a0;
    p[32] = p[33] = p[34] = 1.0;
  } else {
    for (int k = 0; k < kNPV; k++) p[k] = pv[k];
  }
  for (int k = 0; k < kNPAR - kNPV; k++) out[kNPV + k] = strain[k];
  const double shc = include_strain ? strain[eta_cat_shift] : 0.0;
  const double sha = include_strain ? strain[eta_an_shift] : 0.0;
  const int an[4] = {pE_sa, pE_pa, pE_sta, pE_da}, ca[4] = {pE_sc, pE_pc, pE_stc, pE_dc};
  const int nE = sp3s_family ? 3 : 4;  // sp3s*: no d levels
  for (int k = 0; k < nE; k++) {
    p[an[k]] += ev_offset - sha;
    p[ca[k]] += ev_offset - shc;
  }
  return TBGPU_OK;
}
