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

#include "slater_koster.cuh"
#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

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
    bond_frame<NORB>(s, n, sn, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
  else
    bond_frame<NORB>(sn, c_rev_slot[m][n], s, P, dsp, lx, ly, lz, include_strain, d, d0, Vsc);
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
  // the mixed-precision solve runs on the float store or on the recompute
  // product
  if (c.lanczos_f32 && !c.recompute && !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
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
  if (!rc && (c.recompute || c.lanczos_f32)) rc = build_recompute_order(c);
  if (rc || !c.ham_fp32) return rc;
  if ((rc = to_float(c, na * 4 * c.norb * c.norb, c.d_blocks, &c.d_blocks32))) return rc;
  if ((rc = to_float(c, na * c.ons, c.d_onsite, &c.d_onsite32))) return rc;
  TB_CUDA(cudaStreamSynchronize(c.stream));
  cudaFree(c.d_blocks);
  c.d_blocks = nullptr;
  if (!c.lanczos_f32) {  // the mixed solve refines with the double records
    cudaFree(c.d_onsite);
    c.d_onsite = nullptr;
  }
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
