// Slater-Koster two-centre elements and the bond frame, shared by the
// stored assembly (build.cu) and the H*x that recomputes the blocks in every
// product (recompute.cu).  Restates
//   strain_corr_prep                  nemo3d/src/ham/mb_ham_spds_micro.c:2848-2982
//   h3d_offdiag_diag_corr + get_X_Y   nemo3d/src/ham/mb_ham_spds_micro.c:597-1451,
//                                     mb_ham_spds_VoffdEdiag_constructors.h
//   getRelativePosVec                 nemo3d/src/base/geo_struct.c:2224-2297
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

// orbital order s*, s, px, py, pz, dxy, dyz, dzx, dx2-y2, dz2
// (mb_ham_spds_micro.h:97-116); orbital kinds: 0 s*, 1 s, 2 p, 3 d
__host__ __device__ constexpr int kind_of(int o) { return o == 0 ? 0 : o == 1 ? 1 : o < 5 ? 2 : 3; }
__host__ __device__ constexpr int ang_of(int o) { return o < 2 ? 0 : o < 5 ? 1 : 2; }

// Integral parameter indices (sigma, pi, delta) of an (anion kind, cation
// kind) pair (mb_ham_spds_micro.c:58-146).  One list, two copies: constant
// memory for lookups with run-time kinds, a constexpr function for lookups
// that the compiler resolves.
#define TBGPU_VIDX_TABLE                                                  \
  {/* anion s*  with cation s*, s, p, d */                                \
   {{11, -1, -1}, {12, -1, -1}, {16, -1, -1}, {20, -1, -1}},              \
   /* anion s */                                                          \
   {{13, -1, -1}, {10, -1, -1}, {14, -1, -1}, {18, -1, -1}},              \
   /* anion p */                                                          \
   {{17, -1, -1}, {15, -1, -1}, {22, 23, -1}, {24, 26, -1}},              \
   /* anion d */                                                          \
   {{21, -1, -1}, {19, -1, -1}, {25, 27, -1}, {28, 29, 30}}}
static __constant__ int8_t c_vidx[4][4][3] = TBGPU_VIDX_TABLE;
__host__ __device__ constexpr int vidx_of(int ka, int kc, int j) {
  const int8_t t[4][4][3] = TBGPU_VIDX_TABLE;
  return t[ka][kc][j];
}
// strain-correction coefficient index of a kind pair, on-site energy index
// by kind for anion / cation (diag_map_set)
static __constant__ int8_t c_cidx[4][4] = {
    {18, 19, 23, 27}, {20, 17, 21, 25}, {24, 22, 29, 30}, {28, 26, 31, 32}};
static __constant__ int8_t c_eidx[2][4] = {{4, 0, 1, 6}, {5, 2, 3, 7}};

// Harrison scaling (E_const_prep): the 21 two-centre integrals (parameters
// 10..30) share 14 distinct strain exponents; integral k uses exponent slot
// eta_slot(k), slot j is strain parameter slot_eta(j).  Slots that involve
// d orbitals are not needed by the 5-orbital models.
__host__ __device__ constexpr int eta_slot(int k) {
  const int8_t t[21] = {0, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 8, 9, 9, 10, 10, 11, 12, 13};
  return t[k];
}
__host__ __device__ constexpr int slot_eta(int j) {
  const int8_t t[14] = {eta_sss, eta_ststs, eta_ssts, eta_sps, eta_stps, eta_sds, eta_stds,
                        eta_pps, eta_ppp, eta_pds, eta_pdp, eta_dds, eta_ddp, eta_ddd};
  return t[j];
}
__host__ __device__ constexpr bool slot_has_d(int j) {
  return j == 5 || j == 6 || (j >= 9 && j <= 13);
}

// compile-time loop: f(std::integral_constant<int, i>) for i in [I, N)
template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>());
    static_for<I + 1, N>(f);
  }
}

// Slater-Koster element for orbital a on the first atom, b on the second,
// ang(a) <= ang(b), cosines d[] from first to second (Slater & Koster 1954,
// Table I, written with index permutations).
template <typename T>
__device__ __forceinline__ T sk_ordered(int a, int b, const T d[3], T Vs, T Vp, T Vd) {
  const int la = ang_of(a), lb = ang_of(b);
  const T s3 = T(kSqr3);
  if (lb == 0) return Vs;                          // s/s* - s/s*
  if (la == 0 && lb == 1) return d[b - 2] * Vs;    // s - p
  const T l2 = d[0] * d[0], m2 = d[1] * d[1], n2 = d[2] * d[2];
  const T q = n2 - T(0.5) * (l2 + m2);           // 3z2-r2 angular factor
  const T lm2 = l2 - m2;
  // t2g orbitals dxy, dyz, dzx as index pairs (u, v)
  const int tu[3] = {0, 1, 2}, tv[3] = {1, 2, 0};
  if (la == 0) {                                    // s - d
    if (b < 8) return s3 * d[tu[b - 5]] * d[tv[b - 5]] * Vs;
    return (b == 8 ? T(0.5) * s3 * lm2 : q) * Vs;
  }
  if (la == 1 && lb == 1) {                         // p - p
    const T di = d[a - 2], dj = d[b - 2];
    return a == b ? di * di * Vs + (T(1.0) - di * di) * Vp : di * dj * Vs - di * dj * Vp;
  }
  if (la == 1) {                                    // p - d
    const int i = a - 2;
    const T di = d[i];
    if (b < 8) {
      const int u = tu[b - 5], v = tv[b - 5];
      if (i == u) return s3 * d[u] * d[u] * d[v] * Vs + d[v] * (T(1.0) - T(2.0) * d[u] * d[u]) * Vp;
      if (i == v) return s3 * d[v] * d[v] * d[u] * Vs + d[u] * (T(1.0) - T(2.0) * d[v] * d[v]) * Vp;
      const T p3 = d[0] * d[1] * d[2];
      return s3 * p3 * Vs - T(2.0) * p3 * Vp;
    }
    if (b == 8) {
      if (i == 0) return T(0.5) * s3 * di * lm2 * Vs + di * (T(1.0) - lm2) * Vp;
      if (i == 1) return T(0.5) * s3 * di * lm2 * Vs - di * (T(1.0) + lm2) * Vp;
      return T(0.5) * s3 * di * lm2 * Vs - di * lm2 * Vp;
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
      const T pu = d[u1] * d[u1], pv = d[v1] * d[v1];
      return T(3.0) * pu * pv * Vs + (pu + pv - T(4.0) * pu * pv) * Vp + (d[w] * d[w] + pu * pv) * Vd;
    }
    const int u2 = tu[y - 5], v2 = tv[y - 5];
    const int sh = (u1 == u2 || u1 == v2) ? u1 : v1;  // shared index
    const int p = (u1 == sh) ? v1 : u1, r = (u2 == sh) ? v2 : u2;
    const T ds2 = d[sh] * d[sh], pr = d[p] * d[r];
    return T(3.0) * pr * ds2 * Vs + pr * (T(1.0) - T(4.0) * ds2) * Vp + pr * (ds2 - T(1.0)) * Vd;
  }
  if (x < 8) {                                      // t2g - eg
    const T l = d[0], m = d[1], n = d[2];
    if (y == 8) {
      if (x == 5) return T(1.5) * l * m * lm2 * Vs - T(2.0) * l * m * lm2 * Vp + T(0.5) * l * m * lm2 * Vd;
      if (x == 6) return T(1.5) * m * n * lm2 * Vs - m * n * (T(1.0) + T(2.0) * lm2) * Vp + m * n * (T(1.0) + T(0.5) * lm2) * Vd;
      return T(1.5) * n * l * lm2 * Vs + n * l * (T(1.0) - T(2.0) * lm2) * Vp - n * l * (T(1.0) - T(0.5) * lm2) * Vd;
    }
    if (x == 5) return s3 * l * m * q * Vs - T(2.0) * s3 * l * m * n2 * Vp + T(0.5) * s3 * l * m * (T(1.0) + n2) * Vd;
    const T uv = (x == 6) ? m * n : l * n;
    return s3 * uv * q * Vs + s3 * uv * (l2 + m2 - n2) * Vp - T(0.5) * s3 * uv * (l2 + m2) * Vd;
  }
  if (x == 8 && y == 8) return T(0.75) * lm2 * lm2 * Vs + (l2 + m2 - lm2 * lm2) * Vp + (n2 + T(0.25) * lm2 * lm2) * Vd;
  if (x == 8) return T(0.5) * s3 * lm2 * q * Vs - s3 * n2 * lm2 * Vp + T(0.25) * s3 * (T(1.0) + n2) * lm2 * Vd;
  return q * q * Vs + T(3.0) * n2 * (l2 + m2) * Vp + T(0.75) * (l2 + m2) * (l2 + m2) * Vd;
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

// sk_bond for orbitals known at compile time, integrals Vr[k] = parameter
// 10 + k: every table lookup and branch resolves in the compiler, so a warp
// whose lanes hold different bonds evaluates one element without divergence.
template <int I, typename T>
__device__ __forceinline__ T vr_get(const T (&Vr)[21]) {
  if constexpr (I >= 0) return Vr[I - 10];
  else return T(0);
}
template <int A, int C, typename T>
__device__ __forceinline__ T sk_elem(const T d[3], const T (&Vr)[21]) {
  constexpr int ka = kind_of(A), kc = kind_of(C);
  const T Vs = vr_get<vidx_of(ka, kc, 0)>(Vr);
  const T Vp = vr_get<vidx_of(ka, kc, 1)>(Vr);
  const T Vd = vr_get<vidx_of(ka, kc, 2)>(Vr);
  constexpr int la = ang_of(A), lc = ang_of(C);
  if constexpr (la <= lc) {
    return sk_ordered(A, C, d, Vs, Vp, Vd);
  } else {
    const T e = sk_ordered(C, A, d, Vs, Vp, Vd);
    return ((la + lc) & 1) ? -e : e;
  }
}

// Geometry of one bond seen from its cation (site s, neighbour slot n) to
// the anion at site sn: direction cosines of the strained (d) and unstrained
// (d0) bond, anion -> cation, and the strained length r.
__device__ __forceinline__ void bond_geometry(long s, int n, long sn, double a0,
                                              const double *dsp, double lx, double ly,
                                              double lz, double d[3], double d0[3],
                                              double &r) {
  const int m = int(s & 7), mn = c_nnmap[m][n][3];
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
  r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int k = 0; k < 3; k++) {
    d0[k] = v0[k] / r0;
    d[k] = v[k] / r;
  }
}

// The 21 two-centre integrals of the parameter vector P with Harrison's
// scaling (d0/d)^eta, brat = (sqrt(3)/4 a0) / r, one pow per distinct
// exponent, in precision T (the geometry stays double); Vr[k] is parameter
// 10 + k.  NORB = 5 skips the d integrals (left at zero).
template <int NORB, typename T>
__device__ __forceinline__ void scaled_integrals(const double *P, int include_strain, double r,
                                                 T (&Vr)[21]) {
  const double *S = P + kNPV;
  if (!include_strain) {
#pragma unroll
    for (int k = 0; k < 21; k++) Vr[k] = T(P[10 + k]);
    return;
  }
  const T brat = T((0.25 * kSqr3 * P[pA0]) / r);
  T pw[14];
  static_for<0, 14>([&](auto J) {
    constexpr int j = decltype(J)::value;
    if constexpr (NORB == 5 && slot_has_d(j)) pw[j] = T(0);
    else pw[j] = pow(brat, T(S[slot_eta(j)]));
  });
  static_for<0, 21>([&](auto K) {
    constexpr int k = decltype(K)::value;
    Vr[k] = T(P[10 + k]) * pw[eta_slot(k)];
  });
}

// The bond frame of the stored assembly: cosines d, d0 and the full
// parameter vector with scaled integrals in Vsc[10..30].  Both ends of a bond
// call it with the cation's view, so they use the same numbers.
template <int NORB>
__device__ __forceinline__ void bond_frame(long s, int n, long sn, const double *P,
                                           const double *dsp, double lx, double ly,
                                           double lz, int include_strain, double d[3],
                                           double d0[3], double *Vsc) {
  double r;
  bond_geometry(s, n, sn, P[pA0], dsp, lx, ly, lz, d, d0, r);
  for (int k = 0; k < kNPV; k++) Vsc[k] = P[k];
  double Vr[21];
  scaled_integrals<NORB>(P, include_strain, r, Vr);
#pragma unroll
  for (int k = 0; k < 21; k++) Vsc[10 + k] = Vr[k];
}

}  // namespace tbgpu
