// y = (H - shift) x with the bond blocks recomputed inside every product
// (the reference's HamCompute=Recompute: Hmult_spds_col multiplying on the
// fly, nemo3d/src/base/h_cvectr_mult.c:1134-1886).  Only the on-site records
// are stored; each bond's frame (cosines, Harrison-scaled integrals) and its
// Slater-Koster block are evaluated from positions, displacements and
// parameters in every call, by both atoms of the bond, from the cation's
// side, so that both ends use the numbers the stored assembly would store.
//
// Work layout.  Atoms are visited in a work order of eight cations per warp,
// then eight anions per warp, so that a warp's role is uniform.  Phase 1: lane
// = (atom, bond); the 32 lanes evaluate the same block element at the same
// time, each for its own bond (every orbital index, table lookup and branch
// is resolved at compile time: no divergence), and apply the block to the
// neighbour's segment of x.  A cation lane holds the neighbour's x in
// registers and produces its row sums one cation orbital at a time; an anion
// lane holds its NB accumulators and takes the cation neighbour's x one
// orbital at a time.  Bond results go to shared memory.  Phase 2: lane =
// (atom, orbital row) adds the on-site terms (diagonal, dangling-bond sp3
// couplings, spin-orbit) and the four bond sums, writes y and folds the
// fused dot product.
#include <vector>

#include "reduce.cuh"
#include "slater_koster.cuh"
#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

constexpr int kRcAtoms = 8;  // atoms per warp in the recompute work order
// resident blocks per SM asked of the compiler: the 20-state model trades a
// few spilled registers for 12 warps per SM (1.81 -> 1.40 ms at 1.02M atoms),
// the 10-state ones fit 16 warps without spills (1.10 -> 0.92 ms)
__host__ __device__ constexpr int rc_min_blocks(int norb, int nspin) {
  return norb == 10 && nspin == 2 ? 3 : 4;
}

template <typename V>
__device__ __forceinline__ V cmul(double2 a, V b) {
  using T = decltype(b.x);
  V r;
  r.x = T(a.x) * b.x - T(a.y) * b.y;
  r.y = T(a.x) * b.y + T(a.y) * b.x;
  return r;
}
template <typename V> __device__ __forceinline__ V czero() {
  V r;
  r.x = r.y = 0;
  return r;
}

// bond block (cation row c, anion column a) applied from a cation: out[c] =
// sum_a B[c][a] xn[a] per spin, xn = the anion neighbour's segment
template <int NORB, int NSPIN, bool PHASE, typename T, typename VT>
__device__ __forceinline__ void bond_from_cation(const T d[3], const T (&Vr)[21],
                                                 const VT *__restrict__ xn, T scale,
                                                 double2 ph, VT *out) {
  constexpr int NB = NORB * NSPIN;
  VT R[NB];
#pragma unroll
  for (int e = 0; e < NB; e++) {
    const VT u = __ldg(xn + e);
    R[e].x = scale * u.x;
    R[e].y = scale * u.y;
  }
  static_for<0, NORB>([&](auto Cc) {
    constexpr int c = decltype(Cc)::value;
    VT run[NSPIN];
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) run[sp] = czero<VT>();
    static_for<0, NORB>([&](auto Aa) {
      constexpr int a = decltype(Aa)::value;
      const T v = sk_elem<a, c>(d, Vr);
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        run[sp].x = fma(v, R[sp * NORB + a].x, run[sp].x);
        run[sp].y = fma(v, R[sp * NORB + a].y, run[sp].y);
      }
    });
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) out[sp * NORB + c] = PHASE ? cmul(ph, run[sp]) : run[sp];
  });
}

// the same block applied from an anion (transposed): out[a] = sum_c B[c][a]
// xn[c], xn = the cation neighbour's segment
template <int NORB, int NSPIN, bool PHASE, typename T, typename VT>
__device__ __forceinline__ void bond_from_anion(const T d[3], const T (&Vr)[21],
                                                const VT *__restrict__ xn, T scale,
                                                double2 ph, VT *out) {
  constexpr int NB = NORB * NSPIN;
  VT R[NB];
#pragma unroll
  for (int e = 0; e < NB; e++) R[e] = czero<VT>();
  static_for<0, NORB>([&](auto Cc) {
    constexpr int c = decltype(Cc)::value;
    VT xc[NSPIN];
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const VT u = __ldg(xn + sp * NORB + c);
      xc[sp].x = scale * u.x;
      xc[sp].y = scale * u.y;
    }
    static_for<0, NORB>([&](auto Aa) {
      constexpr int a = decltype(Aa)::value;
      const T v = sk_elem<a, c>(d, Vr);
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        R[sp * NORB + a].x = fma(v, xc[sp].x, R[sp * NORB + a].x);
        R[sp * NORB + a].y = fma(v, xc[sp].y, R[sp * NORB + a].y);
      }
    });
  });
#pragma unroll
  for (int e = 0; e < NB; e++) out[e] = PHASE ? cmul(ph, R[e]) : R[e];
}

// T: arithmetic of the elements and products (double, or float with
// complex-float vectors VT for the mixed-precision solve); the bond geometry
// is double in both
template <int NORB, int NSPIN, int WPB, bool DOT, bool PHASE, typename T = double,
          typename VT = double2>
__global__ void __launch_bounds__(WPB * 32, rc_min_blocks(NORB, NSPIN))
    k_spmv_recompute(long cat_warps, long nwarps, const int *__restrict__ order,
                     const int4 *__restrict__ nbr, const unsigned char *__restrict__ site_m,
                     const int *__restrict__ atom_site, const unsigned char *__restrict__ type,
                     const double *__restrict__ dsp, const double *__restrict__ par, int ns,
                     double lx, double ly, double lz, int include_strain,
                     const double *__restrict__ onsite, const VT *__restrict__ x,
                     VT *__restrict__ y, double shift_d, const double *__restrict__ xnorm,
                     int xnorm_idx, double *partial, unsigned int *counter, double *alpha_out,
                     int alpha_idx, const double2 *__restrict__ phase,
                     const unsigned char *__restrict__ skip) {
  constexpr int NB = NORB * NSPIN;
  constexpr int PS = NB + 1;  // padded row: conflict-free accesses
  constexpr int ONS = onsite_len(NB);
  __shared__ VT part[WPB][kRcAtoms][4][PS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long gw = long(blockIdx.x) * WPB + w;
  const bool live = gw < nwarps;  // warp-uniform
  const T scale = T(xnorm ? 1.0 / xnorm[xnorm_idx] : 1.0);
  const T shift = T(shift_d);
  // phase 1: lane = (atom, bond)
  if (live) {
    const bool cat = gw < cat_warps;  // warp-uniform
    const int ai = lane >> 2, n = lane & 3;
    const int a = order[gw * kRcAtoms + ai];
    VT *out = part[w][ai][n];
    int b = -1;
    if (a >= 0 && !(skip && __ldg(skip + a))) {
      const int4 v = nbr[a];
      b = n == 0 ? v.x : n == 1 ? v.y : n == 2 ? v.z : v.w;
    }
    if (b >= 0) {
      const long s = atom_site[a], sn = atom_site[b];
      const int m = site_m[a];
      const int ts = type[s], tn = type[sn];
      const int cs = cat ? ts : tn, as = cat ? tn : ts;
      const double *P = par + (long(cs < ns ? cs : 0) * ns + (as < ns ? as : 0)) * kNPAR;
      double dd[3], d0[3], r;
      if (cat)
        bond_geometry(s, n, sn, P[pA0], dsp, lx, ly, lz, dd, d0, r);
      else
        bond_geometry(sn, c_rev_slot[m][n], s, P[pA0], dsp, lx, ly, lz, dd, d0, r);
      const T d[3] = {T(dd[0]), T(dd[1]), T(dd[2])};
      T Vr[21];
      scaled_integrals<NORB>(P, include_strain, r, Vr);
      const double2 ph = PHASE ? __ldg(phase + long(a) * 4 + n) : make_double2(1.0, 0.0);
      if (cat)
        bond_from_cation<NORB, NSPIN, PHASE>(d, Vr, x + long(b) * NB, scale, ph, out);
      else
        bond_from_anion<NORB, NSPIN, PHASE>(d, Vr, x + long(b) * NB, scale, ph, out);
    } else {
#pragma unroll
      for (int e = 0; e < NB; e++) out[e] = czero<VT>();
    }
  }
  __syncwarp();
  // phase 2: lane = (atom, orbital row), up to 32 / NORB atoms per pass
  constexpr int APW = 32 / NORB;
  const int ai2 = lane / NORB, o = lane - ai2 * NORB;
  double dot = 0.0;
#pragma unroll 1
  for (int base = 0; base < kRcAtoms; base += APW) {
    const int ai = base + ai2;
    if (!live || ai2 >= APW || ai >= kRcAtoms) continue;
    const int a = order[gw * kRcAtoms + ai];
    if (a < 0 || (skip && __ldg(skip + a))) continue;
    const double *rec = onsite + long(a) * ONS;
    const VT *X0 = x + long(a) * NB;
    auto xo = [&](int e) {
      const VT u = __ldg(X0 + e);
      VT r;
      r.x = scale * u.x;
      r.y = scale * u.y;
      return r;
    };
    VT acc[NSPIN];
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const VT v0 = xo(sp * NORB + o);
      const T dg = T(rec[sp * NORB + o]);
      acc[sp].x = dg * v0.x;
      acc[sp].y = dg * v0.y;
    }
    if (o >= 1 && o <= 4 && rec[NB + 1] != 0.0) {  // dangling-bond sp3 couplings
      const T sx = T(rec[NB + 2]), sy = T(rec[NB + 3]), sz = T(rec[NB + 4]);
      const T cxy = T(rec[NB + 5]), cxz = T(rec[NB + 6]), cyz = T(rec[NB + 7]);
      T c1, c2, c3;
      int k1, k2, k3;
      if (o == 1) { c1 = sx; k1 = 2; c2 = sy; k2 = 3; c3 = sz; k3 = 4; }
      else if (o == 2) { c1 = sx; k1 = 1; c2 = cxy; k2 = 3; c3 = cxz; k3 = 4; }
      else if (o == 3) { c1 = sy; k1 = 1; c2 = cxy; k2 = 2; c3 = cyz; k3 = 4; }
      else { c1 = sz; k1 = 1; c2 = cxz; k2 = 2; c3 = cyz; k3 = 3; }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const VT u1 = xo(sp * NORB + k1), u2 = xo(sp * NORB + k2), u3 = xo(sp * NORB + k3);
        acc[sp].x = fma(c1, u1.x, acc[sp].x); acc[sp].y = fma(c1, u1.y, acc[sp].y);
        acc[sp].x = fma(c2, u2.x, acc[sp].x); acc[sp].y = fma(c2, u2.y, acc[sp].y);
        acc[sp].x = fma(c3, u3.x, acc[sp].x); acc[sp].y = fma(c3, u3.y, acc[sp].y);
      }
    }
    if (NSPIN == 2 && o >= 2 && o <= 4) {  // on-site spin-orbit (mb_ham_spds_so.h)
      const T L = T(rec[NB]);
      VT &a0 = acc[0], &a1 = acc[NSPIN - 1];
      if (o == 2) {
        const VT U3 = xo(3), D4 = xo(NORB + 4), D3 = xo(NORB + 3), U4 = xo(4);
        a0.x += L * U3.y; a0.y -= L * U3.x;
        a0.x += L * D4.x; a0.y += L * D4.y;
        a1.x -= L * D3.y; a1.y += L * D3.x;
        a1.x -= L * U4.x; a1.y -= L * U4.y;
      } else if (o == 3) {
        const VT U2 = xo(2), D4 = xo(NORB + 4), D2 = xo(NORB + 2), U4 = xo(4);
        a0.x -= L * U2.y; a0.y += L * U2.x;
        a0.x += L * D4.y; a0.y -= L * D4.x;
        a1.x += L * D2.y; a1.y -= L * D2.x;
        a1.x += L * U4.y; a1.y -= L * U4.x;
      } else {
        const VT D2 = xo(NORB + 2), D3 = xo(NORB + 3), U2 = xo(2), U3 = xo(3);
        a0.x -= L * D2.x; a0.y -= L * D2.y;
        a0.x -= L * D3.y; a0.y += L * D3.x;
        a1.x += L * U2.x; a1.y += L * U2.y;
        a1.x -= L * U3.y; a1.y += L * U3.x;
      }
    }
#pragma unroll
    for (int n = 0; n < 4; n++) {
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const VT t = part[w][ai][n][sp * NORB + o];
        acc[sp].x += t.x;
        acc[sp].y += t.y;
      }
    }
#pragma unroll
    for (int sp = 0; sp < NSPIN; sp++) {
      const VT x0 = xo(sp * NORB + o);
      VT out;
      out.x = acc[sp].x - shift * x0.x;
      out.y = acc[sp].y - shift * x0.y;
      y[long(a) * NB + sp * NORB + o] = out;
      dot += double(x0.x) * double(out.x) + double(x0.y) * double(out.y);
    }
  }
  if (DOT) grid_reduce<WPB * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

template <int NORB, int NSPIN, typename T, typename VT>
int launch_t(Ctx &c, const void *x, void *y, double shift, const double *xnorm, int xidx,
             double *alpha_out, int aidx, cudaStream_t s) {
  constexpr int WPB = 4;
  if (c.rc_warps <= 0) return set_error(TBGPU_E_STATE);
  const unsigned grid = unsigned((c.rc_warps + WPB - 1) / WPB);
  const VT *X = reinterpret_cast<const VT *>(x);
  VT *Y = reinterpret_cast<VT *>(y);
  if (alpha_out) {
    int rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
#define TBGPU_RECOMPUTE(DOT, PH)                                                               \
  k_spmv_recompute<NORB, NSPIN, WPB, DOT, PH, T, VT><<<grid, WPB * 32, 0, s>>>(               \
      c.rc_cat_warps, c.rc_warps, c.d_rc_order, c.d_nbr, c.d_site_m, c.d_atom_site, c.d_type, \
      c.d_dsp, c.d_par, c.nspecies, c.lattice[0], c.lattice[1], c.lattice[2],                 \
      c.include_strain, c.d_onsite, X, Y, shift, xnorm, xidx, DOT ? c.d_partial : nullptr,    \
      DOT ? c.d_counter : nullptr, alpha_out, aidx, c.d_phase, c.d_skip)
  if constexpr (sizeof(T) == sizeof(double)) {
    if (alpha_out && c.bloch) TBGPU_RECOMPUTE(true, true);
    else if (alpha_out) TBGPU_RECOMPUTE(true, false);
    else if (c.bloch) TBGPU_RECOMPUTE(false, true);
    else TBGPU_RECOMPUTE(false, false);
  } else {  // the float product serves the mixed-precision solve at Gamma
    if (c.bloch) return set_error(TBGPU_E_UNSUPPORTED);
    if (alpha_out) TBGPU_RECOMPUTE(true, false);
    else TBGPU_RECOMPUTE(false, false);
  }
#undef TBGPU_RECOMPUTE
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

}  // namespace

// cations in atom order, padded with -1 to a multiple of eight, then the
// anions the same way
int build_recompute_order(Ctx &c) {
  const long na = c.natoms;
  std::vector<unsigned char> m(na);
  TB_CUDA(cudaMemcpyAsync(m.data(), c.d_site_m, na, cudaMemcpyDeviceToHost, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  std::vector<int> order;
  order.reserve(na + 2 * kRcAtoms);
  for (int pass = 0; pass < 2; pass++) {
    for (long a = 0; a < na; a++)
      if ((m[a] < 4) == (pass == 0)) order.push_back(int(a));
    while (order.size() % kRcAtoms) order.push_back(-1);
    if (pass == 0) c.rc_cat_warps = long(order.size()) / kRcAtoms;
  }
  c.rc_warps = long(order.size()) / kRcAtoms;
  if (c.d_rc_order) cudaFree(c.d_rc_order);
  c.d_rc_order = nullptr;
  TB_CUDA(cudaMalloc(&c.d_rc_order, sizeof(int) * (order.empty() ? 1 : order.size())));
  if (!order.empty())
    TB_CUDA(cudaMemcpyAsync(c.d_rc_order, order.data(), sizeof(int) * order.size(),
                            cudaMemcpyHostToDevice, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  return TBGPU_OK;
}

int launch_spmv_recompute(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                          int xidx, double *alpha_out, int aidx, cudaStream_t s) {
#define TBGPU_RC_CASE(NO, NS)                                                                  \
  if (c.norb == NO && c.nspin == NS)                                                           \
    return launch_t<NO, NS, double, double2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  TBGPU_RC_CASE(10, 2) TBGPU_RC_CASE(10, 1) TBGPU_RC_CASE(5, 2) TBGPU_RC_CASE(5, 1)
#undef TBGPU_RC_CASE
  return set_error(TBGPU_E_UNSUPPORTED);
}

// complex-float vectors, float elements and accumulation (mixed precision)
int launch_spmv_recompute_f32(Ctx &c, const float *x, float *y, double shift,
                              const double *xnorm, int xidx, double *alpha_out, int aidx,
                              cudaStream_t s) {
#define TBGPU_RC_CASE(NO, NS)                                                                  \
  if (c.norb == NO && c.nspin == NS)                                                           \
    return launch_t<NO, NS, float, float2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  TBGPU_RC_CASE(10, 2) TBGPU_RC_CASE(10, 1) TBGPU_RC_CASE(5, 2) TBGPU_RC_CASE(5, 1)
#undef TBGPU_RC_CASE
  return set_error(TBGPU_E_UNSUPPORTED);
}

}  // namespace tbgpu
