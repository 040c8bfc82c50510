// y = (H - shift) x over the stored Hamiltonian, optionally with the Lanczos
// alpha = Re<x, y> fused into the epilogue.
//
// Restates Hmult_spds_col_stored / Hv_stored_20_Hzb
// (nemo3d/src/base/Hmult_stored.c:73-172, 176-607) and the alpha dot of
// single_lanczos_iteration (eigen/src/lanczos.c:679-707).
//
// Layout: NORB lanes per atom (one lane per orbital, all spins), 32/NORB atoms
// per warp.  The warp stages its atoms' own and neighbour vector segments in
// shared memory; each lane then streams its row of every bond block (cation:
// row of the stored block, anion: column of the neighbour cation's block,
// i.e. the Hermitian transpose, each bond being stored once).
#include "tbgpu_internal.cuh"
#include "reduce.cuh"
#include "zincblende.cuh"

namespace tbgpu {

template <typename T, typename V>
__device__ __forceinline__ V cmul_r(T v, V a) {
  V r;
  r.x = v * a.x;
  r.y = v * a.y;
  return r;
}
template <typename T, typename V>
__device__ __forceinline__ void cfma_r(V &acc, T v, V a) {
  acc.x = fma(v, a.x, acc.x);
  acc.y = fma(v, a.y, acc.y);
}
// acc += (i*lambda) * a
template <typename T, typename V>
__device__ __forceinline__ void cfma_i(V &acc, T lam, V a) {
  acc.x -= lam * a.y;
  acc.y += lam * a.x;
}
template <typename V> __device__ __forceinline__ V vzero() {
  V r;
  r.x = r.y = 0;
  return r;
}

// PHASE: bonds carry the Bloch phase phase[a*4+n] of H[a][nbr] (periodic
// structures away from the Gamma point).
// HT: element type of the stored Hamiltonian (double, or float for the
// single-precision store); VT: vector element, double2 (arithmetic in double)
// or float2 (the mixed-precision solve: float arithmetic, alpha in double).
template <int NORB, int NSPIN, int WPB, bool DOT, bool PHASE = false, typename HT = double,
          typename VT = double2>
__global__ void __launch_bounds__(WPB * 32)
    k_spmv(long natoms, const int4 *__restrict__ nbr, const unsigned char *__restrict__ site_m,
           const HT *__restrict__ onsite, const HT *__restrict__ blocks,
           const VT *__restrict__ x, VT *__restrict__ y, double shift_d,
           const double *__restrict__ xnorm, int xnorm_idx, double *partial,
           unsigned int *counter, double *alpha_out, int alpha_idx,
           const double2 *__restrict__ phase = nullptr,
           const unsigned char *__restrict__ skip = nullptr) {
  using RT = decltype(VT::x);
  constexpr int NB = NORB * NSPIN;
  constexpr int APW = 32 / NORB;
  constexpr int ONS = onsite_len(NB);
  __shared__ VT xs[WPB][APW][5][NB];  // slots 0..3 neighbours, 4 own
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ai = lane / NORB, o = lane - ai * NORB;
  const long a = (long(blockIdx.x) * WPB + w) * APW + ai;
  // skip: atoms left out of the product (a converged dot of a batched solve)
  const bool act = ai < APW && a < natoms && !(skip && __ldg(skip + a));
  const RT scale = RT(xnorm ? 1.0 / xnorm[xnorm_idx] : 1.0);
  const RT shift = RT(shift_d);
  int nb[4] = {-1, -1, -1, -1};
  int m = 0;
  if (act) {
    const int4 v = nbr[a];
    nb[0] = v.x; nb[1] = v.y; nb[2] = v.z; nb[3] = v.w;
    m = site_m[a];
#pragma unroll
    for (int s = 0; s < NSPIN; s++) {
      const int e = s * NORB + o;
      xs[w][ai][4][e] = cmul_r(scale, x[a * NB + e]);
#pragma unroll
      for (int n = 0; n < 4; n++)
        xs[w][ai][n][e] = nb[n] >= 0 ? cmul_r(scale, x[long(nb[n]) * NB + e]) : vzero<VT>();
    }
  }
  __syncwarp();
  double dot = 0.0;
  if (act) {
    const HT *rec = onsite + a * ONS;
    VT acc[NSPIN];
#pragma unroll
    for (int s = 0; s < NSPIN; s++) acc[s] = cmul_r(RT(rec[s * NORB + o]), xs[w][ai][4][s * NORB + o]);
    // dangling-bond sp3 couplings among s, px, py, pz (surface atoms only)
    if (o >= 1 && o <= 4 && rec[NB + 1] != HT(0)) {
      const RT sx = rec[NB + 2], sy = rec[NB + 3], sz = rec[NB + 4];
      const RT xy = rec[NB + 5], xz = rec[NB + 6], yz = rec[NB + 7];
      RT c1, c2, c3;
      int k1, k2, k3;
      if (o == 1) { c1 = sx; k1 = 2; c2 = sy; k2 = 3; c3 = sz; k3 = 4; }
      else if (o == 2) { c1 = sx; k1 = 1; c2 = xy; k2 = 3; c3 = xz; k3 = 4; }
      else if (o == 3) { c1 = sy; k1 = 1; c2 = xy; k2 = 2; c3 = yz; k3 = 4; }
      else { c1 = sz; k1 = 1; c2 = xz; k2 = 2; c3 = yz; k3 = 3; }
#pragma unroll
      for (int s = 0; s < NSPIN; s++) {
        cfma_r(acc[s], c1, xs[w][ai][4][s * NORB + k1]);
        cfma_r(acc[s], c2, xs[w][ai][4][s * NORB + k2]);
        cfma_r(acc[s], c3, xs[w][ai][4][s * NORB + k3]);
      }
    }
    // on-site spin-orbit (mb_ham_spds_so.h), p orbitals 2,3,4 of both spins
    if (NSPIN == 2 && o >= 2 && o <= 4) {
      const RT L = rec[NB];
      const VT *U = xs[w][ai][4], *D = xs[w][ai][4] + NORB;
      if (o == 2) {
        cfma_i(acc[0], -L, U[3]); cfma_r(acc[0], L, D[4]);
        cfma_i(acc[1], L, D[3]);  cfma_r(acc[1], -L, U[4]);
      } else if (o == 3) {
        cfma_i(acc[0], L, U[2]);  cfma_i(acc[0], -L, D[4]);
        cfma_i(acc[1], -L, D[2]); cfma_i(acc[1], -L, U[4]);
      } else {
        cfma_r(acc[0], -L, D[2]); cfma_i(acc[0], L, D[3]);
        cfma_r(acc[1], L, U[2]);  cfma_i(acc[1], L, U[3]);
      }
    }
    // bonds
    const bool cat = m < 4;
#pragma unroll
    for (int n = 0; n < 4; n++) {
      if (nb[n] < 0) continue;
      const VT *xn = xs[w][ai][n];
      // with phases, the bond's product is formed apart and then rotated
      VT part[NSPIN];
      VT *tgt = acc;
      if (PHASE) {
#pragma unroll
        for (int s = 0; s < NSPIN; s++) part[s] = vzero<VT>();
        tgt = part;
      }
      if (cat) {
        const HT *M = blocks + (a * 4 + n) * (NORB * NORB) + o * NORB;
        RT r[NORB];
        if constexpr (NORB % 2 == 0 && sizeof(HT) == 8) {
          // rows start on 16-byte boundaries when NORB is even (block = NORB^2
          // doubles, row = NORB doubles): 128-bit loads
#pragma unroll
          for (int k = 0; k < NORB; k += 2) {
            const double2 t = __ldg(reinterpret_cast<const double2 *>(M + k));
            r[k] = t.x;
            r[k + 1] = t.y;
          }
        } else {
#pragma unroll
          for (int k = 0; k < NORB; k++) r[k] = __ldg(M + k);
        }
#pragma unroll
        for (int k = 0; k < NORB; k++)
#pragma unroll
          for (int s = 0; s < NSPIN; s++) cfma_r(tgt[s], r[k], xn[s * NORB + k]);
      } else {
        const HT *M = blocks + (long(nb[n]) * 4 + c_rev_slot[m][n]) * (NORB * NORB) + o;
#pragma unroll
        for (int k = 0; k < NORB; k++) {
          const RT v = RT(__ldg(M + k * NORB));
#pragma unroll
          for (int s = 0; s < NSPIN; s++) cfma_r(tgt[s], v, xn[s * NORB + k]);
        }
      }
      if (PHASE) {
        const double2 ph = __ldg(phase + a * 4 + n);
#pragma unroll
        for (int s = 0; s < NSPIN; s++) {
          acc[s].x += RT(ph.x) * part[s].x - RT(ph.y) * part[s].y;
          acc[s].y += RT(ph.x) * part[s].y + RT(ph.y) * part[s].x;
        }
      }
    }
#pragma unroll
    for (int s = 0; s < NSPIN; s++) {
      const VT xo = xs[w][ai][4][s * NORB + o];
      VT out;
      out.x = acc[s].x - shift * xo.x;
      out.y = acc[s].y - shift * xo.y;
      y[a * NB + s * NORB + o] = out;
      dot += double(xo.x) * double(out.x) + double(xo.y) * double(out.y);
    }
  }
  if (DOT) grid_reduce<WPB * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

constexpr int kWPB = 8;

// warps per block of the lane-gather kernel: 8 (variants 0 and 1), 4
// (variant 8) or 2 (variant 9).  The block size sets each block's staging
// array (warps x atoms per warp x 5 segments) and so how many blocks and
// warps an SM holds; every atom computes the same either way.
inline int lane_gather_wpb(const Ctx &c) {
  return c.spmv_variant == 8 ? 4 : c.spmv_variant == 9 ? 2 : kWPB;
}

template <int NORB, int NSPIN, typename HT, typename VT = double2, int WPB = kWPB>
static int launch_ht_w(Ctx &c, const void *x, void *y, double shift,
                       const double *xnorm, int xidx, double *alpha_out, int aidx,
                       cudaStream_t s);

template <int NORB, int NSPIN, typename HT, typename VT = double2>
static int launch_ht(Ctx &c, const void *x, void *y, double shift,
                     const double *xnorm, int xidx, double *alpha_out, int aidx,
                     cudaStream_t s) {
  switch (lane_gather_wpb(c)) {
    case 4:
      return launch_ht_w<NORB, NSPIN, HT, VT, 4>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
    case 2:
      return launch_ht_w<NORB, NSPIN, HT, VT, 2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
    default:
      return launch_ht_w<NORB, NSPIN, HT, VT, kWPB>(c, x, y, shift, xnorm, xidx, alpha_out, aidx,
                                                   s);
  }
}

template <int NORB, int NSPIN, typename HT, typename VT, int WPB>
static int launch_ht_w(Ctx &c, const void *x, void *y, double shift,
                       const double *xnorm, int xidx, double *alpha_out, int aidx,
                       cudaStream_t s) {
  constexpr int kWPB = WPB;  // this launch's block size
  constexpr int APW = 32 / NORB;
  const long per_block = long(kWPB) * APW;
  const unsigned grid = unsigned((c.natoms + per_block - 1) / per_block);
  const VT *X = reinterpret_cast<const VT *>(x);
  VT *Y = reinterpret_cast<VT *>(y);
  const HT *ons = ham_onsite<HT>(c), *blk = ham_blocks<HT>(c);
  if (alpha_out) {
    int rc = ensure_partials(c, int(grid));
    if (rc) return rc;
    if (c.bloch)
      k_spmv<NORB, NSPIN, kWPB, true, true, HT, VT><<<grid, kWPB * 32, 0, s>>>(
          c.natoms, c.d_nbr, c.d_site_m, ons, blk, X, Y, shift, xnorm, xidx, c.d_partial,
          c.d_counter, alpha_out, aidx, c.d_phase, c.d_skip);
    else
      k_spmv<NORB, NSPIN, kWPB, true, false, HT, VT><<<grid, kWPB * 32, 0, s>>>(
          c.natoms, c.d_nbr, c.d_site_m, ons, blk, X, Y, shift, xnorm, xidx, c.d_partial,
          c.d_counter, alpha_out, aidx, nullptr, c.d_skip);
  } else {
    if (c.bloch)
      k_spmv<NORB, NSPIN, kWPB, false, true, HT, VT><<<grid, kWPB * 32, 0, s>>>(
          c.natoms, c.d_nbr, c.d_site_m, ons, blk, X, Y, shift, xnorm, xidx, nullptr, nullptr,
          nullptr, 0, c.d_phase, c.d_skip);
    else
      k_spmv<NORB, NSPIN, kWPB, false, false, HT, VT><<<grid, kWPB * 32, 0, s>>>(
          c.natoms, c.d_nbr, c.d_site_m, ons, blk, X, Y, shift, xnorm, xidx, nullptr, nullptr,
          nullptr, 0, nullptr, c.d_skip);
  }
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

template <int NORB, int NSPIN>
static int launch_t(Ctx &c, const double *x, double *y, double shift,
                    const double *xnorm, int xidx, double *alpha_out, int aidx,
                    cudaStream_t s) {
  return c.ham_fp32
             ? launch_ht<NORB, NSPIN, float>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
             : launch_ht<NORB, NSPIN, double>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
}

int launch_spmv(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (c.recompute) return launch_spmv_recompute(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  // the warp-staged kernel has no phase support: periodic structures away
  // from Gamma take the lane-gather kernel
  if ((c.spmv_variant == 6 || c.spmv_variant == 7) && pen_supported(c))
    return launch_spmv_pen(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.spmv_variant == 5 && lane_supported(c))
    return launch_spmv_lane(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10 && c.spmv_variant == 3 && !c.bloch)
    return launch_spmv_tile(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10 && c.spmv_variant != 1 && c.spmv_variant != 8 && c.spmv_variant != 9 &&
      !c.bloch)
    return launch_spmv_async(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10 && c.nspin == 2) return launch_t<10, 2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10 && c.nspin == 1) return launch_t<10, 1>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 5 && c.nspin == 2) return launch_t<5, 2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 5 && c.nspin == 1) return launch_t<5, 1>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  return set_error(TBGPU_E_UNSUPPORTED);
}

// The mixed-precision product on complex-float vectors: recomputed in float,
// or over the float store (the warp-staged kernel for 10 orbitals, the
// lane-gather kernel for 5); at the Gamma point.
int launch_spmv_f32(Ctx &c, const float *x, float *y, double shift, const double *xnorm,
                    int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (c.bloch) return set_error(TBGPU_E_UNSUPPORTED);
  if (c.recompute)
    return launch_spmv_recompute_f32(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (!c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  if ((c.spmv_variant == 6 || c.spmv_variant == 7) && pen_supported(c))
    return launch_spmv_pen_f32(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.spmv_variant == 5 && lane_supported(c))
    return launch_spmv_lane_f32(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.norb == 10) return launch_spmv_async_f32(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.nspin == 2)
    return launch_ht<5, 2, float, float2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  return launch_ht<5, 1, float, float2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
}

template <int NORB, int NSPIN, typename HT>
static int launch_scratch_ht(Ctx &c, const double *x, double *y, double shift, double *partial,
                             unsigned int *counter, int cap, double *dot_out, cudaStream_t s) {
  constexpr int APW = 32 / NORB;
  const long per_block = long(kWPB) * APW;
  const long grid = (c.natoms + per_block - 1) / per_block;
  if (grid > cap) return set_error(TBGPU_E_ARG);
  const double2 *X = reinterpret_cast<const double2 *>(x);
  double2 *Y = reinterpret_cast<double2 *>(y);
  if (c.bloch)
    k_spmv<NORB, NSPIN, kWPB, true, true, HT><<<unsigned(grid), kWPB * 32, 0, s>>>(
        c.natoms, c.d_nbr, c.d_site_m, ham_onsite<HT>(c), ham_blocks<HT>(c), X, Y, shift,
        nullptr, 0, partial, counter, dot_out, 0, c.d_phase);
  else
    k_spmv<NORB, NSPIN, kWPB, true, false, HT><<<unsigned(grid), kWPB * 32, 0, s>>>(
        c.natoms, c.d_nbr, c.d_site_m, ham_onsite<HT>(c), ham_blocks<HT>(c), X, Y, shift,
        nullptr, 0, partial, counter, dot_out, 0);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// Lane-gather launch with the alpha dot reduced through caller-provided
// scratch (partial[cap] doubles, zeroed counter).  Allocates nothing; fails
// with TBGPU_E_ARG when the launch needs more than cap blocks.
template <int NORB, int NSPIN>
static int launch_scratch_t(Ctx &c, const double *x, double *y, double shift, double *partial,
                            unsigned int *counter, int cap, double *dot_out, cudaStream_t s) {
  return c.ham_fp32
             ? launch_scratch_ht<NORB, NSPIN, float>(c, x, y, shift, partial, counter, cap, dot_out, s)
             : launch_scratch_ht<NORB, NSPIN, double>(c, x, y, shift, partial, counter, cap, dot_out, s);
}

int launch_spmv_scratch(Ctx &c, const double *x, double *y, double shift, double *partial,
                        unsigned int *counter, int cap, double *dot_out, cudaStream_t s) {
  if (c.recompute) return set_error(TBGPU_E_UNSUPPORTED);
  if (c.norb == 10 && !c.bloch)
    return launch_spmv_async_scratch(c, x, y, shift, partial, counter, cap, dot_out, s);
  if (c.norb == 10 && c.nspin == 2)
    return launch_scratch_t<10, 2>(c, x, y, shift, partial, counter, cap, dot_out, s);
  if (c.norb == 10 && c.nspin == 1)
    return launch_scratch_t<10, 1>(c, x, y, shift, partial, counter, cap, dot_out, s);
  if (c.norb == 5 && c.nspin == 2)
    return launch_scratch_t<5, 2>(c, x, y, shift, partial, counter, cap, dot_out, s);
  if (c.norb == 5 && c.nspin == 1)
    return launch_scratch_t<5, 1>(c, x, y, shift, partial, counter, cap, dot_out, s);
  return set_error(TBGPU_E_UNSUPPORTED);
}

}  // namespace tbgpu
