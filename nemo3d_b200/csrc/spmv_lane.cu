// H*x for the 10-orbital (sp3d5s*) models with one lane per (atom, spin).
//
// Same product as k_spmv_async (spmv_async.cu; restates Hv_stored_20_Hzb,
// nemo3d/src/base/Hmult_stored.c:176-607, with the Lanczos alpha dot of
// eigen/src/lanczos.c:679-707 fused), laid out so that the bytes of H reach
// the FMAs without a detour through shared memory:
//
//  * a warp takes one task of 32/NSPIN atoms of one kind (all cations or all
//    anions of one k-pencil of cells), one lane per atom and spin;
//  * a cation lane holds its neighbour's x segment (10 complex, one spin) in
//    registers and streams the rows of its own four bond blocks (one
//    contiguous 3200-byte run per atom in double) with 128-bit read-only
//    loads; an anion lane streams the rows of the four blocks its cation
//    neighbours store and scales each row by the neighbour's x entry (the
//    transposed product), so both read every block row-major and contiguous;
//  * the two spin lanes of an atom read the same block rows in the same
//    instruction (one request), and every block element is used by the lane
//    that loaded it only: nothing is staged, broadcast or shuffled.
//
// Per atom and product that is 400 block elements, 4 x 10 neighbour x
// entries and the on-site record per lane pair, against ~5 kB written to and
// ~13 kB read back from shared memory by the warp-staged kernel.
//
// P > 1 applies the same H to P independent vectors ("columns") in one pass:
// each block row loaded once feeds P columns, and every column's arithmetic
// is exactly that of the P = 1 kernel (same operations in the same order),
// so a column's result is bit-identical to a one-column launch.  UPD fuses
// the Lanczos three-term update into the epilogue (with alpha and beta of
// an earlier run), which the eigenvector pass uses to regenerate several
// segments of the recurrence at once (lanczos.cu).
//
// Work order: tasks of one kind and one pencil, cations then anions of a
// pencil, pencils visited j-block by j-block (the rows of blocks an anion
// reads were read by its cation neighbours' lanes shortly before, so the
// second read is an L2 hit).
#include <algorithm>
#include <atomic>
#include <vector>

#include "tbgpu_internal.cuh"
#include "lanczos_step.cuh"
#include "lane_math.cuh"
#include "reduce.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

using namespace lanemath;
constexpr int kNorbL = 10;
// warps per CTA (one CTA per SM): 16 for one column (128 registers a
// thread); several columns hold more accumulators and neighbour segments,
// and take fewer, larger threads instead of spilling
template <int P, typename VT>
__host__ __device__ constexpr int lane_warps() {
  return P == 1 ? 16 : (sizeof(VT) == sizeof(float2) && P == 2 ? 12 : 8);
}

template <typename VT, int P>
struct LaneCols {
  const VT *x[P];        // input vectors (the r's; q = r * scale)
  VT *y[P];              // output: (H - shift) q, or with UPD the next r
  const VT *rp[P];       // UPD: the r before x
  int it[P];             // scale = 1 / bet[it]; UPD: alpha[it], bet[it-1]
};

template <int NSPIN, int P, typename HT, typename VT, bool DOT, bool UPD>
__global__ void __launch_bounds__(lane_warps<P, VT>() * 32, 1)
    k_spmv_lane(long ntasks, const int *__restrict__ tasks, const int4 *__restrict__ nbr,
                const unsigned char *__restrict__ site_m, const HT *__restrict__ onsite,
                const HT *__restrict__ blocks, LaneCols<VT, P> A,
                const double *__restrict__ bet, const double *__restrict__ alpha,
                double shift_d, double *partial, unsigned int *counter, double *alpha_out,
                int alpha_idx, const unsigned char *__restrict__ skip) {
  using RT = typename RealOf<VT>::T;
  constexpr int kLaneWarps = lane_warps<P, VT>();
  constexpr int NB = kNorbL * NSPIN;
  constexpr int ONS = onsite_len(NB);
  constexpr int APW = 32 / NSPIN;  // atoms per task
  constexpr int BLK = kNorbL * kNorbL;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ai = lane / NSPIN, sp = lane - ai * NSPIN;
  RT scale[P];
  double iq[P], ip[P], al[P], bp[P];
#pragma unroll
  for (int c = 0; c < P; c++) {
    const int it = A.it[c];
    scale[c] = RT(bet ? 1.0 / bet[it] : 1.0);
    if (UPD) {  // as k_update: alpha[it], bet[it], bet[it-1]
      al[c] = alpha[it];
      bp[c] = bet[it];
      iq[c] = 1.0 / bp[c];
      ip[c] = it > 0 ? 1.0 / bet[it - 1] : 0.0;
    }
  }
  const RT shift = RT(shift_d);
  double dot = 0.0;
  const long stride = long(gridDim.x) * kLaneWarps;
  for (long t = long(blockIdx.x) * kLaneWarps + warp; t < ntasks; t += stride) {
    const int a = tasks[t * APW + ai];
    if (a < 0 || (skip && skip[a])) continue;
    const int m = site_m[a];
    const int4 nb4 = nbr[a];
    const int nbv[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
    const long own = long(a) * NB + sp * kNorbL;
    const HT *rec = onsite + long(a) * ONS;
    VT acc[P][kNorbL];
    // on-site diagonal
    RT dg[kNorbL];
#pragma unroll
    for (int i = 0; i < kNorbL; i++) dg[i] = RT(rec[sp * kNorbL + i]);
#pragma unroll
    for (int c = 0; c < P; c++) {
      VT xo[kNorbL];
      load_seg(A.x[c] + own, xo);
#pragma unroll
      for (int i = 0; i < kNorbL; i++) {
        acc[c][i].x = mul_rn(dg[i], xo[i].x);
        acc[c][i].y = mul_rn(dg[i], xo[i].y);
      }
      // dangling-bond sp3 couplings (orbitals 1..4 of this spin)
      if (rec[NB + 1] != HT(0)) {
        const RT sx = RT(rec[NB + 2]), sy = RT(rec[NB + 3]), sz = RT(rec[NB + 4]);
        const RT cxy = RT(rec[NB + 5]), cxz = RT(rec[NB + 6]), cyz = RT(rec[NB + 7]);
        cfma(acc[c][1], sx, xo[2]); cfma(acc[c][1], sy, xo[3]); cfma(acc[c][1], sz, xo[4]);
        cfma(acc[c][2], sx, xo[1]); cfma(acc[c][2], cxy, xo[3]); cfma(acc[c][2], cxz, xo[4]);
        cfma(acc[c][3], sy, xo[1]); cfma(acc[c][3], cxy, xo[2]); cfma(acc[c][3], cyz, xo[4]);
        cfma(acc[c][4], sz, xo[1]); cfma(acc[c][4], cxz, xo[2]); cfma(acc[c][4], cyz, xo[3]);
      }
      if (NSPIN == 2) {  // on-site spin-orbit (mb_ham_spds_so.h): p orbitals 2..4
        const RT L = RT(rec[NB]);
        const VT *other = A.x[c] + long(a) * NB + (1 - sp) * kNorbL;
        const VT o2 = other[2], o3 = other[3], o4 = other[4];
        if (sp == 0) {  // up rows: own = U, other = D
          cfma_im(acc[c][2], -L, xo[3]); cfma(acc[c][2], L, o4);
          cfma_im(acc[c][3], L, xo[2]);  cfma_im(acc[c][3], -L, o4);
          cfma(acc[c][4], -L, o2);       cfma_im(acc[c][4], L, o3);
        } else {        // down rows: own = D, other = U
          cfma_im(acc[c][2], L, xo[3]);  cfma(acc[c][2], -L, o4);
          cfma_im(acc[c][3], -L, xo[2]); cfma_im(acc[c][3], -L, o4);
          cfma(acc[c][4], L, o2);        cfma_im(acc[c][4], L, o3);
        }
      }
    }
    if (m < 4) {
      // cation: y_a[i] += sum_k B_n[i][k] x_nb[k], B_n its own stored block
#pragma unroll 1
      for (int n = 0; n < 4; n++) {
        const int b = nbv[n];
        if (b < 0) continue;
        VT xn[P][kNorbL];
#pragma unroll
        for (int c = 0; c < P; c++) load_seg(A.x[c] + long(b) * NB + sp * kNorbL, xn[c]);
        const HT *blk = blocks + (long(a) * 4 + n) * BLK;
#pragma unroll
        for (int i = 0; i < kNorbL; i += 2) {
          HT r[20];
          load_rows2(blk + i * kNorbL, r);
#pragma unroll
          for (int c = 0; c < P; c++)
#pragma unroll
            for (int k = 0; k < kNorbL; k++) {
              cfma(acc[c][i], RT(r[k]), xn[c][k]);
              cfma(acc[c][i + 1], RT(r[kNorbL + k]), xn[c][k]);
            }
        }
      }
    } else {
      // anion: y_a[k] += sum_i B[i][k] x_nb[i], B the block its cation
      // neighbour stores for the bond (the transposed product)
#pragma unroll 1
      for (int n = 0; n < 4; n++) {
        const int b = nbv[n];
        if (b < 0) continue;
        const HT *blk = blocks + (long(b) * 4 + c_rev_slot[m][n]) * BLK;
        const VT *xb[P];
#pragma unroll
        for (int c = 0; c < P; c++) xb[c] = A.x[c] + long(b) * NB + sp * kNorbL;
#pragma unroll
        for (int i = 0; i < kNorbL; i += 2) {
          HT r[20];
          load_rows2(blk + i * kNorbL, r);
#pragma unroll
          for (int c = 0; c < P; c++) {
            VT x0, x1;
            load_pair(xb[c] + i, x0, x1);
#pragma unroll
            for (int k = 0; k < kNorbL; k++) {
              cfma(acc[c][k], RT(r[k]), x0);
              cfma(acc[c][k], RT(r[kNorbL + k]), x1);
            }
          }
        }
      }
    }
    // epilogue: w = scale * acc - shift * (scale * x)
#pragma unroll
    for (int c = 0; c < P; c++) {
      VT xo[kNorbL];
      load_seg(A.x[c] + own, xo);
      VT rpv[kNorbL];
      if (UPD) {
        if (A.rp[c]) load_seg(A.rp[c] + own, rpv);
#pragma unroll
        for (int i = 0; i < kNorbL; i++)
          if (!A.rp[c]) rpv[i].x = rpv[i].y = RT(0);
      }
#pragma unroll
      for (int i = 0; i < kNorbL; i++) {
        VT xs, out;
        xs.x = mul_rn(scale[c], xo[i].x);
        xs.y = mul_rn(scale[c], xo[i].y);
        out.x = fma_rn(scale[c], acc[c][i].x, -mul_rn(shift, xs.x));
        out.y = fma_rn(scale[c], acc[c][i].y, -mul_rn(shift, xs.y));
        if (UPD) {
          const double2 r = lanczos_update_entry(
              make_double2(double(out.x), double(out.y)),
              make_double2(double(xo[i].x), double(xo[i].y)),
              make_double2(double(rpv[i].x), double(rpv[i].y)), al[c], bp[c], iq[c], ip[c]);
          VT rv;
          rv.x = RT(r.x);
          rv.y = RT(r.y);
          A.y[c][own + i] = rv;
        } else {
          A.y[c][own + i] = out;
        }
        if (DOT) dot += double(xs.x) * double(out.x) + double(xs.y) * double(out.y);
      }
    }
  }
  if (DOT) grid_reduce<kLaneWarps * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

}  // namespace

// ---------------------------------------------------------------------------
// Task list: per pencil of cells, its cations in atom order in tasks of
// 32/nspin atoms, then its anions; pencils j-block by j-block.
static int build_lane_tasks(Ctx &c) {
  const int apw = 32 / c.nspin;
  if (c.d_lane_tasks && c.lane_apw == apw) return TBGPU_OK;
  std::vector<int> site(c.natoms);
  TB_CUDA(cudaMemcpyAsync(site.data(), c.d_atom_site, sizeof(int) * c.natoms,
                          cudaMemcpyDeviceToHost, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  const long npen = long(c.nx) * c.ny;
  const long per_pen = long(c.nz) * 8;
  std::vector<int> start(npen + 1, 0);  // atoms are in site order: pencils are runs
  {
    long a = 0;
    for (long p = 0; p < npen; p++) {
      start[p] = int(a);
      while (a < c.natoms && site[a] / per_pen == p) a++;
    }
    start[npen] = int(c.natoms);
  }
  const int jb_w = std::max(1, std::min(c.lane_jblock > 0 ? c.lane_jblock : 8, c.ny));
  std::vector<int> tasks;
  tasks.reserve(size_t(c.natoms) * 2 + size_t(npen) * 2 * apw);
  std::vector<int> kind[2];
  for (int jb = 0; jb < c.ny; jb += jb_w)
    for (int i = 0; i < c.nx; i++)
      for (int j = jb; j < jb + jb_w && j < c.ny; j++) {
        const long p = long(i) * c.ny + j;
        kind[0].clear();
        kind[1].clear();
        for (int a = start[p]; a < start[p + 1]; a++) kind[(site[a] & 7) >= 4].push_back(a);
        for (int k = 0; k < 2; k++)
          for (size_t q = 0; q < kind[k].size(); q += apw)
            for (int l = 0; l < apw; l++)
              tasks.push_back(q + l < kind[k].size() ? kind[k][q + l] : -1);
      }
  if (c.d_lane_tasks) cudaFree(c.d_lane_tasks);
  c.d_lane_tasks = nullptr;
  TB_CUDA(cudaMalloc(&c.d_lane_tasks, sizeof(int) * tasks.size()));
  TB_CUDA(cudaMemcpyAsync(c.d_lane_tasks, tasks.data(), sizeof(int) * tasks.size(),
                          cudaMemcpyHostToDevice, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  c.lane_ntasks = long(tasks.size()) / apw;
  c.lane_apw = apw;
  return TBGPU_OK;
}

template <int NSPIN, int P, typename HT, typename VT, bool DOT, bool UPD>
static int launch_lane_t(Ctx &c, const LaneCols<VT, P> &A, const double *bet,
                         const double *alpha, double shift, double *alpha_out, int aidx,
                         cudaStream_t s) {
  int rc = build_lane_tasks(c);
  if (rc) return rc;
  const unsigned grid = unsigned(c.sms);
  if (DOT) {
    rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
  k_spmv_lane<NSPIN, P, HT, VT, DOT, UPD><<<grid, lane_warps<P, VT>() * 32, 0, s>>>(
      c.lane_ntasks, c.d_lane_tasks, c.d_nbr, c.d_site_m, ham_onsite<HT>(c), ham_blocks<HT>(c),
      A, bet, alpha, shift, DOT ? c.d_partial : nullptr, DOT ? c.d_counter : nullptr,
      alpha_out, aidx, c.d_skip);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

template <typename HT, typename VT>
static int launch_lane_one(Ctx &c, const VT *x, VT *y, double shift, const double *xnorm,
                           int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  LaneCols<VT, 1> A{};
  A.x[0] = x;
  A.y[0] = y;
  A.rp[0] = nullptr;
  A.it[0] = xidx;
  if (c.nspin == 2)
    return alpha_out
               ? launch_lane_t<2, 1, HT, VT, true, false>(c, A, xnorm, nullptr, shift, alpha_out, aidx, s)
               : launch_lane_t<2, 1, HT, VT, false, false>(c, A, xnorm, nullptr, shift, nullptr, 0, s);
  return alpha_out
             ? launch_lane_t<1, 1, HT, VT, true, false>(c, A, xnorm, nullptr, shift, alpha_out, aidx, s)
             : launch_lane_t<1, 1, HT, VT, false, false>(c, A, xnorm, nullptr, shift, nullptr, 0, s);
}

bool lane_supported(const Ctx &c) {
  return c.norb == kNorbL && !c.bloch && !c.recompute;
}

int launch_spmv_lane(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                     int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (!lane_supported(c)) return set_error(TBGPU_E_UNSUPPORTED);
  const double2 *X = reinterpret_cast<const double2 *>(x);
  double2 *Y = reinterpret_cast<double2 *>(y);
  if (c.ham_fp32)
    return launch_lane_one<float, double2>(c, X, Y, shift, xnorm, xidx, alpha_out, aidx, s);
  return launch_lane_one<double, double2>(c, X, Y, shift, xnorm, xidx, alpha_out, aidx, s);
}

int launch_spmv_lane_f32(Ctx &c, const float *x, float *y, double shift, const double *xnorm,
                         int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (!lane_supported(c) || !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  return launch_lane_one<float, float2>(c, reinterpret_cast<const float2 *>(x),
                                        reinterpret_cast<float2 *>(y), shift, xnorm, xidx,
                                        alpha_out, aidx, s);
}

// Regeneration of p Lanczos segments in one pass (p <= lane_max_cols): column j
// takes r = x[j] at iteration it[j] (q = r / bet[it]) and r_prev = rp[j]
// (null at it = 0) and writes the next r, exactly as one k_spmv_lane launch
// followed by k_update would.
template <typename VT>
int launch_lane_regen(Ctx &c, int p, const VT *const *x, VT *const *y, const VT *const *rp,
                      const int *it, const double *bet, const double *alpha, cudaStream_t s) {
  constexpr bool F32 = sizeof(VT) == sizeof(float2);
  if (!lane_supported(c) || p < 1 || p > lane_max_cols(F32)) return set_error(TBGPU_E_UNSUPPORTED);
  if (F32 && !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
#define TBGPU_REGEN(PP)                                                                       \
  {                                                                                           \
    LaneCols<VT, PP> A{};                                                                     \
    for (int j = 0; j < PP; j++) {                                                            \
      A.x[j] = x[j];                                                                          \
      A.y[j] = y[j];                                                                          \
      A.rp[j] = rp[j];                                                                        \
      A.it[j] = it[j];                                                                        \
    }                                                                                         \
    if (c.ham_fp32)                                                                           \
      return c.nspin == 2                                                                     \
                 ? launch_lane_t<2, PP, float, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s) \
                 : launch_lane_t<1, PP, float, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s); \
    if constexpr (!F32)                                                                       \
      return c.nspin == 2                                                                     \
                 ? launch_lane_t<2, PP, double, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s) \
                 : launch_lane_t<1, PP, double, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s); \
    return set_error(TBGPU_E_UNSUPPORTED);                                                    \
  }
  switch (p) {
    case 1: TBGPU_REGEN(1)
    case 2: TBGPU_REGEN(2)
    case 3:
      if constexpr (F32) TBGPU_REGEN(3)
      break;
    case 4:
      if constexpr (F32) TBGPU_REGEN(4)
      break;
    default: break;
  }
#undef TBGPU_REGEN
  return set_error(TBGPU_E_UNSUPPORTED);
}

template int launch_lane_regen<double2>(Ctx &, int, const double2 *const *, double2 *const *,
                                        const double2 *const *, const int *, const double *,
                                        const double *, cudaStream_t);
template int launch_lane_regen<float2>(Ctx &, int, const float2 *const *, float2 *const *,
                                       const float2 *const *, const int *, const double *,
                                       const double *, cudaStream_t);

}  // namespace tbgpu
