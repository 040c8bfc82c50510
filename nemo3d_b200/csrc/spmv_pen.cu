// H*x for the 10-orbital (sp3d5s*) models on a pencil-interleaved layout
// (H*x variant 6).
//
// Same product as k_spmv_async (spmv_async.cu; restates Hv_stored_20_Hzb,
// nemo3d/src/base/Hmult_stored.c:176-607, with the Lanczos alpha dot of
// eigen/src/lanczos.c:679-707 fused), written as the stencil it is on the
// zincblende grid.  A k-pencil of cells (i, j, 0..nz-1) holds, for each of
// the 8 sites of a cell, a line of nz atoms; every quantity is stored with
// that line's k index fastest:
//
//   vector entry (orbital q, spin s) of site m, cell (i, j, k):
//       [pencil][m][q][k][s]                       (complex)
//   bond block of cation site m (0..3), slot n, row i, columns 2c, 2c+1:
//       [pencil][m][n][i][c][k]                    (pair of real elements)
//   on-site record field f of site m:   [pencil][m][f][k]
//
// A warp takes 32/NSPIN consecutive atoms of one site's line, one lane per
// atom and spin, so every load of the warp -- a block-row pair, a neighbour's
// vector entry, an on-site field -- is one contiguous 128-512-byte run; the
// neighbour along bond n of site m sits at the same k offset for every lane
// (the zincblende neighbour map, Cell.c:599-715), so those reads are
// contiguous too.  Cation lanes stream their own blocks row by row against
// the neighbour's segment held in registers; anion lanes stream the rows of
// the blocks their cation neighbours store (each bond stored once) and
// scale them by the neighbour's entry (the transposed product).  Nothing is
// staged in shared memory.
//
// Lanczos vectors live in this layout inside the solver (lanczos.cu permutes
// the start vector in and the eigenvectors out); the C-ABI products on
// vectors in the reference's order permute around the kernel.  Empty sites
// (outside a dot's atoms) hold zero vector entries and zero blocks, so they
// contribute nothing and stay zero.  P > 1 and UPD as in spmv_lane.cu: P
// columns share every block load and compute exactly as one-column launches;
// UPD fuses the three-term update for the regenerating eigenvector pass.
#include <algorithm>
#include <atomic>
#include <vector>

#include "tbgpu_internal.cuh"
#include "lanczos_step.cuh"
#include "lane_math.cuh"
#include "reduce.cuh"
#include "stage.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

using namespace lanemath;
constexpr int kNorbP = 10;

template <typename HT> struct PairOf;
template <> struct PairOf<double> { using T = double2; };
template <> struct PairOf<float> { using T = float2; };

template <int P, typename VT>
__host__ __device__ constexpr int pen_warps() {
  return P == 1 ? 16 : (sizeof(VT) == sizeof(float2) && P == 2 ? 12 : 8);
}

struct PenGeo {
  int nx, ny, nz;
  int per_x, per_y, per_z;
  long npen;
  long nline;  // atoms of one site's lines: npen * nz
};

__host__ __device__ __forceinline__ long vidx(long p, int m, int q, int k, int s, int nz,
                                              int nspin) {
  return ((((p * 8 + m) * 10 + q) * long(nz) + k) * nspin + s);
}
__host__ __device__ __forceinline__ long bidx(long p, int m, int n, int i, int c, int k,
                                              int nz) {
  return (((((p * 4 + m) * 4 + n) * 10 + i) * 5 + c) * long(nz) + k);
}
__host__ __device__ __forceinline__ long oidx(long p, int m, int f, int k, int nz, int ons) {
  return (((p * 8 + m) * long(ons) + f) * nz + k);
}

// neighbour pencil of (i, j) along (di, dj), -1 outside a closed boundary
__device__ __forceinline__ long nb_pencil(const PenGeo &G, int i, int j, int di, int dj) {
  int ii = i + di, jj = j + dj;
  if (ii < 0 || ii >= G.nx) {
    if (!G.per_x) return -1;
    ii = (ii + G.nx) % G.nx;
  }
  if (jj < 0 || jj >= G.ny) {
    if (!G.per_y) return -1;
    jj = (jj + G.ny) % G.ny;
  }
  return long(ii) * G.ny + jj;
}
__device__ __forceinline__ int nb_k(const PenGeo &G, int k, int dk) {
  int kk = k + dk;
  if (kk < 0 || kk >= G.nz) {
    if (!G.per_z) return -1;
    kk = (kk + G.nz) % G.nz;
  }
  return kk;
}

template <typename VT, int P>
struct PenCols {
  const VT *x[P];   // input vectors (the r's; q = r * scale), pencil layout
  VT *y[P];         // output: (H - shift) q, or with UPD the next r
  const VT *rp[P];  // UPD: the r before x
  int it[P];        // scale = 1 / bet[it]; UPD: alpha[it], bet[it-1]
};

template <int NSPIN, int P, typename HT, typename VT, bool DOT, bool UPD>
__global__ void __launch_bounds__(pen_warps<P, VT>() * 32, 1)
    k_spmv_pen(PenGeo G, const unsigned char *__restrict__ ok, const HT *__restrict__ ons,
               const typename PairOf<HT>::T *__restrict__ blk, PenCols<VT, P> A,
               const double *__restrict__ bet, const double *__restrict__ alpha,
               double shift_d, double *partial, unsigned int *counter, double *alpha_out,
               int alpha_idx) {
  using RT = typename RealOf<VT>::T;
  using HT2 = typename PairOf<HT>::T;
  constexpr int W = pen_warps<P, VT>();
  constexpr int KC = 32 / NSPIN;  // atoms per warp task
  constexpr int NB = kNorbP * NSPIN;
  constexpr int ONS = onsite_len(NB);
  const int nz = G.nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ai = lane / NSPIN, s = lane - ai * NSPIN;
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
  const long nchunk = (G.nline + KC - 1) / KC;
  const long ntasks = nchunk * 8;
  const long stride = long(gridDim.x) * W;
  for (long t = long(blockIdx.x) * W + warp; t < ntasks; t += stride) {
    const int m = int(t & 7);
    const long line = (t >> 3) * KC + ai;  // position along the site's lines
    if (line >= G.nline) continue;
    const long p = line / nz;
    const int k = int(line - p * nz);
    if (!ok[(p * 8 + m) * nz + k]) continue;
    const int i = int(p / G.ny), j = int(p - long(i) * G.ny);
    VT acc[P][kNorbP];
    RT dg[kNorbP];
#pragma unroll
    for (int q = 0; q < kNorbP; q++) dg[q] = RT(ons[oidx(p, m, s * kNorbP + q, k, nz, ONS)]);
    const bool pass = ons[oidx(p, m, NB + 1, k, nz, ONS)] != HT(0);
    RT cpl[6] = {RT(0), RT(0), RT(0), RT(0), RT(0), RT(0)};
    if (pass) {
#pragma unroll
      for (int f = 0; f < 6; f++) cpl[f] = RT(ons[oidx(p, m, NB + 2 + f, k, nz, ONS)]);
    }
    const RT L = NSPIN == 2 ? RT(ons[oidx(p, m, NB, k, nz, ONS)]) : RT(0);
#pragma unroll
    for (int c = 0; c < P; c++) {
      VT xo[kNorbP];
#pragma unroll
      for (int q = 0; q < kNorbP; q++) xo[q] = A.x[c][vidx(p, m, q, k, s, nz, NSPIN)];
#pragma unroll
      for (int q = 0; q < kNorbP; q++) {
        acc[c][q].x = mul_rn(dg[q], xo[q].x);
        acc[c][q].y = mul_rn(dg[q], xo[q].y);
      }
      if (pass) {  // dangling-bond sp3 couplings (orbitals 1..4 of this spin)
        const RT sx = cpl[0], sy = cpl[1], sz = cpl[2], cxy = cpl[3], cxz = cpl[4], cyz = cpl[5];
        cfma(acc[c][1], sx, xo[2]); cfma(acc[c][1], sy, xo[3]); cfma(acc[c][1], sz, xo[4]);
        cfma(acc[c][2], sx, xo[1]); cfma(acc[c][2], cxy, xo[3]); cfma(acc[c][2], cxz, xo[4]);
        cfma(acc[c][3], sy, xo[1]); cfma(acc[c][3], cxy, xo[2]); cfma(acc[c][3], cyz, xo[4]);
        cfma(acc[c][4], sz, xo[1]); cfma(acc[c][4], cxz, xo[2]); cfma(acc[c][4], cyz, xo[3]);
      }
      if (NSPIN == 2) {  // on-site spin-orbit (mb_ham_spds_so.h): p orbitals 2..4
        const VT o2 = A.x[c][vidx(p, m, 2, k, 1 - s, nz, NSPIN)];
        const VT o3 = A.x[c][vidx(p, m, 3, k, 1 - s, nz, NSPIN)];
        const VT o4 = A.x[c][vidx(p, m, 4, k, 1 - s, nz, NSPIN)];
        if (s == 0) {  // up rows: own = U, other = D
          cfma_im(acc[c][2], -L, xo[3]); cfma(acc[c][2], L, o4);
          cfma_im(acc[c][3], L, xo[2]);  cfma_im(acc[c][3], -L, o4);
          cfma(acc[c][4], -L, o2);       cfma_im(acc[c][4], L, o3);
        } else {       // down rows: own = D, other = U
          cfma_im(acc[c][2], L, xo[3]);  cfma(acc[c][2], -L, o4);
          cfma_im(acc[c][3], -L, xo[2]); cfma_im(acc[c][3], -L, o4);
          cfma(acc[c][4], L, o2);        cfma_im(acc[c][4], L, o3);
        }
      }
    }
    if (m < 4) {
      // cation: y[r] += sum_q B_n[r][q] x_nb[q], B_n its own stored block
#pragma unroll 1
      for (int n = 0; n < 4; n++) {
        const long p2 = nb_pencil(G, i, j, c_nnmap[m][n][0], c_nnmap[m][n][1]);
        const int k2 = p2 < 0 ? -1 : nb_k(G, k, c_nnmap[m][n][2]);
        if (k2 < 0) continue;
        const int m2 = c_nnmap[m][n][3];
        VT xn[P][kNorbP];
#pragma unroll
        for (int c = 0; c < P; c++)
#pragma unroll
          for (int q = 0; q < kNorbP; q++) xn[c][q] = A.x[c][vidx(p2, m2, q, k2, s, nz, NSPIN)];
#pragma unroll
        for (int r = 0; r < kNorbP; r++) {
          HT2 b[5];
#pragma unroll
          for (int cc = 0; cc < 5; cc++) b[cc] = __ldg(blk + bidx(p, m, n, r, cc, k, nz));
#pragma unroll
          for (int c = 0; c < P; c++)
#pragma unroll
            for (int cc = 0; cc < 5; cc++) {
              cfma(acc[c][r], RT(b[cc].x), xn[c][2 * cc]);
              cfma(acc[c][r], RT(b[cc].y), xn[c][2 * cc + 1]);
            }
        }
      }
    } else {
      // anion: y[q] += sum_r B[r][q] x_nb[r], B the block its cation
      // neighbour stores for the bond (the transposed product)
#pragma unroll 1
      for (int n = 0; n < 4; n++) {
        const long p2 = nb_pencil(G, i, j, c_nnmap[m][n][0], c_nnmap[m][n][1]);
        const int k2 = p2 < 0 ? -1 : nb_k(G, k, c_nnmap[m][n][2]);
        if (k2 < 0) continue;
        const int mc = c_nnmap[m][n][3], nc = c_rev_slot[m][n];
#pragma unroll
        for (int r = 0; r < kNorbP; r++) {
          HT2 b[5];
#pragma unroll
          for (int cc = 0; cc < 5; cc++) b[cc] = __ldg(blk + bidx(p2, mc, nc, r, cc, k2, nz));
#pragma unroll
          for (int c = 0; c < P; c++) {
            const VT xc = A.x[c][vidx(p2, mc, r, k2, s, nz, NSPIN)];
#pragma unroll
            for (int cc = 0; cc < 5; cc++) {
              cfma(acc[c][2 * cc], RT(b[cc].x), xc);
              cfma(acc[c][2 * cc + 1], RT(b[cc].y), xc);
            }
          }
        }
      }
    }
    // epilogue: w = scale * acc - shift * (scale * x)
#pragma unroll
    for (int c = 0; c < P; c++) {
#pragma unroll
      for (int q = 0; q < kNorbP; q++) {
        const long e = vidx(p, m, q, k, s, nz, NSPIN);
        const VT xv = A.x[c][e];
        VT xs, out;
        xs.x = mul_rn(scale[c], xv.x);
        xs.y = mul_rn(scale[c], xv.y);
        out.x = fma_rn(scale[c], acc[c][q].x, -mul_rn(shift, xs.x));
        out.y = fma_rn(scale[c], acc[c][q].y, -mul_rn(shift, xs.y));
        if (UPD) {
          VT rpv;
          if (A.rp[c]) rpv = A.rp[c][e];
          else rpv.x = rpv.y = RT(0);
          const double2 rr = lanczos_update_entry(
              make_double2(double(out.x), double(out.y)), make_double2(double(xv.x), double(xv.y)),
              make_double2(double(rpv.x), double(rpv.y)), al[c], bp[c], iq[c], ip[c]);
          VT rv;
          rv.x = RT(rr.x);
          rv.y = RT(rr.y);
          A.y[c][e] = rv;
        } else {
          A.y[c][e] = out;
        }
        if (DOT) dot += double(xs.x) * double(out.x) + double(xs.y) * double(out.y);
      }
    }
  }
  if (DOT) grid_reduce<W * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

// ---- the same product with each warp's block rows staged (H*x variant 7) ---
//
// k_spmv_pen keeps only a few of its contiguous block-row loads in flight per
// warp and stalls on their latency.  Here every warp double-buffers the 50
// block rows (10 rows x 5 column pairs, 16 k entries each) of the bond it
// computes next in shared memory by 16-byte cp.async copies, issued while it
// computes the current bond from the other buffer: a cation's own rows at
// its 16-atom k range, or the rows its cation neighbour stores, from an even
// k start two entries early when the neighbour sits at k - 1 (entries outside
// the line are zero-filled and never read).  The arithmetic of every lane is
// k_spmv_pen's, in the same order, so the results are bit-identical and the
// solver's first pass and regenerating pass may use either kernel.  Float
// store, spin-orbit models, closed z boundary and nz a multiple of 16 (each
// 16-atom task inside one line); other contexts use k_spmv_pen.
constexpr int kStgK = 18;                       // staged k entries per row
constexpr int kStgRows = 50;                    // rows of one bond's block
constexpr int kStgBytes = kStgRows * kStgK * 8;  // one buffer (float pairs)

template <int P>
__host__ __device__ constexpr int pen_stg_warps() {
  return P == 1 ? 12 : 8;
}

template <int P, typename VT, bool DOT, bool UPD>
__global__ void __launch_bounds__(pen_stg_warps<P>() * 32, 1)
    k_spmv_pen_stg(PenGeo G, const unsigned char *__restrict__ ok, const float *__restrict__ ons,
                   const float2 *__restrict__ blk, PenCols<VT, P> A,
                   const double *__restrict__ bet, const double *__restrict__ alpha,
                   double shift_d, double *partial, unsigned int *counter, double *alpha_out,
                   int alpha_idx) {
  using RT = typename RealOf<VT>::T;
  using HT = float;
  constexpr int NSPIN = 2;
  constexpr int W = pen_stg_warps<P>();
  constexpr int KC = 16;  // atoms per warp task
  constexpr int NB = kNorbP * NSPIN;
  constexpr int ONS = onsite_len(NB);
  extern __shared__ __align__(16) unsigned char pen_stg_smem[];
  const int nz = G.nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ai = lane >> 1, s = lane & 1;
  float2 *const buf0 = reinterpret_cast<float2 *>(pen_stg_smem + size_t(warp) * 2 * kStgBytes);
  RT scale[P];
  double iq[P], ip[P], al[P], bp[P];
#pragma unroll
  for (int c = 0; c < P; c++) {
    const int it = A.it[c];
    scale[c] = RT(bet ? 1.0 / bet[it] : 1.0);
    if (UPD) {
      al[c] = alpha[it];
      bp[c] = bet[it];
      iq[c] = 1.0 / bp[c];
      ip[c] = it > 0 ? 1.0 / bet[it - 1] : 0.0;
    }
  }
  const RT shift = RT(shift_d);
  double dot = 0.0;
  const long ntasks = (G.nline / KC) * 8;
  const long stride = long(gridDim.x) * W;

  // bond n of task t has a neighbour pencil (the same for all lanes)
  auto bond_valid = [&](long t, int n) -> bool {
    const int m = int(t & 7);
    const long p = ((t >> 3) * KC) / nz;
    const int i = int(p / G.ny), j = int(p - long(i) * G.ny);
    return nb_pencil(G, i, j, c_nnmap[m][n][0], c_nnmap[m][n][1]) >= 0;
  };
  // the next bond with a neighbour pencil at or after (t, n) in this warp's
  // task order; t >= ntasks when none is left
  auto advance = [&](long &t, int &n) {
    while (t < ntasks) {
      for (; n < 4; n++)
        if (bond_valid(t, n)) return;
      t += stride;
      n = 0;
    }
  };
  // copy the 50 rows bond n of task t reads into buffer b (cooperative)
  auto issue = [&](long t, int n, float2 *b) {
    const int m = int(t & 7);
    const long L0 = (t >> 3) * KC;
    const long p = L0 / nz;
    const int k0 = int(L0 - p * nz);
    long pr = p;
    int mr = m, nr = n, kst = k0, cpr = 8;
    if (m >= 4) {
      const int i = int(p / G.ny), j = int(p - long(i) * G.ny);
      pr = nb_pencil(G, i, j, c_nnmap[m][n][0], c_nnmap[m][n][1]);
      mr = c_nnmap[m][n][3];
      nr = c_rev_slot[m][n];
      if (c_nnmap[m][n][2] < 0) {
        kst = k0 - 2;
        cpr = 9;
      }
    }
    const int total = kStgRows * cpr;
    for (int q = lane; q < total; q += 32) {
      const int row = q / cpr, part = q - row * cpr;
      const int r = row / 5, cc = row - r * 5;
      const int e = kst + 2 * part;  // even; nz even: both entries in or both out
      const bool in = e >= 0 && e < nz;
      stage::cp16z(b + row * kStgK + 2 * part, blk + bidx(pr, mr, nr, r, cc, in ? e : 0, nz),
                   in ? 16 : 0);
    }
  };

  // the copy pipeline runs one bond ahead of the computation, across tasks
  long jt = long(blockIdx.x) * W + warp;
  int jn = 0;
  advance(jt, jn);
  int cur = 0;
  if (jt < ntasks) issue(jt, jn, buf0);
  stage::cp_commit();
  for (long t = long(blockIdx.x) * W + warp; t < ntasks; t += stride) {
    const int m = int(t & 7);
    const long line = (t >> 3) * KC + ai;
    const long p = line / nz;
    const int k = int(line - p * nz);
    const int k0 = k - ai;
    const bool active = ok[(p * 8 + m) * nz + k] != 0;
    const int i = int(p / G.ny), j = int(p - long(i) * G.ny);
    VT acc[P][kNorbP];
    if (active) {
      RT dg[kNorbP];
#pragma unroll
      for (int q = 0; q < kNorbP; q++) dg[q] = RT(ons[oidx(p, m, s * kNorbP + q, k, nz, ONS)]);
      const bool pass = ons[oidx(p, m, NB + 1, k, nz, ONS)] != HT(0);
      RT cpl[6] = {RT(0), RT(0), RT(0), RT(0), RT(0), RT(0)};
      if (pass) {
#pragma unroll
        for (int f = 0; f < 6; f++) cpl[f] = RT(ons[oidx(p, m, NB + 2 + f, k, nz, ONS)]);
      }
      const RT L = RT(ons[oidx(p, m, NB, k, nz, ONS)]);
#pragma unroll
      for (int c = 0; c < P; c++) {
        VT xo[kNorbP];
#pragma unroll
        for (int q = 0; q < kNorbP; q++) xo[q] = A.x[c][vidx(p, m, q, k, s, nz, NSPIN)];
#pragma unroll
        for (int q = 0; q < kNorbP; q++) {
          acc[c][q].x = mul_rn(dg[q], xo[q].x);
          acc[c][q].y = mul_rn(dg[q], xo[q].y);
        }
        if (pass) {
          const RT sx = cpl[0], sy = cpl[1], sz = cpl[2], cxy = cpl[3], cxz = cpl[4], cyz = cpl[5];
          cfma(acc[c][1], sx, xo[2]); cfma(acc[c][1], sy, xo[3]); cfma(acc[c][1], sz, xo[4]);
          cfma(acc[c][2], sx, xo[1]); cfma(acc[c][2], cxy, xo[3]); cfma(acc[c][2], cxz, xo[4]);
          cfma(acc[c][3], sy, xo[1]); cfma(acc[c][3], cxy, xo[2]); cfma(acc[c][3], cyz, xo[4]);
          cfma(acc[c][4], sz, xo[1]); cfma(acc[c][4], cxz, xo[2]); cfma(acc[c][4], cyz, xo[3]);
        }
        {
          const VT o2 = A.x[c][vidx(p, m, 2, k, 1 - s, nz, NSPIN)];
          const VT o3 = A.x[c][vidx(p, m, 3, k, 1 - s, nz, NSPIN)];
          const VT o4 = A.x[c][vidx(p, m, 4, k, 1 - s, nz, NSPIN)];
          if (s == 0) {
            cfma_im(acc[c][2], -L, xo[3]); cfma(acc[c][2], L, o4);
            cfma_im(acc[c][3], L, xo[2]);  cfma_im(acc[c][3], -L, o4);
            cfma(acc[c][4], -L, o2);       cfma_im(acc[c][4], L, o3);
          } else {
            cfma_im(acc[c][2], L, xo[3]);  cfma(acc[c][2], -L, o4);
            cfma_im(acc[c][3], -L, xo[2]); cfma_im(acc[c][3], -L, o4);
            cfma(acc[c][4], L, o2);        cfma_im(acc[c][4], L, o3);
          }
        }
      }
    }
#pragma unroll 1
    for (int n = 0; n < 4; n++) {
      if (!bond_valid(t, n)) continue;  // warp-uniform; this bond's rows are in buffer `cur`
      long nt = jt;
      int nn = jn + 1;
      advance(nt, nn);
      if (nt < ntasks) issue(nt, nn, buf0 + (cur ^ 1) * (kStgBytes / 8));
      stage::cp_commit();
      stage::cp_wait<1>();
      __syncwarp();
      const float2 *b0 = buf0 + cur * (kStgBytes / 8);
      const long p2 = nb_pencil(G, i, j, c_nnmap[m][n][0], c_nnmap[m][n][1]);
      const int k2 = nb_k(G, k, c_nnmap[m][n][2]);
      if (active && k2 >= 0) {
        if (m < 4) {
          const int m2 = c_nnmap[m][n][3];
          VT xn[P][kNorbP];
#pragma unroll
          for (int c = 0; c < P; c++)
#pragma unroll
            for (int q = 0; q < kNorbP; q++) xn[c][q] = A.x[c][vidx(p2, m2, q, k2, s, nz, NSPIN)];
#pragma unroll
          for (int r = 0; r < kNorbP; r++) {
            float2 b[5];
#pragma unroll
            for (int cc = 0; cc < 5; cc++) b[cc] = b0[(r * 5 + cc) * kStgK + ai];
#pragma unroll
            for (int c = 0; c < P; c++)
#pragma unroll
              for (int cc = 0; cc < 5; cc++) {
                cfma(acc[c][r], RT(b[cc].x), xn[c][2 * cc]);
                cfma(acc[c][r], RT(b[cc].y), xn[c][2 * cc + 1]);
              }
          }
        } else {
          const int mc = c_nnmap[m][n][3];
          const int off = ai + (c_nnmap[m][n][2] < 0 ? 1 : 0);
#pragma unroll
          for (int r = 0; r < kNorbP; r++) {
            float2 b[5];
#pragma unroll
            for (int cc = 0; cc < 5; cc++) b[cc] = b0[(r * 5 + cc) * kStgK + off];
#pragma unroll
            for (int c = 0; c < P; c++) {
              const VT xc = A.x[c][vidx(p2, mc, r, k2, s, nz, NSPIN)];
#pragma unroll
              for (int cc = 0; cc < 5; cc++) {
                cfma(acc[c][2 * cc], RT(b[cc].x), xc);
                cfma(acc[c][2 * cc + 1], RT(b[cc].y), xc);
              }
            }
          }
        }
      }
      __syncwarp();  // the buffer is refilled two bonds on
      cur ^= 1;
      jt = nt;
      jn = nn;
    }
    (void)k0;
    if (active) {
#pragma unroll
      for (int c = 0; c < P; c++) {
#pragma unroll
        for (int q = 0; q < kNorbP; q++) {
          const long e = vidx(p, m, q, k, s, nz, NSPIN);
          const VT xv = A.x[c][e];
          VT xs, out;
          xs.x = mul_rn(scale[c], xv.x);
          xs.y = mul_rn(scale[c], xv.y);
          out.x = fma_rn(scale[c], acc[c][q].x, -mul_rn(shift, xs.x));
          out.y = fma_rn(scale[c], acc[c][q].y, -mul_rn(shift, xs.y));
          if (UPD) {
            VT rpv;
            if (A.rp[c]) rpv = A.rp[c][e];
            else rpv.x = rpv.y = RT(0);
            const double2 rr = lanczos_update_entry(
                make_double2(double(out.x), double(out.y)),
                make_double2(double(xv.x), double(xv.y)),
                make_double2(double(rpv.x), double(rpv.y)), al[c], bp[c], iq[c], ip[c]);
            VT rv;
            rv.x = RT(rr.x);
            rv.y = RT(rr.y);
            A.y[c][e] = rv;
          } else {
            A.y[c][e] = out;
          }
          if (DOT) dot += double(xs.x) * double(out.x) + double(xs.y) * double(out.y);
        }
      }
    }
  }
  stage::cp_wait<0>();
  if (DOT) grid_reduce<W * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

// ---- layout builders -------------------------------------------------------
__device__ __forceinline__ void site_coords(int site, int nz, long &p, int &k, int &m) {
  m = site & 7;
  const long cell = site >> 3;
  k = int(cell % nz);
  p = cell / nz;
}

// one thread per (cation atom, slot, row): the row's 10 elements as 5 pairs
template <typename HT>
__global__ void k_pen_blocks(long natoms, const int *__restrict__ atom_site,
                             const int4 *__restrict__ nbr, const HT *__restrict__ blocks,
                             typename PairOf<HT>::T *__restrict__ pen, int nz) {
  const long t = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (t >= natoms * 40) return;
  const long a = t / 40;
  const int r40 = int(t - a * 40), n = r40 / 10, row = r40 - n * 10;
  long p;
  int k, m;
  site_coords(atom_site[a], nz, p, k, m);
  if (m >= 4) return;
  const int4 nb = nbr[a];
  const int b = n == 0 ? nb.x : n == 1 ? nb.y : n == 2 ? nb.z : nb.w;
  if (b < 0) return;
  const HT *src = blocks + (a * 4 + n) * 100 + row * 10;
#pragma unroll
  for (int c = 0; c < 5; c++) {
    typename PairOf<HT>::T v;
    v.x = src[2 * c];
    v.y = src[2 * c + 1];
    pen[bidx(p, m, n, row, c, k, nz)] = v;
  }
}

// one thread per (atom, field): the on-site record; the site mask
template <typename HT>
__global__ void k_pen_onsite(long natoms, const int *__restrict__ atom_site,
                             const HT *__restrict__ onsite, HT *__restrict__ pen,
                             unsigned char *__restrict__ ok, int nz, int ons) {
  const long t = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (t >= natoms * ons) return;
  const long a = t / ons;
  const int f = int(t - a * ons);
  long p;
  int k, m;
  site_coords(atom_site[a], nz, p, k, m);
  pen[oidx(p, m, f, k, nz, ons)] = onsite[t];
  if (f == 0) ok[(p * 8 + m) * nz + k] = 1;
}

// reference order (atom, spin, orbital) <-> pencil layout, complex entries
template <typename VT, bool TO_PEN>
__global__ void k_pen_permute(long natoms, const int *__restrict__ atom_site, int nz, int nspin,
                              const VT *__restrict__ in, VT *__restrict__ out) {
  const int nb = 10 * nspin;
  const long t = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (t >= natoms * nb) return;
  const long a = t / nb;
  const int r = int(t - a * nb), s = r / 10, q = r - s * 10;
  long p;
  int k, m;
  site_coords(atom_site[a], nz, p, k, m);
  const long e = vidx(p, m, q, k, s, nz, nspin);
  if (TO_PEN) out[e] = in[t];
  else out[t] = in[e];
}

PenGeo pen_geo(const Ctx &c) {
  PenGeo G;
  G.nx = c.nx;
  G.ny = c.ny;
  G.nz = c.nz;
  G.per_x = c.periodic[0];
  G.per_y = c.periodic[1];
  G.per_z = c.periodic[2];
  G.npen = long(c.nx) * c.ny;
  G.nline = G.npen * c.nz;
  return G;
}

unsigned blocks_for(long n, int threads) { return unsigned((n + threads - 1) / threads); }

}  // namespace

bool pen_supported(const Ctx &c) {
  return c.norb == kNorbP && !c.bloch && !c.recompute && !c.d_skip && c.built &&
         (c.ham_fp32 ? c.d_blocks32 != nullptr : c.d_blocks != nullptr);
}

long pen_length(const Ctx &c) { return c.nsites * c.nb; }

// variant 7: the staged pencil kernel where it applies (float store,
// spin-orbit, closed z, nz a multiple of 16)
bool pen_staged(const Ctx &c) {
  return c.spmv_variant == 7 && c.ham_fp32 && c.nspin == 2 && c.nz % 16 == 0 && !c.periodic[2];
}

// the pencil layout of the stored Hamiltonian (built on first use)
static int build_pen(Ctx &c) {
  if (c.d_pen_blk && c.pen_fp32 == c.ham_fp32) return TBGPU_OK;
  if (c.d_pen_blk) cudaFree(c.d_pen_blk);
  if (c.d_pen_ons) cudaFree(c.d_pen_ons);
  if (!c.d_pen_ok && cudaMalloc(&c.d_pen_ok, size_t(c.nsites)) != cudaSuccess)
    return set_error(TBGPU_E_NOMEM);
  c.d_pen_blk = c.d_pen_ons = nullptr;
  const size_t hs = c.ham_fp32 ? sizeof(float) : sizeof(double);
  const size_t nblk = size_t(c.nsites / 2) * 400;  // cation half of the sites
  const size_t nons = size_t(c.nsites) * c.ons;
  if (cudaMalloc(&c.d_pen_blk, nblk * hs) != cudaSuccess ||
      cudaMalloc(&c.d_pen_ons, nons * hs) != cudaSuccess) {
    if (c.d_pen_blk) cudaFree(c.d_pen_blk);
    c.d_pen_blk = nullptr;
    return set_error(TBGPU_E_NOMEM);
  }
  TB_CUDA(cudaMemsetAsync(c.d_pen_blk, 0, nblk * hs, c.stream));
  TB_CUDA(cudaMemsetAsync(c.d_pen_ons, 0, nons * hs, c.stream));
  TB_CUDA(cudaMemsetAsync(c.d_pen_ok, 0, size_t(c.nsites), c.stream));
  const int T = 256;
  if (c.ham_fp32) {
    k_pen_blocks<float><<<blocks_for(c.natoms * 40, T), T, 0, c.stream>>>(
        c.natoms, c.d_atom_site, c.d_nbr, c.d_blocks32, static_cast<float2 *>(c.d_pen_blk), c.nz);
    k_pen_onsite<float><<<blocks_for(c.natoms * c.ons, T), T, 0, c.stream>>>(
        c.natoms, c.d_atom_site, c.d_onsite32, static_cast<float *>(c.d_pen_ons), c.d_pen_ok,
        c.nz, c.ons);
  } else {
    k_pen_blocks<double><<<blocks_for(c.natoms * 40, T), T, 0, c.stream>>>(
        c.natoms, c.d_atom_site, c.d_nbr, c.d_blocks, static_cast<double2 *>(c.d_pen_blk), c.nz);
    k_pen_onsite<double><<<blocks_for(c.natoms * c.ons, T), T, 0, c.stream>>>(
        c.natoms, c.d_atom_site, c.d_onsite, static_cast<double *>(c.d_pen_ons), c.d_pen_ok,
        c.nz, c.ons);
  }
  TB_CUDA(cudaGetLastError());
  c.pen_fp32 = c.ham_fp32;
  return TBGPU_OK;
}

template <typename VT>
int pen_permute(Ctx &c, const VT *in, VT *out, bool to_pen, cudaStream_t s) {
  const long n = c.natoms * c.nb;
  const int T = 256;
  if (to_pen) {
    TB_CUDA(cudaMemsetAsync(out, 0, sizeof(VT) * size_t(pen_length(c)), s));
    k_pen_permute<VT, true><<<blocks_for(n, T), T, 0, s>>>(c.natoms, c.d_atom_site, c.nz,
                                                           c.nspin, in, out);
  } else {
    k_pen_permute<VT, false><<<blocks_for(n, T), T, 0, s>>>(c.natoms, c.d_atom_site, c.nz,
                                                            c.nspin, in, out);
  }
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}
template int pen_permute<double2>(Ctx &, const double2 *, double2 *, bool, cudaStream_t);
template int pen_permute<float2>(Ctx &, const float2 *, float2 *, bool, cudaStream_t);

template <int NSPIN, int P, typename HT, typename VT, bool DOT, bool UPD>
static int launch_pen_t(Ctx &c, const PenCols<VT, P> &A, const double *bet, const double *alpha,
                        double shift, double *alpha_out, int aidx, cudaStream_t s) {
  int rc = build_pen(c);
  if (rc) return rc;
  const unsigned grid = unsigned(c.sms);
  if (DOT) {
    rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
  using HT2 = typename PairOf<HT>::T;
  if constexpr (NSPIN == 2 && sizeof(HT) == sizeof(float)) {
    if (pen_staged(c)) {
      constexpr int smem = pen_stg_warps<P>() * 2 * kStgBytes;
      static std::atomic<unsigned long long> attr_done{0};
      if (ensure_smem_attr(attr_done, c.device, k_spmv_pen_stg<P, VT, DOT, UPD>, smem))
        return TBGPU_E_CUDA;
      k_spmv_pen_stg<P, VT, DOT, UPD><<<grid, pen_stg_warps<P>() * 32, smem, s>>>(
          pen_geo(c), c.d_pen_ok, static_cast<const float *>(c.d_pen_ons),
          static_cast<const float2 *>(c.d_pen_blk), A, bet, alpha, shift,
          DOT ? c.d_partial : nullptr, DOT ? c.d_counter : nullptr, alpha_out, aidx);
      TB_CUDA(cudaGetLastError());
      return TBGPU_OK;
    }
  }
  k_spmv_pen<NSPIN, P, HT, VT, DOT, UPD><<<grid, pen_warps<P, VT>() * 32, 0, s>>>(
      pen_geo(c), c.d_pen_ok, static_cast<const HT *>(c.d_pen_ons),
      static_cast<const HT2 *>(c.d_pen_blk), A, bet, alpha, shift, DOT ? c.d_partial : nullptr,
      DOT ? c.d_counter : nullptr, alpha_out, aidx);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// one product on pencil-layout vectors (the solver's), alpha fused when
// alpha_out is given
template <typename VT>
int launch_spmv_pen_internal(Ctx &c, const VT *x, VT *y, double shift, const double *xnorm,
                             int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (!pen_supported(c)) return set_error(TBGPU_E_UNSUPPORTED);
  constexpr bool F32 = sizeof(VT) == sizeof(float2);
  if (F32 && !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  PenCols<VT, 1> A{};
  A.x[0] = x;
  A.y[0] = y;
  A.rp[0] = nullptr;
  A.it[0] = xidx;
#define TBGPU_PEN1(HT)                                                                         \
  return c.nspin == 2                                                                         \
             ? (alpha_out ? launch_pen_t<2, 1, HT, VT, true, false>(c, A, xnorm, nullptr, shift, alpha_out, aidx, s) \
                          : launch_pen_t<2, 1, HT, VT, false, false>(c, A, xnorm, nullptr, shift, nullptr, 0, s)) \
             : (alpha_out ? launch_pen_t<1, 1, HT, VT, true, false>(c, A, xnorm, nullptr, shift, alpha_out, aidx, s) \
                          : launch_pen_t<1, 1, HT, VT, false, false>(c, A, xnorm, nullptr, shift, nullptr, 0, s));
  if (c.ham_fp32) {
    TBGPU_PEN1(float)
  }
  if constexpr (!F32) {
    TBGPU_PEN1(double)
  }
#undef TBGPU_PEN1
  return set_error(TBGPU_E_UNSUPPORTED);
}
template int launch_spmv_pen_internal<double2>(Ctx &, const double2 *, double2 *, double,
                                               const double *, int, double *, int, cudaStream_t);
template int launch_spmv_pen_internal<float2>(Ctx &, const float2 *, float2 *, double,
                                              const double *, int, double *, int, cudaStream_t);

// the product on vectors in the reference's order (C-ABI entry points):
// permuted into context scratch, multiplied, permuted back
template <typename VT>
static int launch_pen_ref(Ctx &c, const VT *x, VT *y, double shift, const double *xnorm,
                          int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  const size_t bytes = sizeof(VT) * size_t(pen_length(c));
  if (c.pen_scratch_bytes < 2 * bytes) {
    if (c.d_pen_scratch) cudaFree(c.d_pen_scratch);
    c.d_pen_scratch = nullptr;
    c.pen_scratch_bytes = 0;
    if (cudaMalloc(&c.d_pen_scratch, 2 * bytes) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
    c.pen_scratch_bytes = 2 * bytes;
  }
  VT *px = static_cast<VT *>(c.d_pen_scratch);
  VT *py = px + pen_length(c);
  int rc = pen_permute<VT>(c, x, px, true, s);
  if (!rc) rc = launch_spmv_pen_internal<VT>(c, px, py, shift, xnorm, xidx, alpha_out, aidx, s);
  if (!rc) rc = pen_permute<VT>(c, py, y, false, s);
  return rc;
}

int launch_spmv_pen(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                    int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (!pen_supported(c)) return set_error(TBGPU_E_UNSUPPORTED);
  return launch_pen_ref<double2>(c, reinterpret_cast<const double2 *>(x),
                                 reinterpret_cast<double2 *>(y), shift, xnorm, xidx, alpha_out,
                                 aidx, s);
}

int launch_spmv_pen_f32(Ctx &c, const float *x, float *y, double shift, const double *xnorm,
                        int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (!pen_supported(c) || !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  return launch_pen_ref<float2>(c, reinterpret_cast<const float2 *>(x),
                                reinterpret_cast<float2 *>(y), shift, xnorm, xidx, alpha_out,
                                aidx, s);
}

// p Lanczos segments advanced by one step in one pass on pencil-layout
// vectors (as launch_lane_regen)
template <typename VT>
int launch_pen_regen(Ctx &c, int p, const VT *const *x, VT *const *y, const VT *const *rp,
                     const int *it, const double *bet, const double *alpha, cudaStream_t s) {
  constexpr bool F32 = sizeof(VT) == sizeof(float2);
  if (!pen_supported(c) || p < 1 || p > lane_max_cols(F32)) return set_error(TBGPU_E_UNSUPPORTED);
  if (F32 && !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
#define TBGPU_PREGEN(PP)                                                                      \
  {                                                                                           \
    PenCols<VT, PP> A{};                                                                      \
    for (int j = 0; j < PP; j++) {                                                            \
      A.x[j] = x[j];                                                                          \
      A.y[j] = y[j];                                                                          \
      A.rp[j] = rp[j];                                                                        \
      A.it[j] = it[j];                                                                        \
    }                                                                                         \
    if (c.ham_fp32)                                                                           \
      return c.nspin == 2                                                                     \
                 ? launch_pen_t<2, PP, float, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s) \
                 : launch_pen_t<1, PP, float, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s); \
    if constexpr (!F32)                                                                       \
      return c.nspin == 2                                                                     \
                 ? launch_pen_t<2, PP, double, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s) \
                 : launch_pen_t<1, PP, double, VT, false, true>(c, A, bet, alpha, 0.0, nullptr, 0, s); \
    return set_error(TBGPU_E_UNSUPPORTED);                                                    \
  }
  switch (p) {
    case 1: TBGPU_PREGEN(1)
    case 2: TBGPU_PREGEN(2)
    case 3:
      if constexpr (F32) TBGPU_PREGEN(3)
      break;
    case 4:
      if constexpr (F32) TBGPU_PREGEN(4)
      break;
    default: break;
  }
#undef TBGPU_PREGEN
  return set_error(TBGPU_E_UNSUPPORTED);
}
template int launch_pen_regen<double2>(Ctx &, int, const double2 *const *, double2 *const *,
                                       const double2 *const *, const int *, const double *,
                                       const double *, cudaStream_t);
template int launch_pen_regen<float2>(Ctx &, int, const float2 *const *, float2 *const *,
                                      const float2 *const *, const int *, const double *,
                                      const double *, cudaStream_t);

}  // namespace tbgpu
