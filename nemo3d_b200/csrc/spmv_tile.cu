// H*x for the 10-orbital models over units of two cells (H*x variant 3).
//
// The same product as k_spmv_async (spmv_async.cu; Hv_stored_20_Hzb,
// nemo3d/src/base/Hmult_stored.c:176-607, with the Lanczos alpha dot of
// eigen/src/lanczos.c:679-707 fused) and the same per-lane arithmetic in the
// same order, so y is bit-identical; what changes is how the bytes reach
// shared memory.  A CTA of five warps takes a unit of up to 16 atoms: two
// consecutive cells of one k-pencil.  The unit's on-site records, its own
// vector segments and, per cell, the contiguous run of its cations' bond
// blocks are single 1-D bulk copies (cp.async.bulk, completion counted on an
// mbarrier, no multicast), which cost the load/store unit nothing; the
// pieces outside the unit (a block an anion reads from a cation of another
// cell, a neighbour's vector segment from another cell) are staged once per
// unit with 16-byte cp.async.  A bond inside the unit reads its block or
// segment where the unit already holds it.  Per atom the load/store unit
// moves about 1.4 kB instead of the 5 kB of the three-atom groups.
//
// The unit table (first atom, count, cation runs, per atom its site and per
// slot the stage offsets of its neighbour's segment and of the bond block,
// and the out-of-unit pieces to copy) is built once per context on the host.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "reduce.cuh"
#include "stage.cuh"
#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

using namespace stage;
constexpr int kNorbT = 10;
constexpr int kUnitAtoms = 16;                     // two cells
constexpr int kTileThreads = kUnitAtoms * kNorbT;  // one lane per orbital row
constexpr int kBlkBytes = kNorbT * kNorbT * 8;     // one bond block (800 B)
constexpr int kCatRun = 4 * 4 * kBlkBytes;         // a cell's four cations' blocks
// unit descriptor (ints): header {first atom, count, first cation and
// cation count of cell 0, of cell 1, out-of-unit blocks, out-of-unit
// segments}; per atom its in-cell site; per atom and slot the stage offsets
// of the neighbour's segment and of the bond block (-1: no neighbour); the
// out-of-unit block indices (atom * 4 + slot) and segment atoms
constexpr int kHdr = 8;
constexpr int kOffM = kHdr, kOffX = kOffM + kUnitAtoms, kOffB = kOffX + 4 * kUnitAtoms;
constexpr int kOffItems = kOffB + 4 * kUnitAtoms;

// the arithmetic helpers of k_spmv_async, so both kernels round alike
__device__ __forceinline__ void cfma_r(double2 &acc, double v, double2 a) {
  acc.x = fma(v, a.x, acc.x);
  acc.y = fma(v, a.y, acc.y);
}
__device__ __forceinline__ void cfma_i(double2 &acc, double lam, double2 a) {
  acc.x -= lam * a.y;
  acc.y += lam * a.x;
}

template <int NSPIN>
struct TileLayout {
  static constexpr int NB = kNorbT * NSPIN;
  static constexpr int ONS = onsite_len(NB);
  static constexpr int XS = NB * 16;  // one vector segment (bytes)
  static constexpr int OS = ONS * 8;  // one on-site record (bytes)
  static constexpr int X_CH = XS / 16, BLK_CH = kBlkBytes / 16;
  // stage regions (byte offsets): on-site records, own segments, cation
  // runs of the two cells, out-of-unit blocks, out-of-unit segments
  static constexpr int ons = 0;
  static constexpr int xo = ons + kUnitAtoms * OS;
  static constexpr int cb = xo + kUnitAtoms * XS;
  static constexpr int nb = cb + 2 * kCatRun;
  __host__ __device__ static constexpr int nx(int cap_nb) { return nb + cap_nb * kBlkBytes; }
  __host__ __device__ static constexpr int bytes(int cap_nb, int cap_nx) { return nx(cap_nb) + cap_nx * XS; }
};

// descriptor area of the dynamic shared memory, then 128 bytes for the
// mbarrier, then the stage
__host__ __device__ constexpr int desc_bytes(int stride) { return ((stride * 4 + 127) / 128) * 128; }

template <int NSPIN, bool DOT>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_spmv_tile(long nunits, const int *__restrict__ desc, int dstride, int cap_nb,
                const double *__restrict__ onsite, const double *__restrict__ blocks,
                const double2 *__restrict__ x, double2 *__restrict__ y, double shift,
                const double *__restrict__ xnorm, int xnorm_idx, double *partial,
                unsigned int *counter, double *alpha_out, int alpha_idx, int *status) {
  using L = TileLayout<NSPIN>;
  constexpr int NB = L::NB;
  extern __shared__ __align__(128) unsigned char smem[];
  int *dsm = reinterpret_cast<int *>(smem);
  unsigned char *st = smem + desc_bytes(dstride) + 128;
  const uint32_t mb = smem_addr(smem + desc_bytes(dstride));
  const int t = threadIdx.x;
  const int nx_base = L::nx(cap_nb);
  const double scale = xnorm ? 1.0 / xnorm[xnorm_idx] : 1.0;
  double dot = 0.0;
  if (t == 0) {
    mbar_init(mb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t parity = 0;
  for (long u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int *dg = desc + u * dstride;
    for (int k = t; k < dstride; k += kTileThreads) dsm[k] = __ldg(dg + k);
    __syncthreads();
    const int a0 = dsm[0], count = dsm[1], nnb = dsm[6], nnx = dsm[7];
    if (t == 0) {  // the unit's contiguous pieces: bulk copies
      const uint32_t sbase = smem_addr(st);
      const uint32_t cat0 = uint32_t(dsm[3]) * 4 * kBlkBytes;
      const uint32_t cat1 = uint32_t(dsm[5]) * 4 * kBlkBytes;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(mb, uint32_t(count) * (L::OS + L::XS) + cat0 + cat1);
      bulk_g2s(sbase + L::ons, onsite + long(a0) * L::ONS, uint32_t(count) * L::OS, mb);
      bulk_g2s(sbase + L::xo, x + long(a0) * NB, uint32_t(count) * L::XS, mb);
      if (cat0) bulk_g2s(sbase + L::cb, blocks + long(dsm[2]) * 400, cat0, mb);
      if (cat1) bulk_g2s(sbase + L::cb + kCatRun, blocks + long(dsm[4]) * 400, cat1, mb);
    }
    // the out-of-unit pieces: 16-byte copies, blocks then segments
    const int nbch = nnb * L::BLK_CH, total_ch = nbch + nnx * L::X_CH;
    for (int ch = t; ch < total_ch; ch += kTileThreads) {
      if (ch < nbch) {
        const int item = ch / L::BLK_CH, k = ch - item * L::BLK_CH;
        const unsigned char *src =
            reinterpret_cast<const unsigned char *>(blocks + long(dsm[kOffItems + item]) * 100);
        cp16(st + L::nb + item * kBlkBytes + k * 16, src + k * 16);
      } else {
        const int c2 = ch - nbch;
        const int item = c2 / L::X_CH, k = c2 - item * L::X_CH;
        const unsigned char *src = reinterpret_cast<const unsigned char *>(
            x + long(dsm[kOffItems + cap_nb + item]) * NB);
        cp16(st + nx_base + item * L::XS + k * 16, src + k * 16);
      }
    }
    cp_commit();
    cp_wait<0>();
    const bool late = !mbar_wait(mb, parity);
    if (__syncthreads_or(late)) {
      // a bulk copy that did not complete: report it, give the copies in
      // flight one more bounded wait, and stop (the decision is block-wide,
      // so no thread issues another copy; if the second wait also runs out
      // the CTA ends with that copy outstanding, reported by the status word)
      if (t == 0) atomicExch(status, TBGPU_E_TIMEOUT);
      mbar_wait(mb, parity);
      break;
    }
    parity ^= 1u;
    if (t < count * kNorbT) {
      const int i = t / kNorbT, o = t - i * kNorbT;
      const long a = long(a0) + i;
      const bool cat = dsm[kOffM + i] < 4;
      const double2 *X0 = reinterpret_cast<const double2 *>(st + L::xo) + i * NB;
      const double *rec = reinterpret_cast<const double *>(st + L::ons) + i * L::ONS;
      double2 acc[NSPIN];
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const double2 v = X0[sp * kNorbT + o];
        const double dg = rec[sp * kNorbT + o];
        acc[sp].x = dg * v.x;
        acc[sp].y = dg * v.y;
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
          cfma_r(acc[sp], c1, X0[sp * kNorbT + k1]);
          cfma_r(acc[sp], c2, X0[sp * kNorbT + k2]);
          cfma_r(acc[sp], c3, X0[sp * kNorbT + k3]);
        }
      }
      if (NSPIN == 2 && o >= 2 && o <= 4) {  // on-site spin-orbit (mb_ham_spds_so.h)
        const double Lm = rec[NB];
        const double2 *U = X0, *D = X0 + kNorbT;
        if (o == 2) {
          cfma_i(acc[0], -Lm, U[3]); cfma_r(acc[0], Lm, D[4]);
          cfma_i(acc[NSPIN - 1], Lm, D[3]); cfma_r(acc[NSPIN - 1], -Lm, U[4]);
        } else if (o == 3) {
          cfma_i(acc[0], Lm, U[2]); cfma_i(acc[0], -Lm, D[4]);
          cfma_i(acc[NSPIN - 1], -Lm, D[2]); cfma_i(acc[NSPIN - 1], -Lm, U[4]);
        } else {
          cfma_r(acc[0], -Lm, D[2]); cfma_i(acc[0], Lm, D[3]);
          cfma_r(acc[NSPIN - 1], Lm, U[2]); cfma_i(acc[NSPIN - 1], Lm, U[3]);
        }
      }
      // bonds, neighbours innermost as in k_spmv_async: the lane's element
      // (o, k) is row o of a cation's own block or column o of the block an
      // anion reads from its cation neighbour
      const int bstride = cat ? 1 : kNorbT;
      const double *Mb[4];
      const double2 *xn[4];
      bool has[4];
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const int xoff = dsm[kOffX + i * 4 + n], boff = dsm[kOffB + i * 4 + n];
        has[n] = xoff >= 0;
        xn[n] = reinterpret_cast<const double2 *>(st + (has[n] ? xoff : 0));
        Mb[n] = reinterpret_cast<const double *>(st + (has[n] ? boff : 0)) +
                (cat ? o * kNorbT : o);
      }
      double2 part[4][NSPIN];
#pragma unroll
      for (int n = 0; n < 4; n++)
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) part[n][sp].x = part[n][sp].y = 0.0;
#pragma unroll
      for (int kk = 0; kk < kNorbT; kk++)
#pragma unroll
        for (int n = 0; n < 4; n++) {
          if (!has[n]) continue;
          const double r = Mb[n][kk * bstride];
#pragma unroll
          for (int sp = 0; sp < NSPIN; sp++) cfma_r(part[n][sp], r, xn[n][sp * kNorbT + kk]);
        }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        acc[sp].x += (part[0][sp].x + part[1][sp].x) + (part[2][sp].x + part[3][sp].x);
        acc[sp].y += (part[0][sp].y + part[1][sp].y) + (part[2][sp].y + part[3][sp].y);
      }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const double2 xv = X0[sp * kNorbT + o];
        double2 xs, out;
        xs.x = scale * xv.x;
        xs.y = scale * xv.y;
        out.x = scale * acc[sp].x - shift * xs.x;
        out.y = scale * acc[sp].y - shift * xs.y;
        y[a * NB + sp * kNorbT + o] = out;
        dot += xs.x * out.x + xs.y * out.y;
      }
    }
    __syncthreads();  // the stage is free before the next unit's copies
  }
  if (DOT) grid_reduce<kTileThreads>(dot, partial, counter, alpha_out, alpha_idx, false);
}

}  // namespace

// The unit table of a context (10-orbital models; built on first use).
// Units follow the pencil order of the group work order (pencils visited
// j-block by j-block, eight pencils wide), each pencil cut at even cells.
static int build_tile_units(Ctx &c) {
  if (c.d_units) return TBGPU_OK;
  const long na = c.natoms;
  std::vector<int> asite(na);
  std::vector<int4> nbr(na);
  TB_CUDA(cudaMemcpyAsync(asite.data(), c.d_atom_site, sizeof(int) * na, cudaMemcpyDeviceToHost,
                          c.stream));
  TB_CUDA(cudaMemcpyAsync(nbr.data(), c.d_nbr, sizeof(int4) * na, cudaMemcpyDeviceToHost,
                          c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  const int XS = kNorbT * c.nspin * 16;
  const int OS = onsite_len(kNorbT * c.nspin) * 8;
  const int L_xo = kUnitAtoms * OS, L_cb = L_xo + kUnitAtoms * XS, L_nb = L_cb + 2 * kCatRun;
  auto cell_k = [&](long q) { return int((asite[q] >> 3) % c.nz); };
  // first atom of every pencil (atoms are numbered in site order)
  const long npen = long(c.nx) * c.ny;
  std::vector<long> pstart(npen + 1, na);
  for (long q = na - 1; q >= 0; q--) pstart[asite[q] / (8L * c.nz)] = q;
  for (long p = npen - 1; p >= 0; p--) pstart[p] = std::min(pstart[p], pstart[p + 1]);
  // per unit: header, sites, offsets (out-of-unit items as -(index + 2)
  // until the capacities are known), items
  std::vector<int> head, ofs;
  std::vector<std::vector<int>> unit_nb, unit_nx;
  int cap_nb = 0, cap_nx = 0;
  constexpr int kPB = 8;
  for (int jb = 0; jb < c.ny; jb += kPB)
    for (int i = 0; i < c.nx; i++)
      for (int j = jb; j < jb + kPB && j < c.ny; j++) {
        const long p = long(i) * c.ny + j;
        const long pend = pstart[p + 1];
        for (long a = pstart[p]; a < pend;) {
          const int k0 = cell_k(a) / 2 * 2;
          long b = a;
          while (b < pend && cell_k(b) / 2 * 2 == k0) b++;
          if (b - a > kUnitAtoms) return set_error(TBGPU_E_STATE);
          int ca[2] = {0, 0}, nca[2] = {0, 0};
          for (long q = a; q < b; q++)
            if ((asite[q] & 7) < 4) {
              const int cc = cell_k(q) - k0;
              if (nca[cc]++ == 0) ca[cc] = int(q);
            }
          std::vector<int> nbl, nxl, m(kUnitAtoms, 0), xo(4 * kUnitAtoms, -1),
              bo(4 * kUnitAtoms, -1);
          for (long q = a; q < b; q++) {
            const int ii = int(q - a), sm = asite[q] & 7;
            m[ii] = sm;
            const int cq = cell_k(q) - k0;
            const int nb4[4] = {nbr[q].x, nbr[q].y, nbr[q].z, nbr[q].w};
            for (int n = 0; n < 4; n++) {
              const int bb = nb4[n];
              if (bb < 0) continue;
              const bool inside = bb >= a && bb < b;
              if (inside) {
                xo[ii * 4 + n] = L_xo + int(bb - a) * XS;
              } else {
                auto it = std::find(nxl.begin(), nxl.end(), bb);
                xo[ii * 4 + n] = -(int(it - nxl.begin()) + 2);
                if (it == nxl.end()) nxl.push_back(bb);
              }
              if (sm < 4) {  // the cation's own block, in its cell's run
                bo[ii * 4 + n] =
                    L_cb + cq * kCatRun + (int(q) - ca[cq]) * 4 * kBlkBytes + n * kBlkBytes;
              } else if (inside) {  // the neighbour cation's block, in the unit
                const int cb = cell_k(bb) - k0;
                bo[ii * 4 + n] = L_cb + cb * kCatRun + (bb - ca[cb]) * 4 * kBlkBytes +
                                 kRevSlot[sm][n] * kBlkBytes;
              } else {
                bo[ii * 4 + n] = -(int(nbl.size()) + 2);
                nbl.push_back(bb * 4 + kRevSlot[sm][n]);
              }
            }
          }
          cap_nb = std::max(cap_nb, int(nbl.size()));
          cap_nx = std::max(cap_nx, int(nxl.size()));
          head.insert(head.end(), {int(a), int(b - a), ca[0], nca[0], ca[1], nca[1],
                                   int(nbl.size()), int(nxl.size())});
          head.insert(head.end(), m.begin(), m.end());
          ofs.insert(ofs.end(), xo.begin(), xo.end());
          ofs.insert(ofs.end(), bo.begin(), bo.end());
          unit_nb.push_back(std::move(nbl));
          unit_nx.push_back(std::move(nxl));
          a = b;
        }
      }
  const long nunits = long(unit_nb.size());
  const int L_nx = L_nb + cap_nb * kBlkBytes;
  const int dstride = ((kOffItems + cap_nb + cap_nx + 3) / 4) * 4;
  std::vector<int> desc(size_t(nunits) * dstride, 0);
  for (long u = 0; u < nunits; u++) {
    int *d = desc.data() + u * dstride;
    std::copy_n(head.begin() + u * (kHdr + kUnitAtoms), kHdr + kUnitAtoms, d);
    const int *xo = ofs.data() + u * 8 * kUnitAtoms, *bo = xo + 4 * kUnitAtoms;
    for (int k = 0; k < 4 * kUnitAtoms; k++) {
      d[kOffX + k] = xo[k] < -1 ? L_nx + (-xo[k] - 2) * XS : xo[k];
      d[kOffB + k] = bo[k] < -1 ? L_nb + (-bo[k] - 2) * kBlkBytes : bo[k];
    }
    std::copy(unit_nb[u].begin(), unit_nb[u].end(), d + kOffItems);
    std::copy(unit_nx[u].begin(), unit_nx[u].end(), d + kOffItems + cap_nb);
  }
  TB_CUDA(cudaMalloc(&c.d_units, sizeof(int) * desc.size()));
  TB_CUDA(cudaMemcpyAsync(c.d_units, desc.data(), sizeof(int) * desc.size(),
                          cudaMemcpyHostToDevice, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  c.nunits = nunits;
  c.unit_stride = dstride;
  c.unit_cap_nb = cap_nb;
  c.unit_cap_nx = cap_nx;
  return TBGPU_OK;
}

template <int NSPIN, bool DOT>
static int launch_tile_t(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                         int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  using L = TileLayout<NSPIN>;
  const int smem = desc_bytes(c.unit_stride) + 128 + L::bytes(c.unit_cap_nb, c.unit_cap_nx);
  // the stage size depends on the context's unit table: set on every launch
  if (cudaFuncSetAttribute(k_spmv_tile<NSPIN, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem) != cudaSuccess)
    return set_error(TBGPU_E_UNSUPPORTED);
  const int sms = c.sms;
  int per_sm = 0;
  TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_tile<NSPIN, DOT>,
                                                        kTileThreads, smem));
  if (per_sm < 1) return set_error(TBGPU_E_UNSUPPORTED);
  const unsigned grid = unsigned(std::max<long>(1, std::min<long>(c.nunits, long(sms) * per_sm)));
  if (DOT) {
    const int rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
  k_spmv_tile<NSPIN, DOT><<<grid, kTileThreads, smem, s>>>(
      c.nunits, c.d_units, c.unit_stride, c.unit_cap_nb, c.d_onsite, c.d_blocks,
      reinterpret_cast<const double2 *>(x), reinterpret_cast<double2 *>(y), shift, xnorm, xidx,
      DOT ? c.d_partial : nullptr, DOT ? c.d_counter : nullptr, alpha_out, aidx, c.d_status);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// H*x variant 3: 10-orbital models, double store, Gamma point, no skip mask;
// any other case takes the warp-staged kernel.
int launch_spmv_tile(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                     int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (misaligned16(x) || misaligned16(y)) return set_error(TBGPU_E_ARG);
  if (c.norb != kNorbT || c.ham_fp32 || c.recompute || c.bloch || c.d_skip || !c.d_blocks)
    return launch_spmv_async(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  const int rc = build_tile_units(c);
  if (rc) return rc;
  if (c.nspin == 2)
    return alpha_out ? launch_tile_t<2, true>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
                     : launch_tile_t<2, false>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
  return alpha_out ? launch_tile_t<1, true>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
                   : launch_tile_t<1, false>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
}

}  // namespace tbgpu
