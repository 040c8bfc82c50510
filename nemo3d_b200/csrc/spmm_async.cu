// Y_v = (H - shift) X_v for a block of P vectors at once (the H*Q step of
// the block Lanczos driver, where the reference calls matmul once per block
// vector, NEMO_3D/eigen/src/lanczos_blk.c:443-451), 10-orbital models.
//
// Same staging and work order as k_spmv_async (spmv_async.cu): a warp
// stages, for three atoms, the four bond blocks and the on-site record once
// and the own and neighbour segments of every block vector; each lane holds
// its block row (40 doubles, the four bonds) in registers and applies it to
// all P vectors.  Per atom and vector the blocks then cost 1/P of their
// bytes: DRAM per H*x falls from 2504 to 1856/P + 640 bytes.
#include <cstdint>

#include "tbgpu_internal.cuh"
#include "stage.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

using namespace stage;
constexpr int kNorb = 10;
constexpr int kMaxSmem = 227 * 1024;

template <int NSPIN, int P>
struct MLayout {
  static constexpr int NB = kNorb * NSPIN;
  static constexpr int ONS = onsite_len(NB);
  static constexpr int BLK = kNorb * kNorb;
  static constexpr int BLK_CH = BLK * 8 / 16;
  static constexpr int X_CH = NB;                  // 16-byte chunks per segment
  static constexpr int ONS_CH = ONS * 8 / 16;
  static constexpr int XSEG = 5 * NB * 16;         // own + 4 neighbour segments
  static constexpr int ATOM = 4 * BLK * 8 + ONS * 8 + P * XSEG + 48;
  static constexpr int WARP = kAPW * ATOM;
  static constexpr int WARPS = (kMaxSmem / WARP) > 16 ? 16 : (kMaxSmem / WARP);
  static constexpr int SMEM = WARPS * WARP;
  static __device__ __forceinline__ int blk(int i) { return i * ATOM; }
  static __device__ __forceinline__ int ons(int i) { return i * ATOM + 4 * BLK * 8; }
  static __device__ __forceinline__ int xs(int i, int v) {
    return i * ATOM + 4 * BLK * 8 + ONS * 8 + v * XSEG;
  }
};

template <class L, int P>
__device__ __forceinline__ void issue_block(unsigned char *st, const Meta &M, int lane,
                                            const double *__restrict__ onsite,
                                            const double *__restrict__ blocks,
                                            const double2 *__restrict__ X, long xstride) {
  constexpr int NB = L::NB;
#pragma unroll
  for (int i = 0; i < kAPW; i++) {
    const int m = M.m[i];
    if (m < 0) continue;
    const long a = long(M.a0) + i;
    unsigned char *bk = st + L::blk(i);
    if (m < 4) {
      const unsigned char *src = reinterpret_cast<const unsigned char *>(blocks + a * 4 * L::BLK);
#pragma unroll
      for (int c = lane; c < 4 * L::BLK_CH; c += 32) cp16(bk + c * 16, src + c * 16);
    } else {
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const int b = M.nb[i][n];
        const unsigned char *src = reinterpret_cast<const unsigned char *>(
            blocks + (long(b >= 0 ? b : a) * 4 + c_rev_slot[m][n]) * L::BLK);
#pragma unroll
        for (int c = lane; c < L::BLK_CH; c += 32)
          cp16z(bk + n * L::BLK * 8 + c * 16, src + c * 16, b >= 0 ? 16 : 0);
      }
    }
    if (lane < L::ONS_CH)
      cp16(st + L::ons(i) + lane * 16,
           reinterpret_cast<const unsigned char *>(onsite + a * L::ONS) + lane * 16);
    if (lane < L::X_CH) {
#pragma unroll
      for (int v = 0; v < P; v++) {
        unsigned char *xs = st + L::xs(i, v);
        const double2 *Xv = X + v * xstride;
        cp16(xs + 4 * NB * 16 + lane * 16,
             reinterpret_cast<const unsigned char *>(Xv + a * NB) + lane * 16);
#pragma unroll
        for (int n = 0; n < 4; n++) {
          const int b = M.nb[i][n];
          cp16z(xs + n * NB * 16 + lane * 16,
                reinterpret_cast<const unsigned char *>(Xv + long(b >= 0 ? b : a) * NB) +
                    lane * 16,
                b >= 0 ? 16 : 0);
        }
      }
    }
  }
}

template <int NSPIN, int P>
__global__ void __launch_bounds__(MLayout<NSPIN, P>::WARPS * 32, 1)
    k_spmm_async(long ngroups, const int2 *__restrict__ groups, const int4 *__restrict__ nbr,
                 const unsigned char *__restrict__ site_m, const double *__restrict__ onsite,
                 const double *__restrict__ blocks, const double2 *__restrict__ X,
                 long xstride, double2 *__restrict__ Y, long ystride, double shift) {
  using L = MLayout<NSPIN, P>;
  constexpr int NB = L::NB;
  constexpr int WARPS = L::WARPS;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *st = smem + warp * L::WARP;
  const int ai = lane / kNorb, o = lane - ai * kNorb;
  const long nw = long(gridDim.x) * WARPS;
  long g = long(blockIdx.x) * WARPS + warp;
  Meta cur = load_meta(g, ngroups, groups, nbr, site_m);
  Meta nxt = load_meta(g + nw, ngroups, groups, nbr, site_m);
  for (; g < ngroups; g += nw) {
    issue_block<L, P>(st, cur, lane, onsite, blocks, X, xstride);
    cp_commit();
    const Meta nn = load_meta(g + 2 * nw, ngroups, groups, nbr, site_m);
    cp_wait<0>();
    __syncwarp();
    const int m = ai == 0 ? cur.m[0] : ai == 1 ? cur.m[1] : ai == 2 ? cur.m[2] : -1;
    if (ai < kAPW && m >= 0) {
      const bool cat = m < 4;
      const long a = long(cur.a0) + ai;
      const double *rec = reinterpret_cast<const double *>(st + L::ons(ai));
      const double *bk = reinterpret_cast<const double *>(st + L::blk(ai));
      // this lane's row of the four bond blocks, kept for all P vectors
      const double *Mb = bk + (cat ? o * kNorb : o);
      const int bstride = cat ? 1 : kNorb;
      double r[4][kNorb];
#pragma unroll
      for (int n = 0; n < 4; n++)
#pragma unroll
        for (int kk = 0; kk < kNorb; kk++) r[n][kk] = Mb[n * L::BLK + kk * bstride];
      double dg[NSPIN];
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) dg[sp] = rec[sp * kNorb + o];
      const bool dangling = rec[NB + 1] != 0.0;
      const double Lm = NSPIN == 2 ? rec[NB] : 0.0;
#pragma unroll 1
      for (int v = 0; v < P; v++) {
        const double2 *xs = reinterpret_cast<const double2 *>(st + L::xs(ai, v));
        const double2 *X0 = xs + 4 * NB;
        double2 acc[NSPIN];
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          const double2 xv = X0[sp * kNorb + o];
          acc[sp] = make_double2(dg[sp] * xv.x - shift * xv.x, dg[sp] * xv.y - shift * xv.y);
        }
        if (dangling && o >= 1 && o <= 4) {  // dangling-bond sp3 couplings
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
            const double2 x1 = X0[sp * kNorb + k1], x2 = X0[sp * kNorb + k2],
                          x3 = X0[sp * kNorb + k3];
            acc[sp].x += c1 * x1.x + c2 * x2.x + c3 * x3.x;
            acc[sp].y += c1 * x1.y + c2 * x2.y + c3 * x3.y;
          }
        }
        if (NSPIN == 2 && o >= 2 && o <= 4) {  // on-site spin-orbit (mb_ham_spds_so.h)
          const double2 *U = X0, *D = X0 + kNorb;
          double2 &a0 = acc[0], &a1 = acc[NSPIN - 1];
          if (o == 2) {
            a0.x += Lm * U[3].y; a0.y -= Lm * U[3].x;    // -i L U3
            a0.x += Lm * D[4].x; a0.y += Lm * D[4].y;    //  L D4
            a1.x -= Lm * D[3].y; a1.y += Lm * D[3].x;    //  i L D3
            a1.x -= Lm * U[4].x; a1.y -= Lm * U[4].y;    // -L U4
          } else if (o == 3) {
            a0.x -= Lm * U[2].y; a0.y += Lm * U[2].x;    //  i L U2
            a0.x += Lm * D[4].y; a0.y -= Lm * D[4].x;    // -i L D4
            a1.x += Lm * D[2].y; a1.y -= Lm * D[2].x;    // -i L D2
            a1.x += Lm * U[4].y; a1.y -= Lm * U[4].x;    // -i L U4
          } else {
            a0.x -= Lm * D[2].x; a0.y -= Lm * D[2].y;    // -L D2
            a0.x -= Lm * D[3].y; a0.y += Lm * D[3].x;    //  i L D3
            a1.x += Lm * U[2].x; a1.y += Lm * U[2].y;    //  L U2
            a1.x -= Lm * U[3].y; a1.y += Lm * U[3].x;    //  i L U3
          }
        }
        double2 part[4][NSPIN];
#pragma unroll
        for (int n = 0; n < 4; n++)
#pragma unroll
          for (int sp = 0; sp < NSPIN; sp++) part[n][sp] = make_double2(0.0, 0.0);
#pragma unroll
        for (int kk = 0; kk < kNorb; kk++)
#pragma unroll
          for (int n = 0; n < 4; n++)
#pragma unroll
            for (int sp = 0; sp < NSPIN; sp++) {
              const double2 xv = xs[n * NB + sp * kNorb + kk];
              part[n][sp].x = fma(r[n][kk], xv.x, part[n][sp].x);
              part[n][sp].y = fma(r[n][kk], xv.y, part[n][sp].y);
            }
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          const double2 out = make_double2(
              acc[sp].x + ((part[0][sp].x + part[1][sp].x) + (part[2][sp].x + part[3][sp].x)),
              acc[sp].y + ((part[0][sp].y + part[1][sp].y) + (part[2][sp].y + part[3][sp].y)));
          Y[v * ystride + a * NB + sp * kNorb + o] = out;
        }
      }
    }
    __syncwarp();
    cur = nxt;
    nxt = nn;
  }
  cp_wait<0>();
}

template <int NSPIN, int P>
int launch_mt(Ctx &c, const double *x, long xstride, double *y, long ystride, double shift,
              cudaStream_t s) {
  using L = MLayout<NSPIN, P>;
  static_assert(L::WARPS >= 1, "block too large for shared memory");
  static std::atomic<unsigned long long> attr_done{0};
  if (ensure_smem_attr(attr_done, c.device, k_spmm_async<NSPIN, P>, L::SMEM)) return TBGPU_E_CUDA;
  k_spmm_async<NSPIN, P><<<unsigned(c.sms), L::WARPS * 32, L::SMEM, s>>>(
      c.ngroups, c.d_groups, c.d_nbr, c.d_site_m, c.d_onsite, c.d_blocks,
      reinterpret_cast<const double2 *>(x), xstride / 2, reinterpret_cast<double2 *>(y),
      ystride / 2, shift);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

template <int NSPIN>
int launch_ns(Ctx &c, int p, const double *x, long xs, double *y, long ys, double shift,
              cudaStream_t s) {
  switch (p) {
    case 2: return launch_mt<NSPIN, 2>(c, x, xs, y, ys, shift, s);
    case 3: return launch_mt<NSPIN, 3>(c, x, xs, y, ys, shift, s);
    case 4: return launch_mt<NSPIN, 4>(c, x, xs, y, ys, shift, s);
    case 5: return launch_mt<NSPIN, 5>(c, x, xs, y, ys, shift, s);
    case 6: return launch_mt<NSPIN, 6>(c, x, xs, y, ys, shift, s);
    case 7: return launch_mt<NSPIN, 7>(c, x, xs, y, ys, shift, s);
    case 8: return launch_mt<NSPIN, 8>(c, x, xs, y, ys, shift, s);
  }
  return set_error(TBGPU_E_ARG);
}

}  // namespace

// y + v*ystride = (H - shift)(x + v*xstride), v < p (p <= 8; strides in
// doubles).  Takes the block kernel for the 10-orbital models with the
// double-precision store at the Gamma point and p >= 2, one H*x launch per
// vector otherwise.
int launch_spmm(Ctx &c, int p, const double *x, long xstride, double *y, long ystride,
                double shift, cudaStream_t s) {
  if (p < 1 || p > 8) return set_error(TBGPU_E_ARG);
  if (p >= 2 && c.norb == kNorb && !c.bloch && !c.ham_fp32 && !c.recompute &&
      c.spmv_variant != 1)
    return c.nspin == 2 ? launch_ns<2>(c, p, x, xstride, y, ystride, shift, s)
                        : launch_ns<1>(c, p, x, xstride, y, ystride, shift, s);
  for (int v = 0; v < p; v++) {
    int rc = launch_spmv(c, x + v * xstride, y + v * ystride, shift, nullptr, 0, nullptr, 0, s);
    if (rc) return rc;
  }
  return TBGPU_OK;
}

}  // namespace tbgpu

extern "C" int tbgpu_hx_block_dev(tbgpu_ctx *ctx, int p, double shift, const double *x_dev,
                                  double *y_dev) {
  using namespace tbgpu;
  if (!ctx || !x_dev || !y_dev || p < 1 || p > 8 || misaligned16(x_dev) || misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  set_error(TBGPU_OK);
  const long n = 2 * c.natoms * c.nb;  // doubles per vector
  return launch_spmm(c, p, x_dev, n, y_dev, n, shift, c.stream);
}
