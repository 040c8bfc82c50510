// H*x for the 10-orbital (sp3d5s*) models with asynchronous 16-byte gathers.
//
// Same product as k_spmv (spmv.cu; restates Hv_stored_20_Hzb,
// nemo3d/src/base/Hmult_stored.c:176-607, with the Lanczos alpha dot of
// eigen/src/lanczos.c:679-707 fused).  Each warp owns a private
// shared-memory stage (one or two) holding, for three atoms, the four bond
// blocks (a cation's own 3200-byte run, or the four 800-byte blocks stored
// by an anion's cation neighbours), the own and four neighbour vector
// segments and the on-site record (5056 bytes per atom).  The warp fills a
// stage with coalesced 16-byte cp.async copies (one instruction moves 512
// bytes, nothing is held in registers) and computes it, one lane per orbital
// row, from shared memory; with one stage per warp, the other warps of the
// SM cover its wait, with two it also overlaps its own next copies.  Groups
// (up to three consecutive atoms of one k-pencil of cells) are dealt to
// warps in the work order of the context (pencils visited j-block by
// j-block, see build_work_order), so all SMs sweep the structure together and
// a neighbour's x segment, or a block an anion reads transposed (stored once,
// by the cation), is still in L2 when it is needed the second time.
//
// (A variant that gathered the same bytes with one 1-D TMA bulk copy per
// 300-800-byte segment took 2.4 ms per launch on the 1.02M-atom dot: that
// many small requests are limited by the TMA request rate, not by HBM.)
//
// BULK (the default; variant 4 turns it off): a cation's four blocks, one
// contiguous 3200-byte run, arrive by one 1-D bulk copy (cp.async.bulk, no
// multicast) issued by lane 0 on an mbarrier of the warp's stage instead of
// 200 16-byte cp.async copies, which takes about a third of the staging
// copies off the load/store unit (the bytes written to shared memory stay
// // the same, and so does most of the time: 0.668 against 0.674 ms).  The
// wait on the mbarrier is bounded: a warp whose copy does not arrive reports
// TBGPU_E_TIMEOUT in the status word, waits once more (bounded) for its
// copies in flight and leaves its loop; if that second wait also runs out,
// every warp of the CTA stops issuing copies, and the CTA may end with that
// one copy outstanding.
#include <cstdint>

#include "tbgpu_internal.cuh"
#include "reduce.cuh"
#include "stage.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

using namespace stage;
constexpr int kNorb = 10;
constexpr int kWarpsF32 = 16;  // warps per SM of the float-vector kernel

template <typename T, typename V>
__device__ __forceinline__ void cfma_r(V &acc, T v, V a) {
  acc.x = fma(v, a.x, acc.x);
  acc.y = fma(v, a.y, acc.y);
}
template <typename T, typename V>
__device__ __forceinline__ void cfma_i(V &acc, T lam, V a) {
  acc.x -= lam * a.y;
  acc.y += lam * a.x;
}
template <typename V> struct Scalar;
template <> struct Scalar<double2> { using T = double; };
template <> struct Scalar<float2> { using T = float; };

// HT: element type of the stored Hamiltonian (double, or float for the
// single-precision store); VT: vector element (double2, or float2 for the
// mixed-precision Lanczos, whose products accumulate in float)
template <int NSPIN, int WARPS, int STAGES, typename HT_ = double, typename VT_ = double2>
struct Layout {
  using HT = HT_;
  using VT = VT_;
  using RT = typename Scalar<VT>::T;
  static constexpr int HS = int(sizeof(HT));
  static constexpr int VS = int(sizeof(VT));
  static constexpr int NB = kNorb * NSPIN;
  static constexpr int ONS = onsite_len(NB);
  static constexpr int BLK = kNorb * kNorb;      // elements per bond block
  static constexpr int BLK_CH = BLK * HS / 16;   // 16-byte chunks per block (50 or 25)
  static constexpr int X_CH = NB * VS / 16;      // chunks per vector segment
  static constexpr int ONS_CH = ONS * HS / 16;   // chunks per on-site record
  // per-atom stride, padded by 48 bytes so the three atoms of a warp start
  // on different shared-memory banks
  static constexpr int ATOM = 4 * BLK * HS + 5 * NB * VS + ONS * HS + 48;
  static constexpr int STAGE = kAPW * ATOM;
  static constexpr int WARP = STAGES * STAGE;
  static constexpr int SMEM = WARPS * WARP;
  static __device__ __forceinline__ int blk(int i) { return i * ATOM; }
  static __device__ __forceinline__ int xs(int i) { return i * ATOM + 4 * BLK * HS; }
  static __device__ __forceinline__ int ons(int i) { return i * ATOM + 4 * BLK * HS + 5 * NB * VS; }
};

// Issue the copies of group g into one stage (all lanes; no wait).  BULK:
// the cations' block runs as bulk copies on the stage's mbarrier mb (lane 0
// always arrives once, with the byte count, even for a group without
// cations).
template <class L, bool BULK = false>
__device__ __forceinline__ void issue(unsigned char *st, long g, const Meta &M, int lane,
                                      const typename L::HT *__restrict__ onsite,
                                      const typename L::HT *__restrict__ blocks,
                                      const typename L::VT *__restrict__ x, uint32_t mb = 0) {
  constexpr int NB = L::NB;
  if (BULK && lane == 0) {
    uint32_t ncat = 0;
#pragma unroll
    for (int i = 0; i < kAPW; i++) ncat += M.m[i] >= 0 && M.m[i] < 4;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(mb, ncat * uint32_t(4 * L::BLK * L::HS));
#pragma unroll
    for (int i = 0; i < kAPW; i++)
      if (M.m[i] >= 0 && M.m[i] < 4)
        bulk_g2s(smem_addr(st + L::blk(i)), blocks + (long(M.a0) + i) * 4 * L::BLK,
                 uint32_t(4 * L::BLK * L::HS), mb);
  }
#pragma unroll
  for (int i = 0; i < kAPW; i++) {
    const int m = M.m[i];
    if (m < 0) continue;
    const long a = long(M.a0) + i;
    const bool cat = m < 4;
    unsigned char *bk = st + L::blk(i);
    if (cat) {  // the cation's four blocks are one contiguous run
      if (!BULK) {
        const unsigned char *src =
            reinterpret_cast<const unsigned char *>(blocks + a * 4 * L::BLK);
#pragma unroll
        for (int c = lane; c < 4 * L::BLK_CH; c += 32) cp16(bk + c * 16, src + c * 16);
      }
    } else {
      // a missing neighbour (surface) is zero-filled, not skipped
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const int b = M.nb[i][n];
        const int bytes = b >= 0 ? 16 : 0;
        const unsigned char *src = reinterpret_cast<const unsigned char *>(
            blocks + (long(b >= 0 ? b : a) * 4 + c_rev_slot[m][n]) * L::BLK);
#pragma unroll
        for (int c = lane; c < L::BLK_CH; c += 32)
          cp16z(bk + n * L::BLK * L::HS + c * 16, src + c * 16, bytes);
      }
    }
    unsigned char *xs = st + L::xs(i);
    // own segment in slot 4, neighbours in slots 0..3; one lane per chunk
    if (lane < L::X_CH) {
      cp16(xs + 4 * NB * L::VS + lane * 16, reinterpret_cast<const unsigned char *>(x + a * NB) + lane * 16);
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const int b = M.nb[i][n];
        cp16z(xs + n * NB * L::VS + lane * 16,
              reinterpret_cast<const unsigned char *>(x + long(b >= 0 ? b : a) * NB) + lane * 16,
              b >= 0 ? 16 : 0);
      }
    }
    if (lane < L::ONS_CH)
      cp16(st + L::ons(i) + lane * 16,
           reinterpret_cast<const unsigned char *>(onsite + a * L::ONS) + lane * 16);
  }
}

template <int NSPIN, bool DOT, int WARPS, int STAGES, typename HT = double,
          typename VT = double2, bool BULK = false>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_spmv_async(long ngroups, const int2 *__restrict__ groups, const int4 *__restrict__ nbr,
                 const unsigned char *__restrict__ site_m, const HT *__restrict__ onsite,
                 const HT *__restrict__ blocks, const VT *__restrict__ x,
                 VT *__restrict__ y, double shift_d, const double *__restrict__ xnorm,
                 int xnorm_idx, double *partial, unsigned int *counter, double *alpha_out,
                 int alpha_idx, const unsigned char *__restrict__ skip, int *status = nullptr) {
  using L = Layout<NSPIN, WARPS, STAGES, HT, VT>;
  using RT = typename L::RT;
  constexpr int NB = L::NB;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wbase = smem + warp * L::WARP;
  // BULK: one mbarrier per stage of this warp, after the stages
  const uint32_t mb0 = smem_addr(smem + L::SMEM) + uint32_t(warp * STAGES * 8);
  uint32_t phase = 0;  // bit s: parity of stage s's next completion
  // set when a warp's copies did not land within two bounded waits: every
  // warp of the CTA then stops issuing copies (BULK only)
  __shared__ int s_stop;
  if (BULK) {
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < STAGES; s++) mbar_init(mb0 + 8 * s, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x == 0) s_stop = 0;
    __syncthreads();
  }
  const int ai = lane / kNorb, o = lane - ai * kNorb;
  const RT scale = RT(xnorm ? 1.0 / xnorm[xnorm_idx] : 1.0);
  const RT shift = RT(shift_d);
  double dot = 0.0;
  const long nw = long(gridDim.x) * WARPS;
  long g = long(blockIdx.x) * WARPS + warp;
  // prologue: copies of the first group in flight, metadata of the next
  Meta cur = load_meta(g, ngroups, groups, nbr, site_m, skip);
  if (STAGES > 1 && g < ngroups) issue<L, BULK>(wbase, g, cur, lane, onsite, blocks, x, mb0);
  cp_commit();
  Meta nxt = load_meta(g + nw, ngroups, groups, nbr, site_m, skip);
  int k = 0;
  for (; g < ngroups; g += nw, ++k) {
    if (BULK && __any_sync(0xffffffffu, *reinterpret_cast<volatile int *>(&s_stop) != 0))
      break;  // another warp's copies never landed: issue nothing more
    const long gn = g + nw;
    unsigned char *st = wbase + (k % STAGES) * L::STAGE;
    if (STAGES > 1) {  // next group's copies overlap this group's compute
      if (gn < ngroups)
        issue<L, BULK>(wbase + ((k + 1) % STAGES) * L::STAGE, gn, nxt, lane, onsite, blocks, x,
                       mb0 + 8 * ((k + 1) % STAGES));
      cp_commit();
    } else {           // single stage: other warps overlap this one's wait
      issue<L, BULK>(st, g, cur, lane, onsite, blocks, x, mb0);
      cp_commit();
    }
    const Meta nn = load_meta(gn + nw, ngroups, groups, nbr, site_m, skip);  // two groups ahead
    if (STAGES > 1) cp_wait<1>(); else cp_wait<0>();  // this lane's copies of g landed
    if (BULK) {  // and the stage's bulk copies (warp-uniform decision)
      const int s = k % STAGES;
      const uint32_t par = (phase >> s) & 1u;
      const bool late = !mbar_wait(mb0 + 8 * s, par);
      if (__any_sync(0xffffffffu, late)) {
        if (lane == 0 && status) atomicExch(status, TBGPU_E_TIMEOUT);
        // one more bounded wait for the copies in flight; if they still did
        // not land, the CTA stops issuing copies and may exit with that copy
        // outstanding (the one exit whose shared-memory state is not
        // guaranteed; the status word reports it)
        const bool drained = mbar_wait(mb0 + 8 * s, par);
        if (!drained && lane == 0) *reinterpret_cast<volatile int *>(&s_stop) = 1;
        break;
      }
      phase ^= 1u << s;
    }
    __syncwarp();   // ... and every lane's
    // this lane's atom, selected without indexing the metadata at run time
    const int m = ai == 0 ? cur.m[0] : ai == 1 ? cur.m[1] : ai == 2 ? cur.m[2] : -1;
    int nbv[4];
#pragma unroll
    for (int n = 0; n < 4; n++)
      nbv[n] = ai == 0 ? cur.nb[0][n] : ai == 1 ? cur.nb[1][n] : cur.nb[2][n];
    if (ai < kAPW && m >= 0) {
      const bool cat = m < 4;
      const long a = long(cur.a0) + ai;
      const VT *xs = reinterpret_cast<const VT *>(st + L::xs(ai));
      const VT *X0 = xs + 4 * NB;
      const HT *rec = reinterpret_cast<const HT *>(st + L::ons(ai));
      const HT *bk = reinterpret_cast<const HT *>(st + L::blk(ai));
      VT acc[NSPIN];
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const VT v = X0[sp * kNorb + o];
        const RT dg = rec[sp * kNorb + o];
        acc[sp].x = dg * v.x;
        acc[sp].y = dg * v.y;
      }
      if (o >= 1 && o <= 4 && rec[NB + 1] != HT(0)) {  // dangling-bond sp3 couplings
        const RT sx = rec[NB + 2], sy = rec[NB + 3], sz = rec[NB + 4];
        const RT cxy = rec[NB + 5], cxz = rec[NB + 6], cyz = rec[NB + 7];
        RT c1, c2, c3;
        int k1, k2, k3;
        if (o == 1) { c1 = sx; k1 = 2; c2 = sy; k2 = 3; c3 = sz; k3 = 4; }
        else if (o == 2) { c1 = sx; k1 = 1; c2 = cxy; k2 = 3; c3 = cxz; k3 = 4; }
        else if (o == 3) { c1 = sy; k1 = 1; c2 = cxy; k2 = 2; c3 = cyz; k3 = 4; }
        else { c1 = sz; k1 = 1; c2 = cxz; k2 = 2; c3 = cyz; k3 = 3; }
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) {
          cfma_r(acc[sp], c1, X0[sp * kNorb + k1]);
          cfma_r(acc[sp], c2, X0[sp * kNorb + k2]);
          cfma_r(acc[sp], c3, X0[sp * kNorb + k3]);
        }
      }
      if (NSPIN == 2 && o >= 2 && o <= 4) {  // on-site spin-orbit (mb_ham_spds_so.h)
        const RT Lm = rec[NB];
        const VT *U = X0, *D = X0 + kNorb;
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
      // bonds: one accumulator per neighbour, neighbours innermost so that
      // consecutive FMAs feed independent chains; the lane's block element
      // (o, k) is row o of a cation's own block or column o of the block an
      // anion reads from its cation neighbour
      VT part[4][NSPIN];
#pragma unroll
      for (int n = 0; n < 4; n++)
#pragma unroll
        for (int sp = 0; sp < NSPIN; sp++) part[n][sp].x = part[n][sp].y = RT(0);
      const HT *Mb = bk + (cat ? o * kNorb : o);
      const int bstride = cat ? 1 : kNorb;
#pragma unroll
      for (int kk = 0; kk < kNorb; kk++)
#pragma unroll
        for (int n = 0; n < 4; n++) {
          if (nbv[n] < 0) continue;
          const RT r = Mb[n * L::BLK + kk * bstride];
#pragma unroll
          for (int sp = 0; sp < NSPIN; sp++) cfma_r(part[n][sp], r, xs[n * NB + sp * kNorb + kk]);
        }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        acc[sp].x += (part[0][sp].x + part[1][sp].x) + (part[2][sp].x + part[3][sp].x);
        acc[sp].y += (part[0][sp].y + part[1][sp].y) + (part[2][sp].y + part[3][sp].y);
      }
#pragma unroll
      for (int sp = 0; sp < NSPIN; sp++) {
        const VT xv = X0[sp * kNorb + o];
        VT xo, out;
        xo.x = scale * xv.x;
        xo.y = scale * xv.y;
        out.x = scale * acc[sp].x - shift * xo.x;
        out.y = scale * acc[sp].y - shift * xo.y;
        y[a * NB + sp * kNorb + o] = out;
        dot += double(xo.x) * double(out.x) + double(xo.y) * double(out.y);
      }
    }
    __syncwarp();  // stage k is free before the next iteration overwrites it
    cur = nxt;
    nxt = nn;
  }
  cp_wait<0>();
  if (DOT) grid_reduce<WARPS * 32>(dot, partial, counter, alpha_out, alpha_idx, false);
}

template <int NSPIN, bool DOT, int WARPS, int STAGES, typename HT, typename VT = double2,
          bool BULK = false>
int launch_async_t(Ctx &c, const void *x, void *y, double shift, const double *xnorm,
                   int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  using L = Layout<NSPIN, WARPS, STAGES, HT, VT>;
  constexpr int smem = L::SMEM + (BULK ? WARPS * STAGES * 8 : 0);
  static std::atomic<unsigned long long> attr_done{0};
  if (ensure_smem_attr(attr_done, c.device, k_spmv_async<NSPIN, DOT, WARPS, STAGES, HT, VT, BULK>,
                       smem))
    return TBGPU_E_CUDA;
  const unsigned grid = unsigned(c.sms);
  if (DOT) {
    int rc = ensure_partials(c, int(grid));
    if (rc) return rc;
  }
  k_spmv_async<NSPIN, DOT, WARPS, STAGES, HT, VT, BULK><<<grid, WARPS * 32, smem, s>>>(
      c.ngroups, c.d_groups, c.d_nbr, c.d_site_m, ham_onsite<HT>(c), ham_blocks<HT>(c),
      reinterpret_cast<const VT *>(x), reinterpret_cast<VT *>(y), shift, xnorm, xidx,
      DOT ? c.d_partial : nullptr, DOT ? c.d_counter : nullptr, alpha_out, aidx, c.d_skip,
      c.d_status);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

}  // namespace

template <int WARPS, int STAGES, typename HT, bool BULK = false>
int launch_cfg(Ctx &c, const double *x, double *y, double shift, const double *xnorm, int xidx,
               double *alpha_out, int aidx, cudaStream_t s) {
  using V = double2;
  if (c.nspin == 2)
    return alpha_out
               ? launch_async_t<2, true, WARPS, STAGES, HT, V, BULK>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
               : launch_async_t<2, false, WARPS, STAGES, HT, V, BULK>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
  return alpha_out
             ? launch_async_t<1, true, WARPS, STAGES, HT, V, BULK>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
             : launch_async_t<1, false, WARPS, STAGES, HT, V, BULK>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
}

// complex-float vectors over the single-precision store, float accumulation
// (the mixed-precision Lanczos); alpha is still reduced in double
int launch_spmv_async_f32(Ctx &c, const float *x, float *y, double shift, const double *xnorm,
                          int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (c.norb != kNorb || !c.ham_fp32) return set_error(TBGPU_E_UNSUPPORTED);
  constexpr int W = kWarpsF32;
  if (c.nspin == 2)
    return alpha_out
               ? launch_async_t<2, true, W, 1, float, float2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
               : launch_async_t<2, false, W, 1, float, float2>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
  return alpha_out
             ? launch_async_t<1, true, W, 1, float, float2>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s)
             : launch_async_t<1, false, W, 1, float, float2>(c, x, y, shift, xnorm, xidx, nullptr, 0, s);
}

int launch_spmv_async(Ctx &c, const double *x, double *y, double shift, const double *xnorm,
                      int xidx, double *alpha_out, int aidx, cudaStream_t s) {
  if (c.norb != kNorb) return set_error(TBGPU_E_UNSUPPORTED);
  // variant 0: 14 warps x 1 stage per SM (other warps cover a warp's wait),
  // cation block runs by bulk copy (0.668 ms per launch on the 1.02M-atom
  // dot); variant 4: the same with every piece by cp.async (0.674 ms);
  // variant 2: 7 warps x 2 stages (each warp overlaps its own next copies;
  // 0.91 ms).  Single-precision store: half the block bytes, 16 warps fit.
  if (c.ham_fp32)
    return launch_cfg<16, 1, float>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.spmv_variant == 2)
    return launch_cfg<7, 2, double>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  if (c.spmv_variant == 4)
    return launch_cfg<14, 1, double>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
  return launch_cfg<14, 1, double, true>(c, x, y, shift, xnorm, xidx, alpha_out, aidx, s);
}

template <int NSPIN, int WARPS, typename HT>
static int launch_scratch_async_t(Ctx &c, int sms, const double2 *X, double2 *Y, double shift,
                                  double *partial, unsigned int *counter, double *dot_out,
                                  cudaStream_t s) {
  using L = Layout<NSPIN, WARPS, 1, HT>;
  TB_CUDA(cudaFuncSetAttribute(k_spmv_async<NSPIN, true, WARPS, 1, HT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM));
  k_spmv_async<NSPIN, true, WARPS, 1, HT><<<sms, WARPS * 32, L::SMEM, s>>>(
      c.ngroups, c.d_groups, c.d_nbr, c.d_site_m, ham_onsite<HT>(c), ham_blocks<HT>(c), X, Y,
      shift, nullptr, 0, partial, counter, dot_out, 0, nullptr);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// Launch of the default 10-orbital configuration (one CTA per SM) with the
// alpha dot reduced through caller-provided scratch: partial[cap] doubles
// and a zeroed counter.  Allocates nothing.
int launch_spmv_async_scratch(Ctx &c, const double *x, double *y, double shift,
                              double *partial, unsigned int *counter, int cap, double *dot_out,
                              cudaStream_t s) {
  if (c.norb != kNorb) return set_error(TBGPU_E_UNSUPPORTED);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  if (sms > cap) return set_error(TBGPU_E_ARG);
  const double2 *X = reinterpret_cast<const double2 *>(x);
  double2 *Y = reinterpret_cast<double2 *>(y);
  if (c.ham_fp32)
    return c.nspin == 2
               ? launch_scratch_async_t<2, 16, float>(c, sms, X, Y, shift, partial, counter, dot_out, s)
               : launch_scratch_async_t<1, 16, float>(c, sms, X, Y, shift, partial, counter, dot_out, s);
  return c.nspin == 2
             ? launch_scratch_async_t<2, 14, double>(c, sms, X, Y, shift, partial, counter, dot_out, s)
             : launch_scratch_async_t<1, 14, double>(c, sms, X, Y, shift, partial, counter, dot_out, s);
}

}  // namespace tbgpu
