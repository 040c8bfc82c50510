// Batched Lanczos: many independent dots solved together on one GPU.
//
// The dots are packed into one cell grid, side by side along x and separated
// by empty cells, so the context's Hamiltonian is block diagonal (no bond
// crosses a gap) and every product kernel serves all dots in one launch.
// Each dot keeps its own recurrence, exactly the reference's
// single_lanczos_iteration (NEMO_3D/eigen/src/lanczos.c:421-757) on its
// segment of the vectors: per dot alpha and beta are reduced over the dot's
// segment only, and the convergence test (find_converged_eigval,
// lanczos.c:764-996) runs on each dot's own tridiagonal matrix, with its own
// windows, on the host threads.  Dots iterate in lockstep until the last one
// has converged; each dot's iteration count and eigenvalues are those of the
// check that declared it converged.
//
// Device iteration: w = H r (the unnormalised r of the previous step, one
// launch for all dots), alpha_d = <r, w>_d / beta_d^2 (segmented reduction),
// r' = w/beta_d - alpha_d r/beta_d - beta_d r_prev/beta_prev_d with
// beta'_d = ||r'||_d (segmented reduction), then the device iteration counter
// advances.  The kernels read the iteration from device memory, so one check
// interval (ConvCheckSkipRate iterations) is captured once as a CUDA graph
// and replayed; the ring of r vectors has a size that divides the interval,
// so every replay starts on the same ring slot.  Segmented reductions are
// deterministic: a block covers part of one dot, writes its partial, and the
// last block of that dot sums the dot's partials in block order.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <vector>

#include "host_par.h"
#include "tbgpu_internal.cuh"

namespace tbgpu {

namespace {

constexpr int kBT = 256;             // threads per block of the segmented kernels
constexpr long kChunk = kBT * 8L;    // vector entries per block
constexpr int kMaxK = 32;            // iterations per eigenvector accumulation chunk
constexpr int kMaxVec = 16;          // eigenvectors per dot

struct Seg {
  const int *blk_dot;     // [nblk] dot of the block
  const long *blk_lo;     // [nblk] first entry
  const long *blk_hi;     // [nblk] end entry
  const int *dot_blk0;    // [ndots + 1] first block of each dot
};

__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }
template <typename VT> __device__ __forceinline__ VT narrow(double x, double y);
template <> __device__ __forceinline__ double2 narrow<double2>(double x, double y) {
  return make_double2(x, y);
}
template <> __device__ __forceinline__ float2 narrow<float2>(double x, double y) {
  return make_float2(float(x), float(y));
}

// block sum, then the last block of dot d sums the dot's partials in order;
// returns true in thread 0 of that block with the total in *tot
__device__ __forceinline__ bool seg_reduce(double v, const Seg &S, int d, double *partial,
                                           unsigned *counters, double *tot) {
  __shared__ double red[kBT / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  const int b0 = S.dot_blk0[d], b1 = S.dot_blk0[d + 1];
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBT / 32; i++) t += red[i];
    partial[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(counters + d, 1u) == unsigned(b1 - b0 - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
  double t = 0.0;
  for (int b = b0; b < b1; b++) t += __ldcg(partial + b);
  counters[d] = 0u;
  *tot = t;
  return true;
}

// out[d * stride + idx] = sqrt(sum |x|^2) over dot d
template <typename VT>
__global__ void __launch_bounds__(kBT)
    k_bnorm(Seg S, const VT *__restrict__ x, double *partial, unsigned *counters, double *out,
            long stride, int idx) {
  const int d = S.blk_dot[blockIdx.x];
  double s = 0.0;
  for (long j = S.blk_lo[blockIdx.x] + threadIdx.x; j < S.blk_hi[blockIdx.x]; j += kBT) {
    const double2 v = widen(x[j]);
    s += v.x * v.x + v.y * v.y;
  }
  double t;
  if (seg_reduce(s, S, d, partial, counters, &t)) out[d * stride + idx] = sqrt(t);
}

// y = x / den[d] (each dot's start vector normalised, lanczos_initialize)
template <typename VT>
__global__ void __launch_bounds__(kBT)
    k_bdivide(Seg S, const double2 *__restrict__ x, const double *__restrict__ den,
              VT *__restrict__ y) {
  const double dv = den[S.blk_dot[blockIdx.x]];
  for (long j = S.blk_lo[blockIdx.x] + threadIdx.x; j < S.blk_hi[blockIdx.x]; j += kBT) {
    const double2 v = x[j];
    y[j] = narrow<VT>(v.x / dv, v.y / dv);
  }
}

// alpha[d][it] = Re<r, w>_d / bet[d][it]^2  (w = H r, r unnormalised)
template <typename VT>
__global__ void __launch_bounds__(kBT)
    k_balpha(Seg S, const VT *__restrict__ r, const VT *__restrict__ w, const double *bet,
             double *alpha, long sa, long sb, const int *itp, double *partial,
             unsigned *counters, const unsigned char *__restrict__ done) {
  const int d = S.blk_dot[blockIdx.x];
  if (done[d]) return;  // a converged dot: every block of it leaves
  const int it = *itp;
  double s = 0.0;
  for (long j = S.blk_lo[blockIdx.x] + threadIdx.x; j < S.blk_hi[blockIdx.x]; j += kBT) {
    const double2 a = widen(r[j]), b = widen(w[j]);
    s += a.x * b.x + a.y * b.y;
  }
  double t;
  if (seg_reduce(s, S, d, partial, counters, &t)) {
    const double b = bet[d * sb + it];
    alpha[d * sa + it] = t / (b * b);
  }
}

// r_out = w/bet - (alpha r_c/bet + bet r_p/bet_prev) per dot;
// bet[d][it+1] = ||r_out||_d
template <typename VT>
__global__ void __launch_bounds__(kBT)
    k_bupdate(Seg S, const VT *__restrict__ w, const VT *__restrict__ rc,
              const VT *__restrict__ rp, VT *__restrict__ rout, const double *alpha, double *bet,
              long sa, long sb, const int *itp, double *partial, unsigned *counters,
              const unsigned char *__restrict__ done) {
  const int d = S.blk_dot[blockIdx.x];
  if (done[d]) return;
  const int it = *itp;
  const double al = alpha[d * sa + it], bprev = bet[d * sb + it];
  const double iq = 1.0 / bprev;
  const double ip = it > 0 ? 1.0 / bet[d * sb + it - 1] : 0.0;
  double s = 0.0;
  for (long j = S.blk_lo[blockIdx.x] + threadIdx.x; j < S.blk_hi[blockIdx.x]; j += kBT) {
    const double2 wv = widen(w[j]), cv = widen(rc[j]);
    const double2 q = make_double2(cv.x * iq, cv.y * iq);
    double2 p = make_double2(0.0, 0.0);
    if (it > 0) {
      const double2 pv = widen(rp[j]);
      p = make_double2(pv.x * ip, pv.y * ip);
    }
    const VT r = narrow<VT>(wv.x * iq - (al * q.x + bprev * p.x),
                            wv.y * iq - (al * q.y + bprev * p.y));
    rout[j] = r;
    const double2 rw = widen(r);
    s += rw.x * rw.x + rw.y * rw.y;
  }
  double t;
  if (seg_reduce(s, S, d, partial, counters, &t)) bet[d * sb + it + 1] = sqrt(t);
}

__global__ void k_badvance(int *itp) { *itp += 1; }

// leave dot d out of the products and updates from here on
__global__ void k_bmark(long lo, long hi, int d, unsigned char *skip, unsigned char *done) {
  for (long a = lo + blockIdx.x * (long)blockDim.x + threadIdx.x; a < hi;
       a += (long)gridDim.x * blockDim.x)
    skip[a] = 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) done[d] = 1;
}

template <typename VT>
struct RingPtrs {
  const VT *r[kMaxK];
};

// V[e][j] += sum_k coef[d][k][e] R_k[j] for the nv eigenvectors of this
// chunk (coefficients of dot d for the chunk's nk iterations)
template <typename VT>
__global__ void __launch_bounds__(kBT)
    k_baccum(Seg S, int nk, int nv, RingPtrs<VT> R, const double *__restrict__ coef,
             double2 *__restrict__ V, long dim) {
  __shared__ double cs[kMaxK * kMaxVec];
  const int d = S.blk_dot[blockIdx.x];
  for (int i = threadIdx.x; i < nk * nv; i += kBT) cs[i] = coef[size_t(d) * kMaxK * kMaxVec + i];
  __syncthreads();
  for (long j = S.blk_lo[blockIdx.x] + threadIdx.x; j < S.blk_hi[blockIdx.x]; j += kBT) {
    double2 acc[kMaxVec];
#pragma unroll
    for (int e = 0; e < kMaxVec; e++)
      if (e < nv) acc[e] = V[e * dim + j];
    for (int k = 0; k < nk; k++) {
      const double2 r = widen(__ldg(R.r[k] + j));
#pragma unroll
      for (int e = 0; e < kMaxVec; e++)
        if (e < nv) {
          acc[e].x = fma(cs[k * nv + e], r.x, acc[e].x);
          acc[e].y = fma(cs[k * nv + e], r.y, acc[e].y);
        }
    }
#pragma unroll
    for (int e = 0; e < kMaxVec; e++)
      if (e < nv) V[e * dim + j] = acc[e];
  }
}

int hx_plain(Ctx &c, const double2 *x, double2 *y, cudaStream_t s) {
  return launch_spmv(c, reinterpret_cast<const double *>(x), reinterpret_cast<double *>(y), 0.0,
                     nullptr, 0, nullptr, 0, s);
}
int hx_plain(Ctx &c, const float2 *x, float2 *y, cudaStream_t s) {
  return launch_spmv_f32(c, reinterpret_cast<const float *>(x), reinterpret_cast<float *>(y),
                         0.0, nullptr, 0, nullptr, 0, s);
}

// check points exactly as lanczos_tridiagonal's skip counter places them
std::vector<int> check_points(int start, int skip, int imax) {
  std::vector<int> out;
  int at = 0;
  for (;;) {
    int cnt = 0, nxt = imax;
    for (int it = at + 1; it < imax; it++) {
      cnt++;
      if (start < it && skip <= cnt) {
        nxt = it;
        break;
      }
    }
    if (nxt >= imax) break;
    out.push_back(nxt);
    at = nxt;
  }
  return out;
}

struct DotState {
  std::vector<double> c1, c2;
  std::vector<int> i1, i2;
  bool done = false;
  int final_it = -1;
  std::vector<double> Ta, Tb;  // tridiagonal of the deciding check
};

}  // namespace

struct BatchArgs {
  int conv_start, conv_skip, imax, req1, req2;
  double tol;
  const double *emin1, *emax1, *emin2, *emax2;
};

template <typename VT>
static int solve_batch_t(Ctx &c, int ndots, const int *dot_cells, const BatchArgs &A,
                         const double *r0_dev, double *values, int vstride, int *found,
                         int *iterations, double *V_dev, int maxvec) {
  constexpr bool kMixed = sizeof(VT) == sizeof(float2);
  cudaStream_t s = c.stream;
  const long dim = c.natoms * c.nb;
  // ---- dots: atom ranges from the cell boundaries along x --------------------
  std::vector<int> asite(c.natoms);
  std::vector<int4> nbr(c.natoms);
  TB_CUDA(cudaMemcpyAsync(asite.data(), c.d_atom_site, sizeof(int) * c.natoms,
                          cudaMemcpyDeviceToHost, s));
  TB_CUDA(cudaMemcpyAsync(nbr.data(), c.d_nbr, sizeof(int4) * c.natoms, cudaMemcpyDeviceToHost, s));
  TB_CUDA(cudaStreamSynchronize(s));
  const long plane = long(c.ny) * c.nz;
  std::vector<long> a0(ndots + 1);
  for (int d = 0; d <= ndots; d++) {
    const long cell = long(dot_cells[d]) * plane;  // first cell of the dot
    a0[d] = std::lower_bound(asite.begin(), asite.end(), int(cell * 8),
                             [](int site, int v) { return site < v; }) - asite.begin();
  }
  std::vector<int> dot_of(c.natoms, -1);
  for (int d = 0; d < ndots; d++) {
    if (a0[d + 1] <= a0[d]) return set_error(TBGPU_E_ARG);  // an empty dot
    for (long a = a0[d]; a < a0[d + 1]; a++) dot_of[a] = d;
  }
  for (long a = 0; a < c.natoms; a++) {  // the dots must not touch
    const int b[4] = {nbr[a].x, nbr[a].y, nbr[a].z, nbr[a].w};
    if (dot_of[a] < 0) return set_error(TBGPU_E_ARG);
    for (int n = 0; n < 4; n++)
      if (b[n] >= 0 && dot_of[b[n]] != dot_of[a]) return set_error(TBGPU_E_ARG);
  }
  std::vector<long> e0(ndots + 1);
  for (int d = 0; d <= ndots; d++) e0[d] = a0[d] * c.nb;
  // ---- block table ------------------------------------------------------------
  std::vector<int> bdot, dblk0(ndots + 1);
  std::vector<long> blo, bhi;
  for (int d = 0; d < ndots; d++) {
    dblk0[d] = int(bdot.size());
    for (long j = e0[d]; j < e0[d + 1]; j += kChunk) {
      bdot.push_back(d);
      blo.push_back(j);
      bhi.push_back(std::min(j + kChunk, e0[d + 1]));
    }
  }
  dblk0[ndots] = int(bdot.size());
  const int nblk = int(bdot.size());
  const long SA = A.imax + 1, SB = A.imax + 2;
  // ---- device state -----------------------------------------------------------
  // first-pass ring: a size that divides the check interval (graph replays
  // then start on the same slot), at least 3
  int S1 = 3;
  for (int k = 3; k <= 8; k++)
    if (A.conv_skip % k == 0) {
      S1 = k;
      break;
    }
  // graphs need a stream that can be captured: not the legacy default stream
  bool use_graph = A.conv_skip % S1 == 0 && s != nullptr;
  std::vector<VT *> ring(std::max(S1, kMaxK + 1), nullptr);
  VT *W = nullptr;
  int *d_blk_dot = nullptr, *d_dot_blk0 = nullptr, *d_it = nullptr;
  long *d_blo = nullptr, *d_bhi = nullptr;
  double *d_alpha = nullptr, *d_bet = nullptr, *d_tmp = nullptr, *d_part = nullptr;
  double *d_coef = nullptr, *h_alpha = nullptr, *h_bet = nullptr;
  unsigned *d_cnt = nullptr;
  unsigned char *d_skip = nullptr, *d_done = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  auto cleanup = [&]() {
    cudaStreamSynchronize(s);
    c.d_skip = nullptr;
    cudaFree(d_skip);
    cudaFree(d_done);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (auto p : ring) if (p) cudaFree(p);
    cudaFree(W); cudaFree(d_blk_dot); cudaFree(d_dot_blk0); cudaFree(d_it); cudaFree(d_blo);
    cudaFree(d_bhi); cudaFree(d_alpha); cudaFree(d_bet); cudaFree(d_tmp); cudaFree(d_part);
    cudaFree(d_coef); cudaFree(d_cnt);
    if (h_alpha) cudaFreeHost(h_alpha);
    if (h_bet) cudaFreeHost(h_bet);
  };
#define B_CUDA(call)                 \
  do {                               \
    if ((call) != cudaSuccess) {     \
      cleanup();                     \
      return set_error(TBGPU_E_CUDA); \
    }                                \
  } while (0)
#define B_RC(expr)      \
  do {                  \
    int rc_ = (expr);   \
    if (rc_) {          \
      cleanup();        \
      return rc_;       \
    }                   \
  } while (0)
  const size_t vbytes = sizeof(VT) * dim;
  for (int i = 0; i < S1; i++) B_CUDA(cudaMalloc(&ring[i], vbytes));
  B_CUDA(cudaMalloc(&W, vbytes));
  B_CUDA(cudaMalloc(&d_blk_dot, sizeof(int) * nblk));
  B_CUDA(cudaMalloc(&d_dot_blk0, sizeof(int) * (ndots + 1)));
  B_CUDA(cudaMalloc(&d_blo, sizeof(long) * nblk));
  B_CUDA(cudaMalloc(&d_bhi, sizeof(long) * nblk));
  B_CUDA(cudaMalloc(&d_it, sizeof(int)));
  B_CUDA(cudaMalloc(&d_alpha, sizeof(double) * SA * ndots));
  B_CUDA(cudaMalloc(&d_bet, sizeof(double) * SB * ndots));
  B_CUDA(cudaMalloc(&d_tmp, sizeof(double) * ndots));
  B_CUDA(cudaMalloc(&d_part, sizeof(double) * nblk));
  B_CUDA(cudaMalloc(&d_cnt, sizeof(unsigned) * ndots));
  // converged dots drop out of the products (per-atom mask) and of the
  // segmented updates (per-dot flag)
  B_CUDA(cudaMalloc(&d_skip, c.natoms));
  B_CUDA(cudaMalloc(&d_done, ndots));
  B_CUDA(cudaMemsetAsync(d_skip, 0, c.natoms, s));
  B_CUDA(cudaMemsetAsync(d_done, 0, ndots, s));
  c.d_skip = d_skip;
  // pinned copies of alpha and beta, one slot per check in flight
  constexpr int kAhead = 2;
  constexpr int kSlots = kAhead + 1;
  B_CUDA(cudaMallocHost(&h_alpha, sizeof(double) * SA * ndots * kSlots));
  B_CUDA(cudaMallocHost(&h_bet, sizeof(double) * SB * ndots * kSlots));
  B_CUDA(cudaMemcpyAsync(d_blk_dot, bdot.data(), sizeof(int) * nblk, cudaMemcpyHostToDevice, s));
  B_CUDA(cudaMemcpyAsync(d_dot_blk0, dblk0.data(), sizeof(int) * (ndots + 1),
                         cudaMemcpyHostToDevice, s));
  B_CUDA(cudaMemcpyAsync(d_blo, blo.data(), sizeof(long) * nblk, cudaMemcpyHostToDevice, s));
  B_CUDA(cudaMemcpyAsync(d_bhi, bhi.data(), sizeof(long) * nblk, cudaMemcpyHostToDevice, s));
  B_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned) * ndots, s));
  B_CUDA(cudaMemsetAsync(d_alpha, 0, sizeof(double) * SA * ndots, s));
  B_CUDA(cudaMemsetAsync(d_bet, 0, sizeof(double) * SB * ndots, s));
  const Seg SG{d_blk_dot, d_blo, d_bhi, d_dot_blk0};
  const double2 *R0 = reinterpret_cast<const double2 *>(r0_dev);

  auto start = [&]() -> int {
    k_bnorm<double2><<<nblk, kBT, 0, s>>>(SG, R0, d_part, d_cnt, d_tmp, 1, 0);
    k_bdivide<VT><<<nblk, kBT, 0, s>>>(SG, R0, d_tmp, ring[0]);
    k_bnorm<VT><<<nblk, kBT, 0, s>>>(SG, ring[0], d_part, d_cnt, d_bet, SB, 0);
    if (cudaMemsetAsync(d_it, 0, sizeof(int), s) != cudaSuccess) return set_error(TBGPU_E_CUDA);
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : set_error(TBGPU_E_CUDA);
  };
  // iteration it (host index, for the ring slot) with ring size S
  auto step = [&](int it, int S) -> int {
    VT *rc_ = ring[it % S], *rp_ = ring[(it + S - 1) % S], *ro = ring[(it + 1) % S];
    int r_ = hx_plain(c, rc_, W, s);
    if (r_) return r_;
    k_balpha<VT><<<nblk, kBT, 0, s>>>(SG, rc_, W, d_bet, d_alpha, SA, SB, d_it, d_part, d_cnt,
                                      d_done);
    k_bupdate<VT><<<nblk, kBT, 0, s>>>(SG, W, rc_, rp_, ro, d_alpha, d_bet, SA, SB, d_it, d_part,
                                       d_cnt, d_done);
    k_badvance<<<1, 1, 0, s>>>(d_it);
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : set_error(TBGPU_E_CUDA);
  };

  auto mark = [&](int d) -> int {
    const long n = a0[d + 1] - a0[d];
    k_bmark<<<unsigned(std::max<long>(1, std::min<long>((n + 255) / 256, 1024))), 256, 0, s>>>(
        a0[d], a0[d + 1], d, d_skip, d_done);
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : set_error(TBGPU_E_CUDA);
  };

  // ---- first pass ---------------------------------------------------------------
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, s);
  B_RC(start());
  const std::vector<int> checks = check_points(A.conv_start, A.conv_skip, A.imax);
  std::vector<DotState> st(ndots);
  const double res = 100.0 * A.tol;
  int launched = 0;
  auto run_to = [&](int upto) -> int {  // iterations [launched, upto)
    const int lim = std::min(upto, A.imax - 1);
    while (launched < lim) {
      // (the first iteration always runs uncaptured: the product kernels set
      // their launch attributes on first use)
      if (use_graph && launched > 0 && lim - launched >= A.conv_skip &&
          (launched % S1) == (checks.empty() ? 1 : checks[0] % S1)) {
        if (!gexec) {  // capture one check interval, starting on this ring slot
          if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();  // not capturable here: launch directly
            use_graph = false;
            continue;
          }
          int r_ = TBGPU_OK;
          for (int k = 0; k < A.conv_skip && !r_; k++) r_ = step(launched + k, S1);
          if (cudaStreamEndCapture(s, &graph) != cudaSuccess || r_) return set_error(TBGPU_E_CUDA);
          if (cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) return set_error(TBGPU_E_CUDA);
        }
        if (cudaGraphLaunch(gexec, s) != cudaSuccess) return set_error(TBGPU_E_CUDA);
        launched += A.conv_skip;
      } else {
        int r_ = step(launched, S1);
        if (r_) return r_;
        launched++;
      }
    }
    return TBGPU_OK;
  };
  // The GPU runs up to kAhead check intervals ahead of the host's test; each
  // check in flight copies alpha and beta into its own pinned slot.
  struct Pending {
    int at, slot;
    cudaEvent_t ev;
  };
  std::vector<Pending> pend;
  auto drop_pending = [&]() {
    for (auto &p : pend) cudaEventDestroy(p.ev);
    pend.clear();
  };
  size_t qi = 0;
  auto fill = [&]() -> int {
    while (qi < checks.size() && pend.size() < size_t(kAhead)) {
      const int at = checks[qi];
      int r_ = run_to(at);
      if (r_) return r_;
      const int sl = int(qi % kSlots);
      double *ha = h_alpha + size_t(sl) * SA * ndots, *hb = h_bet + size_t(sl) * SB * ndots;
      cudaEvent_t ev;
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
          cudaMemcpy2DAsync(ha, sizeof(double) * SA, d_alpha, sizeof(double) * SA,
                            sizeof(double) * at, ndots, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaMemcpy2DAsync(hb, sizeof(double) * SB, d_bet, sizeof(double) * SB,
                            sizeof(double) * (at + 1), ndots, cudaMemcpyDeviceToHost,
                            s) != cudaSuccess ||
          cudaEventRecord(ev, s) != cudaSuccess)
        return set_error(TBGPU_E_CUDA);
      pend.push_back({at, sl, ev});
      qi++;
    }
    return TBGPU_OK;
  };
  int final_all = -1;
  {
    int r_ = fill();
    if (r_) {
      drop_pending();
      cleanup();
      return r_;
    }
  }
  while (!pend.empty()) {
    const Pending p = pend.front();
    pend.erase(pend.begin());
    const int at = p.at;
    if (cudaEventSynchronize(p.ev) != cudaSuccess) {
      cudaEventDestroy(p.ev);
      drop_pending();
      cleanup();
      return set_error(TBGPU_E_CUDA);
    }
    cudaEventDestroy(p.ev);
    const double *sa_ = h_alpha + size_t(p.slot) * SA * ndots;
    const double *sb_ = h_bet + size_t(p.slot) * SB * ndots;
    std::atomic<bool> bad{false};
    std::vector<char> was_done(ndots);
    for (int d = 0; d < ndots; d++) was_done[d] = st[d].done;
    parallel_for(ndots, [&](int d) {
      DotState &D = st[d];
      if (D.done) return;
      const double *ha = sa_ + d * SA, *hb = sb_ + d * SB;
      for (int i = 0; i < at; i++)
        if (!std::isfinite(ha[i])) bad = true;
      if (A.req1 > 0 && int(D.c1.size()) <= A.req1)
        check_window(at, ha, hb + 1, A.emin1[d], A.emax1[d], A.tol, res, D.c1, D.i1,
                     0x51ED27ULL * at + 1);
      if (A.req2 > 0 && int(D.c2.size()) <= A.req2)
        check_window(at, ha, hb + 1, A.emin2[d], A.emax2[d], A.tol, res, D.c2, D.i2,
                     0x51ED27ULL * at + 2);
      const bool more =
          (at + 1 < A.imax) && (int(D.c1.size()) < A.req1 || int(D.c2.size()) < A.req2);
      if (!more) {
        D.done = true;
        D.final_it = at;
        D.Ta.assign(ha, ha + at);
        D.Tb.assign(hb, hb + at + 1);  // bet[0..at]
      }
    });
    if (bad) {
      drop_pending();
      cleanup();
      return set_error(TBGPU_E_NUMERIC);
    }
    if (std::all_of(st.begin(), st.end(), [](const DotState &D) { return D.done; })) {
      final_all = at;
      break;
    }
    int r_ = TBGPU_OK;
    for (int d = 0; d < ndots && !r_; d++)
      if (st[d].done && !was_done[d]) r_ = mark(d);
    if (!r_) r_ = fill();
    if (r_) {
      drop_pending();
      cleanup();
      return r_;
    }
  }
  drop_pending();
  if (final_all < 0) {  // iteration limit: the dots not done keep T up to there
    B_RC(run_to(A.imax));
    const int at = launched;
    B_CUDA(cudaMemcpy2DAsync(h_alpha, sizeof(double) * SA, d_alpha, sizeof(double) * SA,
                             sizeof(double) * at, ndots, cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaMemcpy2DAsync(h_bet, sizeof(double) * SB, d_bet, sizeof(double) * SB,
                             sizeof(double) * (at + 1), ndots, cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaStreamSynchronize(s));
    for (int d = 0; d < ndots; d++)
      if (!st[d].done) {
        st[d].done = true;
        st[d].final_it = at;
        st[d].Ta.assign(h_alpha + d * SA, h_alpha + d * SA + at);
        st[d].Tb.assign(h_bet + d * SB, h_bet + d * SB + at + 1);
      }
  }
  B_CUDA(cudaEventRecord(t1, s));
  B_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  c.stats.solve_ms = ms;
  c.stats.lanczos_iterations = launched;
  // results per dot, ascending
  std::vector<std::vector<std::pair<double, int>>> fd(ndots);
  int total = 0;
  for (int d = 0; d < ndots; d++) {
    for (size_t k = 0; k < st[d].c1.size(); k++) fd[d].push_back({st[d].c1[k], st[d].i1[k]});
    for (size_t k = 0; k < st[d].c2.size(); k++) fd[d].push_back({st[d].c2[k], st[d].i2[k]});
    std::stable_sort(fd[d].begin(), fd[d].end(),
                     [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
                       return x.first < y.first;
                     });
    const int n = std::min(int(fd[d].size()), vstride);
    for (int k = 0; k < n; k++) values[size_t(d) * vstride + k] = fd[d][k].first;
    if (found) found[d] = n;
    if (iterations) iterations[d] = st[d].final_it;
    total += n;
  }
  c.stats.vectors_ms = 0.0;
  c.stats.refine_ms = 0.0;
  // ---- second pass: eigenvectors ---------------------------------------------------
  const int nvec = std::min(std::max(maxvec, 0), kMaxVec);
  std::vector<int> nv_dot(ndots, 0);
  int maxit = 0;
  for (int d = 0; d < ndots; d++) {
    nv_dot[d] = std::min(nvec, int(fd[d].size()));
    for (int k = 0; k < nv_dot[d]; k++) maxit = std::max(maxit, fd[d][k].second);
  }
  if (V_dev && nvec > 0 && maxit > 0) {
    // coefficients per dot: inverse iteration on the dot's tridiagonal at the
    // iteration of each eigenvalue's convergence; 1/bet folded in
    std::vector<double> coef(size_t(ndots) * maxit * nvec, 0.0);
    bool bad = false;
    parallel_for(ndots, [&](int d) {
      Rng rng{0x9E3779B97F4A7C15ULL ^ (0x100000001B3ULL * (unsigned long long)(d + 1))};
      std::vector<double> x;
      for (int k = 0; k < nv_dot[d]; k++) {
        const int req = fd[d][k].second;
        if (!inverse_iteration(req, st[d].Ta.data(), st[d].Tb.data() + 1, fd[d][k].first, rng, x)) {
          bad = true;
          return;
        }
        for (int it = 0; it < req; it++)
          coef[(size_t(d) * maxit + it) * nvec + k] = x[it] / st[d].Tb[it];
      }
    });
    if (bad) {
      cleanup();
      return set_error(TBGPU_E_NUMERIC);
    }
    const int K = kMaxK;
    const int S2 = K + 1;
    for (int i = S1; i < S2; i++) B_CUDA(cudaMalloc(&ring[i], vbytes));
    B_CUDA(cudaMalloc(&d_coef, sizeof(double) * ndots * kMaxK * kMaxVec));
    B_CUDA(cudaMemsetAsync(V_dev, 0, sizeof(double2) * dim * nvec, s));
    // each dot regenerates its recurrence up to its own last needed
    // iteration and then drops out
    std::vector<int> dot_maxit(ndots, 0);
    for (int d = 0; d < ndots; d++)
      for (int k = 0; k < nv_dot[d]; k++) dot_maxit[d] = std::max(dot_maxit[d], fd[d][k].second);
    B_CUDA(cudaMemsetAsync(d_skip, 0, c.natoms, s));
    B_CUDA(cudaMemsetAsync(d_done, 0, ndots, s));
    cudaEventRecord(t0, s);
    B_RC(start());
    for (int d = 0; d < ndots; d++)
      if (dot_maxit[d] == 0) B_RC(mark(d));
    std::vector<double> ch(size_t(ndots) * kMaxK * kMaxVec);
    int it0 = 0;
    for (int it = 0; it < maxit; it++) {
      B_RC(step(it, S2));
      for (int d = 0; d < ndots; d++)
        if (dot_maxit[d] == it + 1) B_RC(mark(d));
      if ((it + 1 - it0) == K || it == maxit - 1) {
        const int nk = it + 1 - it0;
        RingPtrs<VT> P{};
        for (int k = 0; k < nk; k++) P.r[k] = ring[(it0 + k) % S2];
        std::fill(ch.begin(), ch.end(), 0.0);
        for (int d = 0; d < ndots; d++)
          for (int k = 0; k < nk; k++)
            for (int e = 0; e < nvec; e++)
              ch[size_t(d) * kMaxK * kMaxVec + k * nvec + e] =
                  coef[(size_t(d) * maxit + it0 + k) * nvec + e];
        // the stream is in order: the coefficients of the previous chunk
        // have been consumed when this copy runs
        B_CUDA(cudaMemcpyAsync(d_coef, ch.data(), sizeof(double) * ch.size(),
                               cudaMemcpyHostToDevice, s));
        k_baccum<VT><<<nblk, kBT, 0, s>>>(SG, nk, nvec, P, d_coef,
                                          reinterpret_cast<double2 *>(V_dev), dim);
        B_CUDA(cudaGetLastError());
        B_CUDA(cudaStreamSynchronize(s));  // ch is reused for the next chunk
        it0 = it + 1;
      }
    }
    cudaEventRecord(t1, s);
    B_CUDA(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&ms, t0, t1);
    c.stats.vectors_ms = ms;
    c.d_skip = nullptr;  // the refinement's products cover every dot
    if (kMixed) {  // double-precision Rayleigh-Ritz, dot by dot
      std::vector<double> vals(size_t(ndots) * nvec, 0.0);
      for (int d = 0; d < ndots; d++)
        for (int k = 0; k < nv_dot[d]; k++) vals[size_t(d) * nvec + k] = fd[d][k].first;
      c.state_resid.assign(size_t(ndots) * nvec, 0.0);
      c.state_delta.assign(size_t(ndots) * nvec, 0.0);
      std::vector<long> off(ndots), len(ndots);
      for (int d = 0; d < ndots; d++) {
        off[d] = e0[d];
        len[d] = e0[d + 1] - e0[d];
      }
      cudaEventRecord(t0, s);
      B_RC(refine_ritz(c, V_dev, nvec, dim, ndots, off.data(), len.data(), vals.data(),
                       c.state_resid.data(), c.state_delta.data(), s, nv_dot.data()));
      cudaEventRecord(t1, s);
      B_CUDA(cudaStreamSynchronize(s));
      cudaEventElapsedTime(&ms, t0, t1);
      c.stats.refine_ms = ms;
      for (int d = 0; d < ndots; d++)
        for (int k = 0; k < std::min(nv_dot[d], vstride); k++)
          values[size_t(d) * vstride + k] = vals[size_t(d) * nvec + k];
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cleanup();
#undef B_CUDA
#undef B_RC
  return total;
}

int solve_batch(Ctx &c, int ndots, const int *dot_cells, const BatchArgs &A, const double *r0_dev,
                double *values, int vstride, int *found, int *iterations, double *V_dev,
                int maxvec) {
  if (!c.built) return set_error(TBGPU_E_STATE);
  if (c.bloch) return set_error(TBGPU_E_UNSUPPORTED);
  if (ndots < 1 || !dot_cells || !r0_dev || !values || vstride < 1 || A.imax < 2 ||
      A.conv_skip < 1 || A.tol <= 0.0 || !A.emin1 || !A.emax1 || !A.emin2 || !A.emax2 ||
      maxvec > kMaxVec)
    return set_error(TBGPU_E_ARG);
  for (int d = 0; d < ndots; d++)
    if (dot_cells[d] < 0 || dot_cells[d + 1] <= dot_cells[d] || dot_cells[d + 1] > c.nx)
      return set_error(TBGPU_E_ARG);
  if (c.lanczos_f32)
    return solve_batch_t<float2>(c, ndots, dot_cells, A, r0_dev, values, vstride, found,
                                 iterations, V_dev, maxvec);
  return solve_batch_t<double2>(c, ndots, dot_cells, A, r0_dev, values, vstride, found,
                                iterations, V_dev, maxvec);
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_eigensolve_lanczos_batched(
    tbgpu_ctx *ctx, int ndots, const int *dot_cells, int ConvCheckStartIter,
    int ConvCheckSkipRate, int imax, int requested1, int requested2, const double *emin1,
    const double *emax1, const double *emin2, const double *emax2, double tolerance,
    const double *r0_dev, double *values, int values_stride, int *found, int *iterations,
    double *vectors_dev, int max_vectors) {
  if (!ctx || misaligned16(r0_dev) || misaligned16(vectors_dev)) return set_error(TBGPU_E_ARG);
  BatchArgs A{ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2, tolerance,
              emin1, emax1, emin2, emax2};
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  const int rc = solve_batch(c, ndots, dot_cells, A, r0_dev, values, values_stride, found,
                             iterations, vectors_dev, max_vectors);
  if (rc < 0) return rc;
  // a bounded device-side wait that ran out in any product of the solve
  const int st = take_status(c);
  return st ? st : rc;
}
