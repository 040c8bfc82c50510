// Lanczos eigensolver driver with the semantics of the reference's
// eigensolve_lanczos (eigen/src/lanczos.c:1823-2089).
//
// Device side, per iteration n (single_lanczos_iteration, lanczos.c:421-757):
//   k_spmv (fused):  w = H q_n with q_n = r_{n-1} / beta_{n-1} formed on the
//                    fly, alpha_n = Re<q_n, w>            (spmv.cu)
//   k_update:        r_n = w - (alpha_n q_n + beta_{n-1} q_{n-1}),
//                    beta_n = ||r_n||
// Vectors are kept as the unnormalised r's in a ring of buffers; q's are
// formed on the fly, so an iteration moves the Hamiltonian once and six
// vector-lengths of data.  alpha/beta live in device memory; the host never
// waits inside the recurrence.
//
// Host side: the convergence test (find_converged_eigval, lanczos.c:764-996)
// runs on a copy of the tridiagonal matrix while the GPU continues with the
// next batch of iterations; the iteration count and the tridiagonal matrix
// used are those of the check that declared convergence, as in the
// reference.  Eigenvectors: second pass (eigenvectorsLanczos, method 3,
// lanczos.c:1364-1689) with the Ritz combination accumulated in chunks of
// iterations (k_accum) rather than one axpy per eigenvector per iteration.
#include <chrono>
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstring>
#include <vector>

#include "host_par.h"
#include "lanczos_step.cuh"
#include "reduce.cuh"
#include "tbgpu_internal.cuh"

namespace tbgpu {

constexpr int kRedThreads = 256;

int ensure_partials(Ctx &c, int nblocks) {
  if (nblocks <= c.partial_cap) return TBGPU_OK;
  if (c.d_partial) cudaFree(c.d_partial);
  c.d_partial = nullptr;
  c.partial_cap = 0;
  if (cudaMalloc(&c.d_partial, sizeof(double) * nblocks) != cudaSuccess)
    return set_error(TBGPU_E_NOMEM);
  c.partial_cap = nblocks;
  return TBGPU_OK;
}

static unsigned red_grid(const Ctx &c, long n2) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  long want = (n2 + kRedThreads - 1) / kRedThreads;
  long g = std::min<long>(want, long(sms) * 8);
  return unsigned(std::max<long>(g, 1));
}

// Vector kernels for complex double (double2) or, in the mixed-precision
// solve, complex float (float2) Lanczos vectors; arithmetic and the norms
// are double in both.
__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }
template <typename VT> __device__ __forceinline__ VT narrow(double x, double y);
template <> __device__ __forceinline__ double2 narrow<double2>(double x, double y) {
  return make_double2(x, y);
}
template <> __device__ __forceinline__ float2 narrow<float2>(double x, double y) {
  return make_float2(float(x), float(y));
}

// out[idx] = sqrt(sum |x|^2)
template <typename VT>
__global__ void __launch_bounds__(kRedThreads)
    k_norm(long n2, const VT *__restrict__ x, double *partial, unsigned *counter,
           double *out, int idx) {
  double s = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    const double2 v = widen(x[j]);
    s += v.x * v.x + v.y * v.y;
  }
  grid_reduce<kRedThreads>(s, partial, counter, out, idx, true);
}

// y = x / (*den)   (lanczos_initialize divides by the norm, eigsys3d_par.c:199-211)
template <typename VT>
__global__ void k_divide(long n2, const double2 *__restrict__ x, const double *den,
                         VT *__restrict__ y) {
  const double d = *den;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    const double2 v = x[j];
    y[j] = narrow<VT>(v.x / d, v.y / d);
  }
}

// r_n = w - (alpha q + beta_prev q_prev), q = rc/bet[it], q_prev = rp/bet[it-1];
// bet[it+1] = ||r_n||.  bet[0] is the norm of the start vector.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads)
    k_update(long n2, const VT *__restrict__ w, const VT *__restrict__ rc,
             const VT *__restrict__ rp, VT *__restrict__ rout,
             const double *alpha, double *bet, int it, double *partial, unsigned *counter) {
  const double al = alpha[it], bprev = bet[it];
  const double iq = 1.0 / bprev;
  const double ip = it > 0 ? 1.0 / bet[it - 1] : 0.0;
  double s = 0.0;
  auto entry = [&](const VT wj, const VT cj, const VT pj) {
    const double2 pv = it > 0 ? widen(pj) : make_double2(0.0, 0.0);
    const double2 rr = lanczos_update_entry(widen(wj), widen(cj), pv, al, bprev, iq, ip);
    const VT r = narrow<VT>(rr.x, rr.y);
    const double2 rw = widen(r);  // the norm of the vector as stored
    s += rw.x * rw.x + rw.y * rw.y;
    return r;
  };
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nth = (long)gridDim.x * blockDim.x;
  if constexpr (sizeof(VT) == sizeof(float2)) {
    // complex floats two at a time: 16-byte loads and stores (the vectors
    // start on 16-byte boundaries); each entry computes as one at a time
    const long n4 = n2 / 2;
    const float4 *w4 = reinterpret_cast<const float4 *>(w);
    const float4 *c4 = reinterpret_cast<const float4 *>(rc);
    const float4 *p4 = reinterpret_cast<const float4 *>(rp);
    float4 *o4 = reinterpret_cast<float4 *>(rout);
    for (long j = tid; j < n4; j += nth) {
      const float4 a = w4[j], c = c4[j];
      const float4 p = it > 0 ? p4[j] : make_float4(0.f, 0.f, 0.f, 0.f);
      const VT r0 = entry(VT{a.x, a.y}, VT{c.x, c.y}, VT{p.x, p.y});
      const VT r1 = entry(VT{a.z, a.w}, VT{c.z, c.w}, VT{p.z, p.w});
      o4[j] = make_float4(r0.x, r0.y, r1.x, r1.y);
    }
    if ((n2 & 1) && tid == 0) {  // an odd length's last entry
      const long j = n2 - 1;
      rout[j] = entry(w[j], rc[j], it > 0 ? rp[j] : VT{});
    }
  } else {
    for (long j = tid; j < n2; j += nth) rout[j] = entry(w[j], rc[j], it > 0 ? rp[j] : VT{});
  }
  grid_reduce<kRedThreads>(s, partial, counter, bet, it + 1, true);
}

// Folded operator F = factor (H - s2)(H - s1) + offset (matvect_mult2,
// nemo3d/src/base/h_cvectr_mult.c:156-198), after its two products:
// w = factor * w + offset * q with q = rc / bet[it] (rc itself when bet is
// null), and, with alpha_out, alpha = Re<q, w> reduced deterministically.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads)
    k_fold_combine(long n2, const VT *__restrict__ rc, const double *bet, int it, double factor,
                   double offset, VT *__restrict__ w, double *partial, unsigned *counter,
                   double *alpha_out, int aidx) {
  const double iq = bet ? 1.0 / bet[it] : 1.0;
  double s = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    const double2 cv = widen(rc[j]), wv = widen(w[j]);
    const double qx = cv.x * iq, qy = cv.y * iq;
    const VT o = narrow<VT>(factor * wv.x + offset * qx, factor * wv.y + offset * qy);
    w[j] = o;
    const double2 ov = widen(o);
    s += qx * ov.x + qy * ov.y;
  }
  if (alpha_out) grid_reduce<kRedThreads>(s, partial, counter, alpha_out, aidx, false);
}

// out[idx] = Re<a, b> (deterministic)
__global__ void __launch_bounds__(kRedThreads)
    k_rdot(long n2, const double2 *__restrict__ a, const double2 *__restrict__ b,
           double *partial, unsigned *counter, double *out, int idx) {
  double s = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x)
    s += a[j].x * b[j].x + a[j].y * b[j].y;
  grid_reduce<kRedThreads>(s, partial, counter, out, idx, false);
}

// y = F x on double vectors in the reference's order (tmp: one vector)
int fold_product(Ctx &c, const double *x, double *y, double *tmp, cudaStream_t s) {
  int rc = launch_spmv(c, x, tmp, c.fold_s1, nullptr, 0, nullptr, 0, s);
  if (!rc) rc = launch_spmv(c, tmp, y, c.fold_s2, nullptr, 0, nullptr, 0, s);
  if (rc) return rc;
  const long n2 = c.natoms * c.nb;
  k_fold_combine<double2><<<red_grid(c, n2), kRedThreads, 0, s>>>(
      n2, reinterpret_cast<const double2 *>(x), nullptr, 0, c.fold_factor, c.fold_offset,
      reinterpret_cast<double2 *>(y), nullptr, nullptr, nullptr, 0);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// Rayleigh quotients <v, H v> / <v, v> of nv double vectors in the reference's
// order (the energies of a folded solve's eigenvectors)
static int rayleigh_quotients(Ctx &c, const double *V, int nv, std::vector<double> &out,
                              cudaStream_t s) {
  const long n2 = c.natoms * c.nb;
  double *y = nullptr, *d = nullptr;
  out.assign(nv, 0.0);
  if (solver_alloc(c.device, &y, sizeof(double2) * n2, s) != cudaSuccess ||
      solver_alloc(c.device, &d, sizeof(double) * 2 * std::max(nv, 1), s) != cudaSuccess) {
    if (y) cudaFreeAsync(y, s);
    return set_error(TBGPU_E_NOMEM);
  }
  const unsigned rg = red_grid(c, n2);
  int rc = ensure_partials(c, int(rg));
  for (int e = 0; e < nv && !rc; e++) {
    const double2 *v = reinterpret_cast<const double2 *>(V) + size_t(e) * n2;
    rc = launch_spmv(c, reinterpret_cast<const double *>(v), y, 0.0, nullptr, 0, nullptr, 0, s);
    if (rc) break;
    k_rdot<<<rg, kRedThreads, 0, s>>>(n2, v, reinterpret_cast<const double2 *>(y), c.d_partial,
                                      c.d_counter, d, 2 * e);
    k_rdot<<<rg, kRedThreads, 0, s>>>(n2, v, v, c.d_partial, c.d_counter, d, 2 * e + 1);
  }
  std::vector<double> h(2 * std::max(nv, 1));
  if (!rc && (cudaMemcpyAsync(h.data(), d, sizeof(double) * 2 * nv, cudaMemcpyDeviceToHost, s) !=
                  cudaSuccess ||
              cudaStreamSynchronize(s) != cudaSuccess))
    rc = set_error(TBGPU_E_CUDA);
  for (int e = 0; e < nv && !rc; e++) out[e] = h[2 * e] / h[2 * e + 1];
  cudaFreeAsync(y, s);
  cudaFreeAsync(d, s);
  return rc;
}

constexpr int kMaxChunk = 32;
constexpr int kVecGroup = 16;
// the regenerating eigenvector pass accumulates up to 64 rows (its columns'
// chunks together) into groups of 8 eigenvectors
constexpr int kRegenRows = 64;
constexpr int kRegenGroup = 8;
template <typename VT, int ROWS = kMaxChunk>
struct ChunkPtrs {
  const VT *r[ROWS];
};

// Coefficients of one chunk, passed by value: the kernel reads them from the
// parameter bank as FMA operands (no shared-memory traffic per element).
template <int ROWS = kMaxChunk, int VG = kVecGroup>
struct ChunkCoef {
  double c[ROWS][VG];
};

// V[e] += sum_k coef[k][e] * R_k for one group of NV vectors (memory bound:
// the chunk's r-vectors and the NV eigenvectors are streamed once).  Every
// launch runs all kMaxChunk rows: the caller points the rows past the
// chunk's end at a valid vector and leaves their coefficients zero, so the
// loop has no guards and the r-values are loaded eight at a time ahead of
// their FMAs with registers held to 64 (four blocks per SM) up to 8
// vectors: 2.9 against 4.8 ms per 32-vector chunk of 8 eigenvectors at
// 20.5M entries (5.4 against 3.3 TB/s), where one load per iteration under
// the compiler's own scheduling left each thread waiting on memory with too
// few warps resident.
constexpr int kAccumBatch = 8;
template <int NV, typename VT>
constexpr int accum_min_blocks() {  // float vectors: more registers to widen them
  return sizeof(VT) != sizeof(double2) ? (NV <= 12 ? 2 : 1) : NV <= 8 ? 4 : NV <= 12 ? 2 : 1;
}
template <int NV, typename VT, int ROWS, int VG>
__global__ void __launch_bounds__(256, accum_min_blocks<NV, VT>())
    k_accum(long n2, ChunkPtrs<VT, ROWS> R, ChunkCoef<ROWS, VG> C, double2 *__restrict__ V) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    double2 acc[NV];
#pragma unroll
    for (int e = 0; e < NV; e++) acc[e] = V[e * n2 + j];
#pragma unroll
    for (int k0 = 0; k0 < ROWS; k0 += kAccumBatch) {
      double2 r[kAccumBatch];
#pragma unroll
      for (int b = 0; b < kAccumBatch; b++) r[b] = widen(__ldg(R.r[k0 + b] + j));
#pragma unroll
      for (int b = 0; b < kAccumBatch; b++)
#pragma unroll
        for (int e = 0; e < NV; e++) {
          acc[e].x = fma(C.c[k0 + b][e], r[b].x, acc[e].x);
          acc[e].y = fma(C.c[k0 + b][e], r[b].y, acc[e].y);
        }
    }
#pragma unroll
    for (int e = 0; e < NV; e++) V[e * n2 + j] = acc[e];
  }
}

template <typename VT, int ROWS = kMaxChunk, int VG = kVecGroup>
static void launch_accum(int nv, unsigned grid, cudaStream_t s, long n2,
                         const ChunkPtrs<VT, ROWS> &R, const ChunkCoef<ROWS, VG> &C,
                         double2 *V) {
  switch (nv) {
#define TBGPU_ACCUM_CASE(N) \
  case N:                   \
    if constexpr (N <= VG) k_accum<N, VT, ROWS, VG><<<grid, 256, 0, s>>>(n2, R, C, V); \
    break;
    TBGPU_ACCUM_CASE(1) TBGPU_ACCUM_CASE(2) TBGPU_ACCUM_CASE(3) TBGPU_ACCUM_CASE(4)
    TBGPU_ACCUM_CASE(5) TBGPU_ACCUM_CASE(6) TBGPU_ACCUM_CASE(7) TBGPU_ACCUM_CASE(8)
    TBGPU_ACCUM_CASE(9) TBGPU_ACCUM_CASE(10) TBGPU_ACCUM_CASE(11) TBGPU_ACCUM_CASE(12)
    TBGPU_ACCUM_CASE(13) TBGPU_ACCUM_CASE(14) TBGPU_ACCUM_CASE(15) TBGPU_ACCUM_CASE(16)
#undef TBGPU_ACCUM_CASE
    default: break;
  }
}

// number of 32-bit words of two vectors that differ (bit comparison)
__global__ void k_count_diff(long nwords, const unsigned *__restrict__ a,
                             const unsigned *__restrict__ b, unsigned long long *count) {
  unsigned long long d = 0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < nwords;
       j += (long)gridDim.x * blockDim.x)
    d += a[j] != b[j];
  for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
  if ((threadIdx.x & 31) == 0 && d) atomicAdd(count, d);
}

// ---------------------------------------------------------------------------
// Host: tridiagonal eigenvalues (Sturm bisection in place of LAPACK dstebz,
// lanczos.c:793-811) and inverse iteration (originalInverseIteration,
// lanczos.c:378-418; solve_rtridiag_ii, lanczos.c:249-308).

static int sturm_below(int n, const double *d, const double *e2, double x) {
  int cnt = 0;
  double q = d[0] - x;
  if (q < 0) cnt++;
  for (int i = 1; i < n; i++) {
    if (std::fabs(q) < 1e-300) q = q < 0 ? -1e-300 : 1e-300;
    q = d[i] - x - e2[i - 1] / q;
    if (q < 0) cnt++;
  }
  return cnt;
}

// Sturm counts of kLanes shift points in one pass over T: the counts of
// independent shifts are independent chains of divisions, which the core
// overlaps (one chain alone waits on each division).  Each count is the
// same arithmetic as sturm_below.
constexpr int kLanes = 8;
static void sturm_below_multi(int n, const double *d, const double *e2, const double *x,
                              int *cnt) {
  double q[kLanes];
  int c[kLanes];
  for (int k = 0; k < kLanes; k++) {
    q[k] = d[0] - x[k];
    c[k] = q[k] < 0;
  }
  for (int i = 1; i < n; i++) {
    const double di = d[i], ei = e2[i - 1];
    for (int k = 0; k < kLanes; k++) {
      double qk = q[k];
      if (std::fabs(qk) < 1e-300) qk = qk < 0 ? -1e-300 : 1e-300;
      qk = di - x[k] - ei / qk;
      c[k] += qk < 0;
      q[k] = qk;
    }
  }
  for (int k = 0; k < kLanes; k++) cnt[k] = c[k];
}

// eigenvalues of T (diag d, off-diagonal e) in (vl, vu], ascending: one
// bisection per eigenvalue, kLanes eigenvalues advanced together
static std::vector<double> tri_eigs(int n, const double *d, const double *e, double vl,
                                    double vu) {
  std::vector<double> e2(std::max(n - 1, 1));
  double lo = d[0], hi = d[0];
  for (int i = 0; i < n - 1; i++) e2[i] = e[i] * e[i];
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < n - 1 ? std::fabs(e[i]) : 0.0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
  }
  const int c0 = sturm_below(n, d, e2.data(), vl), c1 = sturm_below(n, d, e2.data(), vu);
  const int ne = std::max(c1 - c0, 0);
  std::vector<double> w(ne);
  const int ngroups = (ne + kLanes - 1) / kLanes;
  parallel_for(ngroups, [&](int gi) {
    double a[kLanes], b[kLanes], mid[kLanes];
    int idx[kLanes], cnt[kLanes], its[kLanes];
    bool live[kLanes];
    for (int k = 0; k < kLanes; k++) {
      const int j = gi * kLanes + k;
      live[k] = j < ne;
      idx[k] = c0 + j;
      a[k] = std::max(vl, lo);
      b[k] = std::min(vu, hi);
      its[k] = 0;
    }
    for (;;) {
      bool any = false;
      for (int k = 0; k < kLanes; k++) {
        if (live[k]) {  // the same stopping rule as one bisection alone
          const double tol = 1e-13 + 2.2e-16 * std::max(std::fabs(a[k]), std::fabs(b[k]));
          if (its[k] >= 200 || b[k] - a[k] <= tol) live[k] = false;
        }
        mid[k] = live[k] ? 0.5 * (a[k] + b[k]) : a[k];
        any = any || live[k];
      }
      if (!any) break;
      sturm_below_multi(n, d, e2.data(), mid, cnt);
      for (int k = 0; k < kLanes; k++) {
        if (!live[k]) continue;
        if (cnt[k] > idx[k]) b[k] = mid[k];
        else a[k] = mid[k];
        its[k]++;
      }
    }
    for (int k = 0; k < kLanes; k++) {
      const int j = gi * kLanes + k;
      if (j < ne) w[j] = 0.5 * (a[k] + b[k]);
    }
  });
  return w;
}

// 20 solves with T - (lambda + 1e-8) on the leading m x m block; x out
bool inverse_iteration(int m, const double *d, const double *e, double lambda, Rng &rng,
                       std::vector<double> &x) {
  std::vector<double> ds(m), g(m), y(m);
  x.assign(m, 0.0);
  for (int i = 0; i < m; i++) ds[i] = d[i] - (lambda + 1e-8);
  double nrm = 0.0;
  for (int i = 0; i < m; i++) {
    y[i] = rng.next();
    nrm += y[i] * y[i];
  }
  nrm = std::sqrt(nrm);
  for (int i = 0; i < m; i++) y[i] /= nrm;
  for (int it = 0; it < 20; it++) {
    double piv = ds[0];
    if (piv == 0.0) return false;
    x[0] = y[0] / piv;
    for (int j = 1; j < m; j++) {
      g[j] = e[j - 1] / piv;
      piv = ds[j] - e[j - 1] * g[j];
      if (piv == 0.0) return false;
      x[j] = (y[j] - e[j - 1] * x[j - 1]) / piv;
    }
    for (int j = m - 1; j > 0; j--) x[j - 1] -= g[j] * x[j];
    nrm = 0.0;
    for (int i = 0; i < m; i++) nrm += x[i] * x[i];
    nrm = std::sqrt(nrm);
    for (int i = 0; i < m; i++) y[i] = x[i] / nrm;
  }
  x = y;
  return true;
}

// inverse_iteration for up to kLanes eigenvalues at once, the solves of the
// lanes interleaved (independent division chains) and each lane's arithmetic
// that of inverse_iteration: x[k] (length m) and ok[k] per lane k < nl.
static void inverse_iteration_multi(int m, const double *d, const double *e, const double *lam,
                                    Rng *rng, int nl, std::vector<double> *x, bool *ok) {
  std::vector<double> ds(size_t(m) * kLanes), g(size_t(m) * kLanes), y(size_t(m) * kLanes),
      xv(size_t(m) * kLanes);
  double nrm[kLanes];
  for (int k = 0; k < kLanes; k++) {
    ok[k] = k < nl;
    nrm[k] = 0.0;
  }
  for (int k = 0; k < nl; k++) {
    for (int i = 0; i < m; i++) {
      ds[size_t(i) * kLanes + k] = d[i] - (lam[k] + 1e-8);
      const double r = rng[k].next();
      y[size_t(i) * kLanes + k] = r;
      nrm[k] += r * r;
    }
    nrm[k] = std::sqrt(nrm[k]);
    for (int i = 0; i < m; i++) y[size_t(i) * kLanes + k] /= nrm[k];
  }
  for (int it = 0; it < 20; it++) {
    double piv[kLanes];
    for (int k = 0; k < kLanes; k++) {
      piv[k] = ds[k];
      if (k < nl && piv[k] == 0.0) ok[k] = false;
      xv[k] = ok[k] ? y[k] / piv[k] : 0.0;
    }
    for (int j = 1; j < m; j++) {
      const double ej = e[j - 1];
      const size_t o = size_t(j) * kLanes, op = size_t(j - 1) * kLanes;
      for (int k = 0; k < kLanes; k++) {
        if (!ok[k]) continue;
        const double gj = ej / piv[k];
        g[o + k] = gj;
        piv[k] = ds[o + k] - ej * gj;
        if (piv[k] == 0.0) {
          ok[k] = false;
          continue;
        }
        xv[o + k] = (y[o + k] - ej * xv[op + k]) / piv[k];
      }
    }
    for (int j = m - 1; j > 0; j--)
      for (int k = 0; k < kLanes; k++)
        if (ok[k]) xv[size_t(j - 1) * kLanes + k] -= g[size_t(j) * kLanes + k] * xv[size_t(j) * kLanes + k];
    for (int k = 0; k < kLanes; k++) nrm[k] = 0.0;
    for (int i = 0; i < m; i++)
      for (int k = 0; k < kLanes; k++) nrm[k] += xv[size_t(i) * kLanes + k] * xv[size_t(i) * kLanes + k];
    for (int k = 0; k < kLanes; k++) nrm[k] = std::sqrt(nrm[k]);
    for (int i = 0; i < m; i++)
      for (int k = 0; k < kLanes; k++)
        if (ok[k]) y[size_t(i) * kLanes + k] = xv[size_t(i) * kLanes + k] / nrm[k];
  }
  for (int k = 0; k < nl; k++) {
    if (!ok[k]) continue;
    x[k].resize(m);
    for (int i = 0; i < m; i++) x[k][i] = y[size_t(i) * kLanes + k];
  }
}

// find_converged_eigval, method 2 (lanczos.c:764-996).  The inverse
// iterations of the candidates run in parallel; the acceptance pass then
// walks the candidates in ascending order exactly as the reference does.
void check_window(int it, const double *al, const double *be, double emin, double emax,
                  double tol, double res, std::vector<double> &conv, std::vector<int> &conv_it,
                  unsigned long long seed) {
  const std::vector<double> ev = tri_eigs(it, al, be, emin, emax);
  const int ne = int(ev.size());
  std::vector<char> cand(ne, 0), ok(ne, 0);
  for (int i = 0; i < ne; i++) {
    if (i > 0 && std::fabs(ev[i - 1] - ev[i]) < std::fabs(1e-80 + ev[i]) * res) continue;
    bool done = false;
    for (double c : conv)
      if (std::fabs(c - ev[i]) < res) done = true;
    cand[i] = !done;
  }
  std::vector<int> cl;  // the candidates, kLanes at a time
  for (int i = 0; i < ne; i++)
    if (cand[i]) cl.push_back(i);
  parallel_for((int(cl.size()) + kLanes - 1) / kLanes, [&](int gi) {
    const int nl = std::min(kLanes, int(cl.size()) - gi * kLanes);
    double lam[kLanes];
    Rng rng[kLanes];
    std::vector<double> x[kLanes];
    bool good[kLanes];
    for (int k = 0; k < nl; k++) {
      const int i = cl[gi * kLanes + k];
      lam[k] = ev[i];
      rng[k] = Rng{seed ^ (0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1))};
    }
    inverse_iteration_multi(it, al, be, lam, rng, nl, x, good);
    for (int k = 0; k < nl; k++) {
      const int i = cl[gi * kLanes + k];
      if (!good[k]) continue;
      bool flag = true;
      for (int q = std::max(it - 2, 0); q < it; q++)
        if (std::fabs(x[k][q]) > tol) flag = false;
      ok[i] = flag;
    }
  });
  for (int i = 0; i < ne; i++) {
    if (!cand[i] || !ok[i]) continue;
    bool done = false;  // may have converged earlier in this same pass
    for (double c : conv)
      if (std::fabs(c - ev[i]) < res) done = true;
    if (done) continue;
    conv.push_back(ev[i]);
    conv_it.push_back(it);
  }
}

struct Timers {
  cudaEvent_t t0, t1, t2, t3;
};

// H*x of one Lanczos step on the context's stored Hamiltonian
static int spmv_step(Ctx &c, const double2 *x, double2 *y, const double *bet, int it,
                     double *alpha, cudaStream_t s) {
  return launch_spmv(c, reinterpret_cast<const double *>(x), reinterpret_cast<double *>(y), 0.0,
                     bet, it, alpha, it, s);
}
static int spmv_step(Ctx &c, const float2 *x, float2 *y, const double *bet, int it,
                     double *alpha, cudaStream_t s) {
  return launch_spmv_f32(c, reinterpret_cast<const float *>(x), reinterpret_cast<float *>(y), 0.0,
                         bet, it, alpha, it, s);
}

// check batches the first pass keeps queued ahead of the host's convergence
// test: the iterations past convergence that run for nothing (at most
// kAhead * ConvCheckSkipRate) against the GPU idling while a test runs
constexpr int kAhead = 4;

template <typename VT>
static int solve_t(Ctx &c, const SolveArgs &A, const double *r0_dev, double *values,
                   int *conv_iters, int *iterations, double *V_dev, int maxvec) {
  constexpr bool kMixed = sizeof(VT) == sizeof(float2);
  if (!c.built) return set_error(TBGPU_E_STATE);
  if (A.imax < 2 || A.conv_skip < 1 || !values || !r0_dev) return set_error(TBGPU_E_ARG);
  if (kMixed && c.bloch) return set_error(TBGPU_E_UNSUPPORTED);
  c.state_resid.clear();
  c.state_delta.clear();
  c.stats.refine_ms = 0.0;
  c.stats.vec_segments = 0;
  c.stats.vec_mismatch = 0;
  c.stats.update_ms = 0.0;
  c.stats.check_ms = 0.0;
  c.stats.wait_ms = 0.0;
  // eigenvector pass by regeneration (tbgpu_set_eigenvector_pass): both
  // passes run a register-streaming kernel whose columns compute as
  // one-column launches -- the pencil kernel when variant 6 is set and
  // applies, else the lane kernel (variant 5)
  const bool f32_ok = !kMixed || c.ham_fp32;
  // folded-spectrum operator (tbgpu_set_fold): two products per step, plain
  // second run for the eigenvectors, double precision only
  const bool fold = c.fold;
  if (fold && kMixed) return set_error(TBGPU_E_UNSUPPORTED);
  c.fold_energy.clear();
  bool regen = !fold && c.vec_pass == 1 && V_dev && maxvec > 0 && lane_supported(c) && f32_ok;
  const int keep_variant = c.spmv_variant;
  const bool pen_variant = keep_variant == 6 || keep_variant == 7;
  if (regen) c.spmv_variant = pen_supported(c) && pen_variant ? keep_variant : 5;
  // the pencil kernels keep the Lanczos vectors in their own layout: the
  // start vector is permuted in and the eigenvectors out
  const bool pen = (c.spmv_variant == 6 || c.spmv_variant == 7) && pen_supported(c) && f32_ok;
  if (!pen && (c.spmv_variant == 6 || c.spmv_variant == 7)) c.spmv_variant = regen ? 5 : 0;
  const long n2_ref = c.natoms * c.nb;           // complex entries, reference order
  const long n2 = pen ? pen_length(c) : n2_ref;  // of the solver's vectors
  const size_t vbytes = sizeof(VT) * n2;        // one Lanczos vector
  const size_t ebytes = sizeof(double2) * n2;   // one eigenvector (always double)
  cudaStream_t s = c.stream;
  const unsigned rg = red_grid(c, n2);
  int rc = ensure_partials(c, int(rg));
  if (rc) return rc;
  long launches = 0;
  c.stats.spmv_ms = 0.0;
  c.stats.spmv_launches = 0;

  // device state
  const int S1 = 3;  // ring of r's for the first pass
  VT *ring[kMaxChunk + 1] = {nullptr};
  VT *W = nullptr;
  double *d_alpha = nullptr, *d_bet = nullptr, *d_tmp = nullptr;
  double *h_alpha = nullptr, *h_bet = nullptr;
  std::vector<cudaEvent_t> spmv_ev, upd_ev;
  // regeneration: the first pass saves r_it and r_{it-1} at every it = 0,
  // L, 2L, ...
  const int L = std::max(c.vec_segment, 16);
  const int P = std::max(1, std::min(c.vec_columns, lane_max_cols(kMixed)));
  std::vector<VT *> ck_cur, ck_prev, rr;  // checkpoints; the pass-2 rings
  unsigned long long *d_diff = nullptr;
  double *r0_pen = nullptr;  // pencil layout: the start vector
  double *V_pen = nullptr;   // ... and the eigenvectors before they go out
  VT *Tf = nullptr;          // folded operator: the first product
  auto drop_checkpoints = [&]() {
    for (VT *q : ck_cur) if (q) cudaFreeAsync(q, s);
    for (VT *q : ck_prev) if (q) cudaFreeAsync(q, s);
    ck_cur.clear();
    ck_prev.clear();
  };
  auto cleanup = [&]() {
    c.spmv_variant = keep_variant;
    drop_checkpoints();
    for (VT *q : rr) if (q) cudaFreeAsync(q, s);
    rr.clear();
    if (d_diff) cudaFreeAsync(d_diff, s);
    d_diff = nullptr;
    if (r0_pen) cudaFreeAsync(r0_pen, s);
    r0_pen = nullptr;
    if (V_pen) cudaFreeAsync(V_pen, s);
    V_pen = nullptr;
    if (Tf) cudaFreeAsync(Tf, s);
    Tf = nullptr;
    for (int i = 0; i <= kMaxChunk; i++)
      if (ring[i]) cudaFreeAsync(ring[i], s);
    if (W) cudaFreeAsync(W, s);
    if (d_alpha) cudaFreeAsync(d_alpha, s);
    if (d_bet) cudaFreeAsync(d_bet, s);
    if (d_tmp) cudaFreeAsync(d_tmp, s);
    if (h_alpha) cudaFreeHost(h_alpha);
    if (h_bet) cudaFreeHost(h_bet);
    for (auto e : spmv_ev) cudaEventDestroy(e);
    for (auto e : upd_ev) cudaEventDestroy(e);
  };
#define SOLVE_CUDA(call)                 \
  do {                                   \
    if ((call) != cudaSuccess) {         \
      cleanup();                         \
      return set_error(TBGPU_E_CUDA);    \
    }                                    \
  } while (0)
#define SOLVE_RC(expr)        \
  do {                        \
    int rc_ = (expr);         \
    if (rc_) {                \
      cleanup();              \
      return rc_;             \
    }                         \
  } while (0)
  // per-solve buffers from the solver's pool (memory kept between solves)
  const int dev = c.device;
  for (int i = 0; i < S1; i++) SOLVE_CUDA(solver_alloc(dev, &ring[i], vbytes, s));
  SOLVE_CUDA(solver_alloc(dev, &W, vbytes, s));
  if (fold) SOLVE_CUDA(solver_alloc(dev, &Tf, vbytes, s));
  SOLVE_CUDA(solver_alloc(dev, &d_alpha, sizeof(double) * (A.imax + 1), s));
  SOLVE_CUDA(solver_alloc(dev, &d_bet, sizeof(double) * (A.imax + 2), s));
  SOLVE_CUDA(solver_alloc(dev, &d_tmp, sizeof(double) * 4, s));
  SOLVE_CUDA(cudaMallocHost(&h_alpha, sizeof(double) * (A.imax + 2) * (kAhead + 1)));
  SOLVE_CUDA(cudaMallocHost(&h_bet, sizeof(double) * (A.imax + 2) * (kAhead + 1)));
  Timers tm;
  cudaEventCreate(&tm.t0);
  cudaEventCreate(&tm.t1);
  cudaEventCreate(&tm.t2);
  cudaEventCreate(&tm.t3);

  if (pen) {
    SOLVE_CUDA(solver_alloc(dev, &r0_pen, ebytes, s));
    SOLVE_RC(pen_permute<double2>(c, reinterpret_cast<const double2 *>(r0_dev),
                                  reinterpret_cast<double2 *>(r0_pen), true, s));
    r0_dev = r0_pen;
  }
  // start vector: r = r0 / ||r0||; bet[0] = ||r||
  auto start = [&](double *bet) -> int {
    k_norm<double2><<<rg, kRedThreads, 0, s>>>(n2, reinterpret_cast<const double2 *>(r0_dev),
                                              c.d_partial, c.d_counter, d_tmp, 0);
    k_divide<VT><<<rg, kRedThreads, 0, s>>>(n2, reinterpret_cast<const double2 *>(r0_dev), d_tmp,
                                            ring[0]);
    k_norm<VT><<<rg, kRedThreads, 0, s>>>(n2, ring[0], c.d_partial, c.d_counter, bet, 0);
    launches += 3;
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : set_error(TBGPU_E_CUDA);
  };
  // one Lanczos iteration with ring size S
  auto step = [&](int it, int S, double *bet) -> int {
    VT *rc_ = ring[it % S], *rp_ = ring[(it + S - 1) % S], *ro = ring[(it + 1) % S];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.profiling) {
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventRecord(e0, s);
    }
    int r_;
    if (fold) {  // W = F q: T = (H - s1) q, W = (H - s2) T, W = factor W + offset q, alpha
      r_ = pen ? launch_spmv_pen_internal<VT>(c, rc_, Tf, c.fold_s1, bet, it, nullptr, 0, s)
               : launch_spmv(c, reinterpret_cast<const double *>(rc_),
                             reinterpret_cast<double *>(Tf), c.fold_s1, bet, it, nullptr, 0, s);
      if (!r_)
        r_ = pen ? launch_spmv_pen_internal<VT>(c, Tf, W, c.fold_s2, nullptr, 0, nullptr, 0, s)
                 : launch_spmv(c, reinterpret_cast<const double *>(Tf),
                               reinterpret_cast<double *>(W), c.fold_s2, nullptr, 0, nullptr, 0,
                               s);
      if (!r_) {
        k_fold_combine<VT><<<rg, kRedThreads, 0, s>>>(n2, rc_, bet, it, c.fold_factor,
                                                      c.fold_offset, W, c.d_partial, c.d_counter,
                                                      d_alpha, it);
        launches += 2;
      }
    } else {
      r_ = pen ? launch_spmv_pen_internal<VT>(c, rc_, W, 0.0, bet, it, d_alpha, it, s)
               : spmv_step(c, rc_, W, bet, it, d_alpha, s);
    }
    if (r_) return r_;
    if (c.profiling) {
      cudaEventRecord(e1, s);
      spmv_ev.push_back(e0);
      spmv_ev.push_back(e1);
    }
    k_update<VT><<<rg, kRedThreads, 0, s>>>(n2, W, rc_, it > 0 ? rp_ : nullptr, ro, d_alpha, bet,
                                            it, c.d_partial, c.d_counter);
    if (c.profiling) {
      cudaEvent_t e2 = nullptr;
      cudaEventCreate(&e2);
      cudaEventRecord(e2, s);
      upd_ev.push_back(e2);  // the update runs from e1 to e2
    }
    launches += 2;
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : set_error(TBGPU_E_CUDA);
  };

  // ---- first pass: eigenvalues --------------------------------------------
  cudaEventRecord(tm.t0, s);
  SOLVE_RC(start(d_bet));
  std::vector<double> c1, c2;
  std::vector<int> i1, i2;
  Rng rng{0x9E3779B97F4A7C15ULL};  // starts of the eigenvector inverse iterations
  const double res = 100.0 * A.tol;
  // the acceptance bound on a tridiagonal eigenvector's last components;
  // the complex-float recurrence may raise it to its own rounding floor: a
  // set floor, or (negative setting) 2^-24 times the Gershgorin bound of the
  // tridiagonal matrix so far, the recurrence's rounding level
  auto accept_bound = [&](int at, const double *al, const double *be) {
    if (!kMixed || c.mixed_accept == 0.0) return A.tol;
    double floor = c.mixed_accept;
    if (floor < 0.0) {
      double g = 0.0;
      for (int i = 0; i < at; i++)
        g = std::max(g, std::fabs(al[i]) + std::fabs(be[i]) + (i > 0 ? std::fabs(be[i - 1]) : 0.0));
      floor = std::ldexp(g, -24);
    }
    return std::max(A.tol, floor);
  };
  // check points exactly as lanczos_tridiagonal's skip counter places them
  auto next_check = [&](int after, int skip_at_after) {
    int skip = skip_at_after;
    for (int it = after + 1; it < A.imax; it++) {
      skip++;
      if (A.conv_start < it && A.conv_skip <= skip) return it;
    }
    return A.imax;  // none before the iteration limit
  };
  // all check points below the iteration limit
  std::vector<int> checks;
  for (int at = next_check(0, 0); at < A.imax; at = next_check(at, 0)) checks.push_back(at);
  // The GPU runs up to kAhead check batches ahead of the host's test (a
  // file-scope constant); each check in flight copies alpha/beta into its
  // own pinned slot.
  const size_t slot = size_t(A.imax) + 2;
  int launched = 0;  // iterations enqueued
  int final_it = -1;
  struct Pending {
    int at, slot;
    cudaEvent_t ev;
  };
  std::vector<Pending> pend;
  // checkpoint of iteration it: copies of r_it and r_{it-1} (stream ordered,
  // after the step that wrote them, before any step overwrites them); when
  // device memory runs short the solve falls back to the second run
  const size_t ring_need = size_t(P) * (kRegenRows / P + 2) * vbytes + (512ull << 20);
  // free device memory is read once, at the first checkpoint; the pass
  // allocates nothing else, so the checkpoints draw on that budget
  size_t ck_budget = 0;
  bool ck_budget_read = false;
  auto checkpoint = [&](int it) -> int {
    if (!ck_budget_read) {
      size_t fre = 0, tot = 0;
      cudaMemGetInfo(&fre, &tot);
      fre += solver_pool_spare(dev);  // the pool's memory kept from earlier solves
      ck_budget = fre > ring_need ? fre - ring_need : 0;
      ck_budget_read = true;
    }
    const size_t need = (it > 0 ? 2 : 1) * vbytes;
    VT *a = nullptr, *b = nullptr;
    bool ok = ck_budget > 2 * vbytes && solver_alloc(dev, &a, vbytes, s) == cudaSuccess;
    if (ok && it > 0) ok = solver_alloc(dev, &b, vbytes, s) == cudaSuccess;
    if (ok) ck_budget -= need;
    if (!ok) {
      cudaGetLastError();  // a failed allocation is not an error of the solve
      if (a) cudaFreeAsync(a, s);
      drop_checkpoints();
      regen = false;
      return TBGPU_OK;
    }
    if (cudaMemcpyAsync(a, ring[it % S1], vbytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        (b && cudaMemcpyAsync(b, ring[(it + S1 - 1) % S1], vbytes, cudaMemcpyDeviceToDevice,
                              s) != cudaSuccess))
      return set_error(TBGPU_E_CUDA);
    ck_cur.push_back(a);
    ck_prev.push_back(b);
    return TBGPU_OK;
  };
  auto enqueue_until = [&](int upto) -> int {  // launch iterations [launched, upto)
    const int lim = std::min(upto, A.imax - 1);
    for (; launched < lim; launched++) {
      if (regen && launched % L == 0) {
        int r_ = checkpoint(launched);
        if (r_) return r_;
      }
      int r_ = step(launched, S1, d_bet);
      if (r_) return r_;
    }
    return TBGPU_OK;
  };
  size_t qi = 0;  // next check to enqueue
  auto fill = [&]() -> int {
    while (qi < checks.size() && pend.size() < size_t(kAhead)) {
      const int at = checks[qi];
      int r_ = enqueue_until(at);
      if (r_) return r_;
      const int sl = int(qi % (kAhead + 1));
      cudaEvent_t ev;
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return set_error(TBGPU_E_CUDA);
      cudaMemcpyAsync(h_alpha + sl * slot, d_alpha, sizeof(double) * at, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(h_bet + sl * slot, d_bet, sizeof(double) * (at + 1), cudaMemcpyDeviceToHost, s);
      if (cudaEventRecord(ev, s) != cudaSuccess) return set_error(TBGPU_E_CUDA);
      pend.push_back({at, sl, ev});
      qi++;
    }
    return TBGPU_OK;
  };
  std::vector<double> Ta, Tb;
  const double *hb_final = h_bet;  // beta copy used by the second pass
  std::vector<double> hb_restore;
  const bool restore = A.restore_its > 0;
  if (restore) {
    // the tridiagonal matrix and eigenvalues of an earlier solve
    // (eigensolve_lanczos with restoreState, lanczos.c:1912-1955): no first
    // pass; every value's eigenvector uses the whole restored matrix
    final_it = launched = A.restore_its;
    Ta.assign(A.restore_alpha, A.restore_alpha + final_it);
    Tb.assign(A.restore_beta, A.restore_beta + final_it);
    hb_restore.assign(size_t(final_it) + 1, 1.0);  // bet[0]: the normalised start
    for (int it = 1; it <= final_it; it++) hb_restore[it] = Tb[it - 1];
    hb_final = hb_restore.data();
    for (int k = 0; k < A.restore_n; k++) {
      c2.push_back(A.restore_values[k]);
      i2.push_back(final_it);
    }
  } else {
  SOLVE_RC(fill());
  while (!pend.empty()) {
    Pending p = pend.front();
    pend.erase(pend.begin());
    const auto w0 = std::chrono::steady_clock::now();
    SOLVE_CUDA(cudaEventSynchronize(p.ev));
    const auto w1 = std::chrono::steady_clock::now();
    c.stats.wait_ms += std::chrono::duration<double, std::milli>(w1 - w0).count();
    cudaEventDestroy(p.ev);
    const double *ha = h_alpha + p.slot * slot, *hb = h_bet + p.slot * slot;
    Ta.assign(ha, ha + p.at);
    // off-diagonal: beta_n couples n and n+1, beta_n = bet[n+1]
    Tb.assign(hb + 1, hb + 1 + p.at);
    for (double v : Ta)
      if (!std::isfinite(v)) {
        cleanup();
        return set_error(TBGPU_E_NUMERIC);
      }
    const auto k0 = std::chrono::steady_clock::now();
    const double tol_acc = accept_bound(p.at, Ta.data(), Tb.data());
    if (A.req1 > 0 && int(c1.size()) <= A.req1)
      check_window(p.at, Ta.data(), Tb.data(), A.emin1, A.emax1, tol_acc, res, c1, i1,
                   0x51ED27ULL * p.at + 1);
    if (A.req2 > 0 && int(c2.size()) <= A.req2)
      check_window(p.at, Ta.data(), Tb.data(), A.emin2, A.emax2, tol_acc, res, c2, i2,
                   0x51ED27ULL * p.at + 2);
    c.stats.check_ms +=
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - k0).count();
    const bool more = (p.at + 1 < A.imax) &&
                      (int(c1.size()) < A.req1 || int(c2.size()) < A.req2);
    if (!more) {
      final_it = p.at;
      hb_final = hb;
      break;
    }
    SOLVE_RC(fill());
  }
  for (auto &p : pend) cudaEventDestroy(p.ev);
  pend.clear();
  if (final_it < 0) {  // no check declared convergence: run to the iteration limit
    SOLVE_RC(enqueue_until(A.imax));
    final_it = launched;
  }
  }  // first pass
  SOLVE_CUDA(cudaEventRecord(tm.t1, s));
  SOLVE_CUDA(cudaStreamSynchronize(s));
  if (!restore && final_it == launched) {  // stopped by the iteration limit: T up to there
    SOLVE_CUDA(cudaMemcpy(h_alpha, d_alpha, sizeof(double) * final_it, cudaMemcpyDeviceToHost));
    SOLVE_CUDA(cudaMemcpy(h_bet, d_bet, sizeof(double) * (final_it + 1), cudaMemcpyDeviceToHost));
    Ta.assign(h_alpha, h_alpha + final_it);
    Tb.assign(h_bet + 1, h_bet + 1 + final_it);
    hb_final = h_bet;
  }
  c.alpha = Ta;
  c.beta = Tb;
  std::vector<std::pair<double, int>> found;
  for (size_t k = 0; k < c1.size(); k++) found.push_back({c1[k], i1[k]});
  for (size_t k = 0; k < c2.size(); k++) found.push_back({c2[k], i2[k]});
  std::stable_sort(found.begin(), found.end(),
                   [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
                     return x.first < y.first;
                   });
  const int ne = int(found.size());
  for (int k = 0; k < ne; k++) {
    values[k] = found[k].first;
    if (conv_iters) conv_iters[k] = found[k].second;
  }
  if (iterations) *iterations = final_it;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, tm.t0, tm.t1);
  c.stats.solve_ms = ms;
  c.stats.vectors_ms = 0.0;
  c.stats.lanczos_iterations = launched;

  // ---- second pass: eigenvectors -------------------------------------------
  const int nvec = std::min(ne, std::max(maxvec, 0));
  // the eigenvectors accumulate in the solver's layout (Vacc) and, in the
  // pencil layout, are permuted into V_dev at the end
  double *Vacc = V_dev;
  auto vec_target = [&]() -> int {
    if (pen) {
      if (solver_alloc(dev, &V_pen, ebytes * nvec, s) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
      Vacc = V_pen;
    }
    return cudaMemsetAsync(Vacc, 0, ebytes * nvec, s) == cudaSuccess ? TBGPU_OK
                                                                    : set_error(TBGPU_E_CUDA);
  };
  auto vec_out = [&]() -> int {
    if (!pen) return TBGPU_OK;
    for (int e = 0; e < nvec; e++) {
      int r_ = pen_permute<double2>(c, reinterpret_cast<const double2 *>(V_pen) + size_t(e) * n2,
                                    reinterpret_cast<double2 *>(V_dev) + size_t(e) * n2_ref,
                                    false, s);
      if (r_) return r_;
    }
    return TBGPU_OK;
  };
  std::vector<double> coef_all;
  if (!V_dev || nvec <= 0) drop_checkpoints();
  if (V_dev && nvec > 0) {
    // Ritz coefficients on the truncated tridiagonal of each eigenvalue
    int maxit = 0;
    for (int k = 0; k < nvec; k++) maxit = std::max(maxit, found[k].second);
    std::vector<double> &coef = coef_all;
    coef.assign(size_t(maxit) * nvec, 0.0);
    std::vector<double> x;
    for (int k = 0; k < nvec; k++) {
      const int req = found[k].second;
      if (!inverse_iteration(req, Ta.data(), Tb.data(), found[k].first, rng, x)) {
        cleanup();
        return set_error(TBGPU_E_NUMERIC);
      }
      // q_it = r_{it-1} / bet[it]; fold the 1/bet into the coefficient
      for (int it = 0; it < req; it++) coef[size_t(it) * nvec + k] = x[it] * (1.0 / hb_final[it]);
    }
    // bet of the first pass up to maxit is needed on the host
    if (maxit > final_it) maxit = final_it;
    const int nseg = (maxit + L - 1) / L;
    if (regen && int(ck_cur.size()) < nseg) regen = false;  // (cannot happen: maxit <= launched)
    c.stats.vec_segments = 0;
    c.stats.vec_mismatch = 0;
  }
  if (V_dev && nvec > 0 && regen) {
    // ---- eigenvector pass by regeneration: P segments at a time ------------
    int maxit = 0;
    for (int k = 0; k < nvec; k++) maxit = std::max(maxit, found[k].second);
    if (maxit > final_it) maxit = final_it;
    const int nseg = (maxit + L - 1) / L;
    const int K = kRegenRows / P;  // accumulation rows per column
    const int R = K + 2;           // ring per column: K inputs, the previous r, the output
    rr.assign(size_t(P) * R, nullptr);
    for (auto &q : rr) SOLVE_CUDA(solver_alloc(dev, &q, vbytes, s));
    SOLVE_CUDA(solver_alloc(dev, &d_diff, sizeof(unsigned long long) * std::max(nseg, 1), s));
    SOLVE_CUDA(cudaMemsetAsync(d_diff, 0, sizeof(unsigned long long) * std::max(nseg, 1), s));
    SOLVE_RC(vec_target());
    cudaEventRecord(tm.t2, s);
    std::vector<char> checked(nseg, 0);
    for (int g0 = 0; g0 < nseg; g0 += P) {
      const int ncol = std::min(P, nseg - g0);
      int len[4] = {0, 0, 0, 0}, steps = 0;
      for (int q = 0; q < ncol; q++) {
        const int seg = g0 + q;
        len[q] = std::min(L, maxit - seg * L);
        steps = std::max(steps, len[q]);
        SOLVE_CUDA(cudaMemcpyAsync(rr[q * R], ck_cur[seg], vbytes, cudaMemcpyDeviceToDevice, s));
        if (seg > 0)
          SOLVE_CUDA(cudaMemcpyAsync(rr[q * R + R - 1], ck_prev[seg], vbytes,
                                     cudaMemcpyDeviceToDevice, s));
      }
      int j0 = 0;
      for (int j = 0; j < steps; j++) {
        int na = 0;  // only the last segment can be short: the active columns are a prefix
        while (na < ncol && len[na] > j) na++;
        const VT *xs[4] = {nullptr, nullptr, nullptr, nullptr};
        const VT *rps[4] = {nullptr, nullptr, nullptr, nullptr};
        VT *ys[4] = {nullptr, nullptr, nullptr, nullptr};
        int its[4] = {0, 0, 0, 0};
        for (int q = 0; q < na; q++) {
          const int seg = g0 + q;
          xs[q] = rr[q * R + j % R];
          rps[q] = (seg == 0 && j == 0) ? nullptr : rr[q * R + (j + R - 1) % R];
          ys[q] = rr[q * R + (j + 1) % R];
          its[q] = seg * L + j;
        }
        SOLVE_RC(pen ? launch_pen_regen<VT>(c, na, xs, ys, rps, its, d_bet, d_alpha, s)
                     : launch_lane_regen<VT>(c, na, xs, ys, rps, its, d_bet, d_alpha, s));
        launches++;
        if (j + 1 - j0 == K || j == steps - 1) {  // accumulate the columns' inputs j0..j
          ChunkPtrs<VT, kRegenRows> Pr{};
          int rowit[kRegenRows];
          int nr = 0;
          for (int q = 0; q < ncol; q++)
            for (int jj = j0; jj <= j && jj < len[q]; jj++) {
              Pr.r[nr] = rr[q * R + jj % R];
              rowit[nr++] = (g0 + q) * L + jj;
            }
          for (int k = nr; k < kRegenRows; k++) Pr.r[k] = Pr.r[0];  // zero coefficients
          for (int g = 0; g < nvec; g += kRegenGroup) {
            const int nv = std::min(kRegenGroup, nvec - g);
            ChunkCoef<kRegenRows, kRegenGroup> Cf{};
            for (int k = 0; k < nr; k++)
              for (int e = 0; e < nv; e++) Cf.c[k][e] = coef_all[size_t(rowit[k]) * nvec + g + e];
            launch_accum<VT, kRegenRows, kRegenGroup>(
                nv, rg, s, n2, Pr, Cf, reinterpret_cast<double2 *>(Vacc) + size_t(g) * n2);
            launches++;
          }
          j0 = j + 1;
        }
      }
      // a full segment's last output is the next segment's first-pass start
      for (int q = 0; q < ncol; q++) {
        const int seg = g0 + q;
        if (len[q] == L && seg + 1 < int(ck_cur.size())) {
          k_count_diff<<<rg, kRedThreads, 0, s>>>(long(vbytes / 4),
                                                   reinterpret_cast<const unsigned *>(rr[q * R + L % R]),
                                                   reinterpret_cast<const unsigned *>(ck_cur[seg + 1]),
                                                   d_diff + seg);
          launches++;
          checked[seg] = 1;
        }
      }
    }
    cudaEventRecord(tm.t3, s);
    std::vector<unsigned long long> hd(std::max(nseg, 1), 0ull);
    SOLVE_CUDA(cudaMemcpyAsync(hd.data(), d_diff, sizeof(unsigned long long) * hd.size(),
                               cudaMemcpyDeviceToHost, s));
    SOLVE_CUDA(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&ms, tm.t2, tm.t3);
    c.stats.vectors_ms = ms;
    c.stats.vec_segments = nseg;
    for (int q = 0; q < nseg; q++) c.stats.vec_mismatch += checked[q] && hd[q] != 0;
    SOLVE_RC(vec_out());
    if (kMixed) {  // double-precision Rayleigh-Ritz of the Ritz vectors
      cudaEventRecord(tm.t2, s);
      c.state_resid.assign(nvec, 0.0);
      c.state_delta.assign(nvec, 0.0);
      const long off = 0;
      SOLVE_RC(refine_ritz(c, V_dev, nvec, n2_ref, 1, &off, &n2_ref, values, c.state_resid.data(),
                           c.state_delta.data(), s));
      cudaEventRecord(tm.t3, s);
      SOLVE_CUDA(cudaStreamSynchronize(s));
      cudaEventElapsedTime(&ms, tm.t2, tm.t3);
      c.stats.refine_ms = ms;
    }
  } else if (V_dev && nvec > 0) {
    // ---- eigenvector pass: the reference's second run ----------------------
    int maxit = 0;
    for (int k = 0; k < nvec; k++) maxit = std::max(maxit, found[k].second);
    if (maxit > final_it) maxit = final_it;
    const std::vector<double> &coef = coef_all;
    // chunk size limited by free memory
    size_t fre = 0, tot = 0;
    cudaMemGetInfo(&fre, &tot);
    fre += solver_pool_spare(dev);
    int K = kMaxChunk;
    while (K > 2 && size_t(K + 1 - S1) * vbytes + (256ull << 20) > fre) K /= 2;
    const int S2 = K + 1;
    for (int i = S1; i < S2; i++) SOLVE_CUDA(solver_alloc(dev, &ring[i], vbytes, s));
    SOLVE_RC(vec_target());
    cudaEventRecord(tm.t2, s);
    SOLVE_RC(start(d_bet));
    int it0 = 0;
    for (int it = 0; it < maxit; it++) {
      SOLVE_RC(step(it, S2, d_bet));
      if ((it + 1 - it0) == K || it == maxit - 1) {
        ChunkPtrs<VT> Pr{};
        const int nk = it + 1 - it0;
        for (int k = 0; k < kMaxChunk; k++)  // rows past nk: a valid vector, zero coefficients
          Pr.r[k] = ring[(it0 + (k < nk ? k : 0)) % S2];
        for (int g = 0; g < nvec; g += kVecGroup) {
          const int nv = std::min(kVecGroup, nvec - g);
          ChunkCoef<> Cf{};
          for (int k = 0; k < nk; k++)
            for (int e = 0; e < nv; e++) Cf.c[k][e] = coef[size_t(it0 + k) * nvec + g + e];
          launch_accum<VT>(nv, rg, s, n2, Pr, Cf, reinterpret_cast<double2 *>(Vacc) + size_t(g) * n2);
          launches++;
        }
        it0 = it + 1;
      }
    }
    cudaEventRecord(tm.t3, s);
    SOLVE_CUDA(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&ms, tm.t2, tm.t3);
    c.stats.vectors_ms = ms;
    SOLVE_RC(vec_out());
    if (kMixed) {  // double-precision Rayleigh-Ritz of the Ritz vectors
      cudaEventRecord(tm.t2, s);
      c.state_resid.assign(nvec, 0.0);
      c.state_delta.assign(nvec, 0.0);
      const long off = 0;
      SOLVE_RC(refine_ritz(c, V_dev, nvec, n2_ref, 1, &off, &n2_ref, values, c.state_resid.data(),
                           c.state_delta.data(), s));
      cudaEventRecord(tm.t3, s);
      SOLVE_CUDA(cudaStreamSynchronize(s));
      cudaEventElapsedTime(&ms, tm.t2, tm.t3);
      c.stats.refine_ms = ms;
    }
  }
  if (fold && V_dev && nvec > 0)  // the energies of the folded solve's eigenvectors
    SOLVE_RC(rayleigh_quotients(c, V_dev, nvec, c.fold_energy, s));
  if (c.profiling) {
    SOLVE_CUDA(cudaStreamSynchronize(s));
    double tot = 0.0;
    for (size_t k = 0; k + 1 < spmv_ev.size(); k += 2) {
      float t = 0.f;
      cudaEventElapsedTime(&t, spmv_ev[k], spmv_ev[k + 1]);
      tot += t;
    }
    c.stats.spmv_ms = tot;
    c.stats.spmv_launches = long(spmv_ev.size() / 2);
    double upd = 0.0;
    for (size_t k = 0; k < upd_ev.size() && 2 * k + 1 < spmv_ev.size(); k++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, spmv_ev[2 * k + 1], upd_ev[k]);
      upd += t;
    }
    c.stats.update_ms = upd;
  }
  c.stats.kernel_launches = launches;
  cudaEventDestroy(tm.t0);
  cudaEventDestroy(tm.t1);
  cudaEventDestroy(tm.t2);
  cudaEventDestroy(tm.t3);
  cleanup();
  // the solve returns with its work done (the buffers go back to the pool
  // in stream order)
  if (cudaStreamSynchronize(s) != cudaSuccess) return set_error(TBGPU_E_CUDA);
#undef SOLVE_CUDA
#undef SOLVE_RC
  return ne;
}

int solve(Ctx &c, const SolveArgs &A, const double *r0_dev, double *values, int *conv_iters,
          int *iterations, double *V_dev, int maxvec) {
  if (c.lanczos_f32)
    return solve_t<float2>(c, A, r0_dev, values, conv_iters, iterations, V_dev, maxvec);
  return solve_t<double2>(c, A, r0_dev, values, conv_iters, iterations, V_dev, maxvec);
}

}  // namespace tbgpu
