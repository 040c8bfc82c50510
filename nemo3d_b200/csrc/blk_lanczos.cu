// Block Lanczos eigenvalues on the GPU (eigensolve_blk_lanczos,
// NEMO_3D/eigen/src/lanczos_blk.c:2145-2540, with eigenvaluesBlockLanczos
// 1680-1760, block_lanczos_blocktridiagonal 1412-1678, single_iteration
// 392-550 and find_block_converged_eigvalues_Method4 553-634).
//
// One block step, p vectors at a time (Q: current block, Qold: previous
// block, R: residual block, all [p][n] complex in HBM):
//   [Q, B] = qr(R)            (not at the first step)
//   R_i    = H Q_i            (one multi-vector H*x launch, spmm_async.cu)
//   R     -= Qold B^H         (not at the first step)
//   A      = Q^H R            (Hermitian p x p; lower triangle computed)
//   R     -= Q A
// B and A fill the block-tridiagonal (band, kd = p) matrix whose window
// eigenvalues the host tracks between convergence checks (Method 4: values
// that agree with the previous check to `tolerance` count as converged).
// The QR is a Cholesky QR applied twice (Gram matrix on the GPU, 6x6
// factorisation on the host) instead of the reference's modified
// Gram-Schmidt: the same R factor, two passes over the block instead of
// p(p-1)/2.  Deflation of a (near) dependent block vector is not supported.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "tbgpu_internal.cuh"

namespace tbgpu {

using cplx = std::complex<double>;

namespace {

constexpr int kMaxP = 8;
constexpr int kDotThreads = 256;

struct BlockPtrs {
  const double2 *v[kMaxP];
};
struct BlockOut {
  double2 *v[kMaxP];
};
struct SmallMat {  // m[k][i], column i of the combination for output vector i
  double2 m[kMaxP][kMaxP];
};

// G[i][j] = sum conj(X_i) Y_j over the lower triangle i >= j (P(P+1)/2
// complex dots, each vector read once); per-block partials are summed in
// block order by the last block to finish (deterministic).
template <int P>
__global__ void __launch_bounds__(kDotThreads)
    k_bdots(long n2, BlockPtrs X, BlockPtrs Y, double *partial, unsigned *counter, double *out) {
  constexpr int K = P * (P + 1) / 2;
  double acc[2 * K];
#pragma unroll
  for (int t = 0; t < 2 * K; t++) acc[t] = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    double2 x[P], y[P];
#pragma unroll
    for (int i = 0; i < P; i++) {
      x[i] = __ldg(X.v[i] + j);
      y[i] = __ldg(Y.v[i] + j);
    }
    int t = 0;
#pragma unroll
    for (int i = 0; i < P; i++)
#pragma unroll
      for (int jj = 0; jj <= i; jj++, t++) {
        acc[2 * t] += x[i].x * y[jj].x + x[i].y * y[jj].y;
        acc[2 * t + 1] += x[i].x * y[jj].y - x[i].y * y[jj].x;
      }
  }
  __shared__ double red[kDotThreads / 32][2 * K];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 2 * K; t++) {
    double v = acc[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][t] = v;
  }
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x < 2 * K) {
    double v = 0.0;
    for (int ww = 0; ww < kDotThreads / 32; ww++) v += red[ww][threadIdx.x];
    partial[size_t(blockIdx.x) * 2 * K + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x < 2 * K) {
      double v = 0.0;
      for (unsigned b = 0; b < gridDim.x; b++)
        v += static_cast<volatile double *>(partial)[size_t(b) * 2 * K + threadIdx.x];
      out[threadIdx.x] = v;
    }
    if (threadIdx.x == 0) *counter = 0;
  }
}

// Y_i = zs * Z_i + sum_k X_k M[k][i] for i < ny, k < nx (Z may alias Y)
template <int P>
__global__ void __launch_bounds__(256)
    k_bcombine(long n2, int nx, BlockPtrs X, SmallMat M, int ny, BlockOut Y, double zs,
               BlockPtrs Z) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n2;
       j += (long)gridDim.x * blockDim.x) {
    double2 x[P];
#pragma unroll
    for (int k = 0; k < P; k++)
      if (k < nx) x[k] = __ldg(X.v[k] + j);
#pragma unroll
    for (int i = 0; i < P; i++) {
      if (i >= ny) break;
      double2 acc = make_double2(0.0, 0.0);
      if (zs != 0.0) {
        const double2 z = Z.v[i][j];
        acc = make_double2(zs * z.x, zs * z.y);
      }
#pragma unroll
      for (int k = 0; k < P; k++)
        if (k < nx) {
          const double2 m = M.m[k][i];
          acc.x += m.x * x[k].x - m.y * x[k].y;
          acc.y += m.x * x[k].y + m.y * x[k].x;
        }
      Y.v[i][j] = acc;
    }
  }
}

// ---- host linear algebra on p x p blocks ----------------------------------
using Mat = std::vector<cplx>;  // row-major p x p

// G = U^H U with U upper triangular, positive diagonal; false if G is not
// numerically positive definite (a dependent block vector)
bool cholesky_upper(int p, const Mat &G, Mat &U) {
  U.assign(size_t(p) * p, cplx(0.0, 0.0));
  for (int j = 0; j < p; j++) {
    double d = G[j * p + j].real();
    for (int k = 0; k < j; k++) d -= std::norm(U[k * p + j]);
    if (!(d > 0.0)) return false;
    const double ujj = std::sqrt(d);
    U[j * p + j] = ujj;
    for (int i = j + 1; i < p; i++) {
      cplx s = G[j * p + i];
      for (int k = 0; k < j; k++) s -= std::conj(U[k * p + j]) * U[k * p + i];
      U[j * p + i] = s / ujj;
    }
  }
  return true;
}

Mat upper_inverse(int p, const Mat &U) {
  Mat V(size_t(p) * p, cplx(0.0, 0.0));
  for (int j = 0; j < p; j++) {
    V[j * p + j] = 1.0 / U[j * p + j];
    for (int i = j - 1; i >= 0; i--) {
      cplx s(0.0, 0.0);
      for (int k = i + 1; k <= j; k++) s += U[i * p + k] * V[k * p + j];
      V[i * p + j] = -s / U[i * p + i];
    }
  }
  return V;
}

Mat matmul(int p, const Mat &A, const Mat &B) {
  Mat C(size_t(p) * p, cplx(0.0, 0.0));
  for (int i = 0; i < p; i++)
    for (int k = 0; k < p; k++)
      for (int j = 0; j < p; j++) C[i * p + j] += A[i * p + k] * B[k * p + j];
  return C;
}

// Method 4 of the reference (lanczos_blk.c:553-634)
void method4(const std::vector<double> &fresh, std::vector<double> &old, std::vector<double> &conv,
             int requested, int &n_nosuccess, double tolerance) {
  const double resolution = 100.0 * tolerance;
  std::vector<double> tmp;
  std::vector<double> olds = old;
  for (double v : fresh) {
    for (double &o : olds)
      if (std::fabs(v - o) < tolerance) {
        tmp.push_back(v);
        o = 500.0;
        break;
      }
    if (int(tmp.size()) == requested) break;
  }
  for (double &cv : conv)
    for (double &t : tmp)
      if (std::fabs(cv - t) < resolution) {
        cv = t;
        t = 500.0;
        break;
      }
  for (double t : tmp)
    if (std::fabs(t) < 490.0) {
      conv.push_back(t);
      n_nosuccess = 0;
      if (int(conv.size()) == requested) break;
    }
  old = fresh;
}

}  // namespace

struct BlkArgs {
  int start, skip, imax, req1, req2, p, max_no_success;
  double emin1, emax1, emin2, emax2, tol;
};

template <int P>
static int blk_run(Ctx &c, const BlkArgs &A, const double *r0_dev, std::vector<double> &values,
                   int &found1_out, int &found2_out, int &iters_out) {
  const long n2 = c.natoms * c.nb;
  const size_t vbytes = sizeof(double2) * n2;
  cudaStream_t s = c.stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  const unsigned grid = unsigned(std::max<long>(1, std::min<long>((n2 + 255) / 256, long(sms) * 8)));
  constexpr int K = P * (P + 1) / 2;
  double2 *Q = nullptr, *Qo = nullptr, *R = nullptr;
  double *partial = nullptr, *dres = nullptr;
  unsigned *counter = nullptr;
  int rc = TBGPU_OK;
  auto fail = [&](int code) {
    rc = code;
    return code;
  };
  if (cudaMalloc(&Q, vbytes * P) != cudaSuccess || cudaMalloc(&Qo, vbytes * P) != cudaSuccess ||
      cudaMalloc(&R, vbytes * P) != cudaSuccess ||
      cudaMalloc(&partial, sizeof(double) * 2 * K * grid) != cudaSuccess ||
      cudaMalloc(&dres, sizeof(double) * 2 * K) != cudaSuccess ||
      cudaMalloc(&counter, sizeof(unsigned)) != cudaSuccess) {
    cudaFree(Q); cudaFree(Qo); cudaFree(R); cudaFree(partial); cudaFree(dres); cudaFree(counter);
    return set_error(TBGPU_E_NOMEM);
  }
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned), s) != cudaSuccess) rc = TBGPU_E_CUDA;
  auto ptrs = [&](double2 *base) {
    BlockPtrs b{};
    for (int i = 0; i < P; i++) b.v[i] = base + size_t(i) * n2;
    return b;
  };
  auto outs = [&](double2 *base) {
    BlockOut b{};
    for (int i = 0; i < P; i++) b.v[i] = base + size_t(i) * n2;
    return b;
  };
  // lower-triangle dots -> full Hermitian p x p matrix G[i][j] = X_i^H Y_j
  auto dots = [&](double2 *X, double2 *Y, Mat &G) -> int {
    k_bdots<P><<<grid, kDotThreads, 0, s>>>(n2, ptrs(X), ptrs(Y), partial, counter, dres);
    if (cudaGetLastError() != cudaSuccess) return fail(TBGPU_E_CUDA);
    double h[2 * K];
    if (cudaMemcpyAsync(h, dres, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return fail(TBGPU_E_CUDA);
    G.assign(size_t(P) * P, cplx(0.0, 0.0));
    int t = 0;
    for (int i = 0; i < P; i++)
      for (int j = 0; j <= i; j++, t++) {
        G[i * P + j] = cplx(h[2 * t], h[2 * t + 1]);
        G[j * P + i] = std::conj(G[i * P + j]);
      }
    for (int i = 0; i < P; i++) G[i * P + i] = cplx(G[i * P + i].real(), 0.0);
    return TBGPU_OK;
  };
  // Y = zs*Z + X M   (M[k][i] multiplies X_k into Y_i)
  auto combine = [&](double2 *X, const Mat &M, double2 *Y, double zs, double2 *Z) -> int {
    SmallMat sm{};
    for (int k = 0; k < P; k++)
      for (int i = 0; i < P; i++) sm.m[k][i] = make_double2(M[k * P + i].real(), M[k * P + i].imag());
    k_bcombine<P><<<grid, 256, 0, s>>>(n2, P, ptrs(X), sm, P, outs(Y), zs, ptrs(Z ? Z : Y));
    return cudaGetLastError() == cudaSuccess ? TBGPU_OK : fail(TBGPU_E_CUDA);
  };
  // [Q, B] = qr(R), Cholesky QR twice; B upper triangular
  auto qr = [&](Mat &B) -> int {
    Mat G, U, U2;
    if (dots(R, R, G)) return rc;
    if (!cholesky_upper(P, G, U)) return fail(TBGPU_E_NUMERIC);
    if (combine(R, upper_inverse(P, U), Q, 0.0, nullptr)) return rc;
    if (dots(Q, Q, G)) return rc;
    if (!cholesky_upper(P, G, U2)) return fail(TBGPU_E_NUMERIC);
    // Q = Q U2^{-1} in place: write through R as scratch, then swap roles
    if (combine(Q, upper_inverse(P, U2), R, 0.0, nullptr)) return rc;
    std::swap(Q, R);
    B = matmul(P, U2, U);
    return TBGPU_OK;
  };

  // band (block tridiagonal) matrix, lower storage, kd = P
  const int ld = P + 1;
  std::vector<cplx> band;
  int tsize = 0;
  std::vector<double> old1, old2, conv1, conv2;
  int nos1 = 0, nos2 = 0, skip = 0, it = 0;
  const int added = 1;
  // start block: R = r0, Q = qr(R)
  if (cudaMemcpyAsync(R, r0_dev, vbytes * P, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    rc = TBGPU_E_CUDA;
  Mat B;
  if (!rc) qr(B);
  bool converged = false;
  while (!rc) {
    if (it != 0 && qr(B)) break;
    // R_i = H Q_i, the block at once
    if (launch_spmm(c, P, reinterpret_cast<const double *>(Q), 2 * n2,
                    reinterpret_cast<double *>(R), 2 * n2, 0.0, s))
      rc = TBGPU_E_CUDA;
    if (rc) break;
    if (it != 0) {  // R -= Qold B^H
      Mat M(size_t(P) * P);
      for (int k = 0; k < P; k++)
        for (int i = 0; i < P; i++) M[k * P + i] = -std::conj(B[i * P + k]);
      if (combine(Qo, M, R, 1.0, R)) break;
    }
    Mat Al;
    if (dots(Q, R, Al)) break;  // Al[i][j] = Q_i^H R_j
    {                           // R -= Q A, A[k][i] = Q_k^H R_i
      Mat M(size_t(P) * P);
      for (int k = 0; k < P; k++)
        for (int i = 0; i < P; i++) M[k * P + i] = -Al[k * P + i];
      if (combine(Q, M, R, 1.0, R)) break;
    }
    std::swap(Q, Qo);
    // band entries of this block: B couples it to the previous block
    band.resize(size_t(tsize + P) * ld, cplx(0.0, 0.0));
    if (it != 0)
      for (int j = 0; j < P; j++)
        for (int i = 0; i <= j; i++)  // T(tsize + i, tsize - P + j) = B[i][j]
          band[size_t(tsize - P + j) * ld + (P + i - j)] = B[i * P + j];
    for (int j = 0; j < P; j++)
      for (int i = j; i < P; i++) band[size_t(tsize + j) * ld + (i - j)] = Al[i * P + j];
    tsize += P;
    ++skip;
    if (A.start < it) {
      if (int(conv1.size()) < A.req1) nos1++;
      if (int(conv2.size()) < A.req2) nos2++;
    }
    if (A.start < it && A.skip <= skip) {
      skip = 0;
      std::vector<double> w;
      if (A.req1 > 0 && int(conv1.size()) < A.req1) {
        band_eigenvalues(tsize, P, band.data(), A.emin1, A.emax1, A.tol, w);
        // the highest requested+1 values of the window, top down
        std::vector<double> fresh;
        const int m = int(w.size()), take = std::min(A.req1 + added, m);
        for (int i = 0; i < take; i++) fresh.push_back(w[m - 1 - i]);
        method4(fresh, old1, conv1, A.req1, nos1, A.tol);
      }
      if (A.req2 > 0 && int(conv2.size()) < A.req2) {
        band_eigenvalues(tsize, P, band.data(), A.emin2, A.emax2, A.tol, w);
        std::vector<double> fresh;
        const int m = int(w.size()), take = std::min(A.req2 + added, m);
        for (int i = 0; i < take; i++) fresh.push_back(w[i]);
        method4(fresh, old2, conv2, A.req2, nos2, A.tol);
      }
    }
    const bool done = (int(conv1.size()) >= A.req1 && int(conv2.size()) >= A.req2) ||
                      it + 2 == A.imax;
    const bool stalled = nos1 >= A.max_no_success || nos2 >= A.max_no_success;
    ++it;
    if (done || stalled) {
      converged = true;
      break;
    }
    if (it + 1 >= A.imax) break;
  }
  (void)converged;
  cudaStreamSynchronize(s);
  cudaFree(Q); cudaFree(Qo); cudaFree(R); cudaFree(partial); cudaFree(dres); cudaFree(counter);
  if (rc) return set_error(rc);
  values.assign(conv1.begin(), conv1.end());
  values.insert(values.end(), conv2.begin(), conv2.end());
  std::sort(values.begin(), values.end());
  found1_out = int(conv1.size());
  found2_out = int(conv2.size());
  iters_out = it;
  return TBGPU_OK;
}

int solve_block(Ctx &c, const BlkArgs &A, const double *r0_dev, std::vector<double> &values,
                int &f1, int &f2, int &iters) {
  switch (A.p) {
    case 1: return blk_run<1>(c, A, r0_dev, values, f1, f2, iters);
    case 2: return blk_run<2>(c, A, r0_dev, values, f1, f2, iters);
    case 3: return blk_run<3>(c, A, r0_dev, values, f1, f2, iters);
    case 4: return blk_run<4>(c, A, r0_dev, values, f1, f2, iters);
    case 5: return blk_run<5>(c, A, r0_dev, values, f1, f2, iters);
    case 6: return blk_run<6>(c, A, r0_dev, values, f1, f2, iters);
    case 7: return blk_run<7>(c, A, r0_dev, values, f1, f2, iters);
    case 8: return blk_run<8>(c, A, r0_dev, values, f1, f2, iters);
    default: return set_error(TBGPU_E_ARG);
  }
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_eigensolve_blk_lanczos_dev(
    tbgpu_ctx *ctx, int ConvCheckStartIter, int ConvCheckSkipRate, int imax, int requested1,
    int requested2, double emin1, double emax1, double emin2, double emax2, double tolerance,
    int p, int max_no_success, const double *r0_dev, double *values, int *found_vb,
    int *found_cb, int *iterations) {
  if (!ctx || !r0_dev || !values || p < 1 || p > kMaxP || imax < 2 || ConvCheckSkipRate < 1 ||
      requested1 < 0 || requested2 < 0 || tolerance <= 0.0)
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  set_error(TBGPU_OK);
  BlkArgs A{ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2, p,
            max_no_success > 0 ? max_no_success : 1 << 30,
            emin1, emax1, emin2, emax2, tolerance};
  std::vector<double> vals;
  int f1 = 0, f2 = 0, it = 0;
  int rc = solve_block(c, A, r0_dev, vals, f1, f2, it);
  if (rc) return rc;
  for (size_t k = 0; k < vals.size(); k++) values[k] = vals[k];
  if (found_vb) *found_vb = f1;
  if (found_cb) *found_cb = f2;
  if (iterations) *iterations = it;
  return int(vals.size());
}

extern "C" int tbgpu_eigensolve_blk_lanczos(
    tbgpu_ctx *ctx, int ConvCheckStartIter, int ConvCheckSkipRate, int imax, int requested1,
    int requested2, double emin1, double emax1, double emin2, double emax2, double tolerance,
    int p, int max_no_success, const tbgpu_dcomplex *r0, double *values, int *found_vb,
    int *found_cb, int *iterations) {
  if (!ctx || !r0 || p < 1 || p > kMaxP) return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t bytes = sizeof(double2) * size_t(c.natoms) * c.nb * p;
  double *d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  int rc = TBGPU_OK;
  if (cudaMemcpyAsync(d, r0, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
    rc = set_error(TBGPU_E_CUDA);
  if (!rc)
    rc = tbgpu_eigensolve_blk_lanczos_dev(ctx, ConvCheckStartIter, ConvCheckSkipRate, imax,
                                          requested1, requested2, emin1, emax1, emin2, emax2,
                                          tolerance, p, max_no_success, d, values, found_vb,
                                          found_cb, iterations);
  cudaStreamSynchronize(c.stream);
  cudaFree(d);
  return rc;
}
