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

// Eigenvector y of the Hermitian band matrix T (lower storage, kd) for the
// eigenvalue lam by inverse iteration with a banded LU of T - lam I (partial
// pivoting; U has 2 kd superdiagonals), orthogonalised in every step against
// the vectors in `ortho` (the earlier members of a cluster of equal values)
// so that degenerate eigenvalues get independent vectors.
bool band_eigvec(int n, int kd, const std::vector<cplx> &ab, double lam,
                 const std::vector<std::vector<cplx>> &ortho, unsigned long long seed,
                 std::vector<cplx> &y) {
  const int ld = kd + 1, w = 3 * kd + 1, off = 2 * kd;  // row i: columns i-kd .. i+2kd
  std::vector<cplx> M(size_t(n) * w, cplx(0.0, 0.0));
  auto at = [&](int i, int j) -> cplx & { return M[size_t(i) * w + (j - i + kd)]; };
  double norm = 0.0;
  for (int j = 0; j < n; j++)
    for (int i = j; i <= std::min(n - 1, j + kd); i++) {
      const cplx v = ab[size_t(j) * ld + (i - j)];
      at(i, j) = v;
      if (i != j) at(j, i) = std::conj(v);
      norm = std::max(norm, std::abs(v));
    }
  for (int i = 0; i < n; i++) at(i, i) -= lam;
  const double tiny = std::max(norm, 1.0) * 1e-14;
  std::vector<int> piv(n);
  for (int j = 0; j < n; j++) {  // LU with row pivoting inside the band
    int pr = j;
    double best = std::abs(at(j, j));
    for (int i = j + 1; i <= std::min(n - 1, j + kd); i++)
      if (std::abs(at(i, j)) > best) { best = std::abs(at(i, j)); pr = i; }
    piv[j] = pr;
    const int hi = std::min(n - 1, j + off);
    if (pr != j)
      for (int c = j; c <= hi; c++) std::swap(at(j, c), at(pr, c));
    if (std::abs(at(j, j)) < tiny) at(j, j) = tiny;  // exact eigenvalue: perturb the pivot
    for (int i = j + 1; i <= std::min(n - 1, j + kd); i++) {
      const cplx l = at(i, j) / at(j, j);
      at(i, j) = l;
      if (l == cplx(0.0, 0.0)) continue;
      for (int c = j + 1; c <= hi; c++) at(i, c) -= l * at(j, c);
    }
  }
  unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto urand = [&]() {
    st = st * 6364136223846793005ULL + 1442695040888963407ULL;
    return double(st >> 11) / double(1ULL << 53) - 0.5;
  };
  y.assign(n, cplx(0.0, 0.0));
  for (int i = 0; i < n; i++) y[i] = cplx(urand(), urand());
  auto orth_norm = [&]() -> bool {
    for (const auto &u : ortho) {
      cplx d(0.0, 0.0);
      for (int i = 0; i < n; i++) d += std::conj(u[i]) * y[i];
      for (int i = 0; i < n; i++) y[i] -= d * u[i];
    }
    double nn = 0.0;
    for (int i = 0; i < n; i++) nn += std::norm(y[i]);
    if (!(nn > 0.0)) return false;
    nn = 1.0 / std::sqrt(nn);
    for (int i = 0; i < n; i++) y[i] *= nn;
    return true;
  };
  if (!orth_norm()) return false;
  for (int itr = 0; itr < 4; itr++) {
    for (int j = 0; j < n; j++) {  // forward: apply the row swaps and L
      if (piv[j] != j) std::swap(y[j], y[piv[j]]);
      for (int i = j + 1; i <= std::min(n - 1, j + kd); i++) y[i] -= at(i, j) * y[j];
    }
    for (int i = n - 1; i >= 0; i--) {  // back: U
      cplx v = y[i];
      for (int c = i + 1; c <= std::min(n - 1, i + off); c++) v -= at(i, c) * y[c];
      y[i] = v / at(i, i);
    }
    if (!orth_norm()) return false;
  }
  return true;
}

// Eigenpairs of a small Hermitian m x m matrix G (row-major), largest first:
// cyclic Jacobi on the real symmetric embedding [[Re, -Im], [Im, Re]], whose
// eigenvalues are those of G twice over; one complex vector is kept per pair.
void herm_eig_desc(int m, const Mat &G, std::vector<double> &w, std::vector<std::vector<cplx>> &U) {
  const int n = 2 * m;
  std::vector<double> A(size_t(n) * n), V(size_t(n) * n, 0.0);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++) {
      const cplx g = G[i * m + j];
      A[i * n + j] = g.real();
      A[(i + m) * n + (j + m)] = g.real();
      A[i * n + (j + m)] = -g.imag();
      A[(i + m) * n + j] = g.imag();
    }
  for (int i = 0; i < n; i++) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) off += A[i * n + j] * A[i * n + j];
    if (off < 1e-30) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = A[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double th = 0.5 * (A[q * n + q] - A[p * n + p]) / apq;
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; k++) {  // A <- J^T A J, V <- V J
          const double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - sn * akq;
          A[k * n + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          const double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - sn * aqk;
          A[q * n + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - sn * vkq;
          V[k * n + q] = sn * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; i++) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return A[a * n + a] > A[b * n + b]; });
  w.clear();
  U.clear();
  for (int idx : ord) {
    std::vector<cplx> z(m);
    for (int i = 0; i < m; i++) z[i] = cplx(V[i * n + idx], V[(i + m) * n + idx]);
    for (const auto &u : U) {
      cplx d(0.0, 0.0);
      for (int i = 0; i < m; i++) d += std::conj(u[i]) * z[i];
      for (int i = 0; i < m; i++) z[i] -= d * u[i];
    }
    double nn = 0.0;
    for (int i = 0; i < m; i++) nn += std::norm(z[i]);
    if (nn < 0.25) continue;  // the partner of a vector already kept
    nn = 1.0 / std::sqrt(nn);
    for (int i = 0; i < m; i++) z[i] *= nn;
    U.push_back(z);
    w.push_back(A[idx * n + idx]);
    if (int(U.size()) == m) break;
  }
}

}  // namespace

struct BlkArgs {
  int start, skip, imax, req1, req2, p, max_no_success;
  double emin1, emax1, emin2, emax2, tol;
};

template <int P>
static int blk_run(Ctx &c, const BlkArgs &A, const double *r0_dev, std::vector<double> &values,
                   int &found1_out, int &found2_out, int &iters_out, double *V_dev,
                   int maxvec) {
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
  // the tensor-core dots keep 256 partial sums per CTA and the full 8 x 8
  // product
  const bool tc = c.block_dots == 1;
  const int tc_grid = tc ? bdots_tc_grid(c, n2) : 0;
  double *tc_part = nullptr, *tc_out = nullptr;
  if (tc && (cudaMalloc(&tc_part, sizeof(double) * 256 * size_t(tc_grid)) != cudaSuccess ||
             cudaMalloc(&tc_out, sizeof(double) * 2 * kMaxP * kMaxP) != cudaSuccess)) {
    cudaFree(tc_part); cudaFree(tc_out);
    cudaFree(Q); cudaFree(Qo); cudaFree(R); cudaFree(partial); cudaFree(dres); cudaFree(counter);
    return set_error(TBGPU_E_NOMEM);
  }
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
    G.assign(size_t(P) * P, cplx(0.0, 0.0));
    if (tc) {
      const double2 *xp[P], *yp[P];
      for (int i = 0; i < P; i++) {
        xp[i] = X + size_t(i) * n2;
        yp[i] = Y + size_t(i) * n2;
      }
      if (launch_bdots_tc(c, P, xp, yp, n2, tc_part, counter, tc_grid, tc_out, s))
        return fail(TBGPU_E_CUDA);
      double h[2 * kMaxP * kMaxP];
      if (cudaMemcpyAsync(h, tc_out, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return fail(TBGPU_E_CUDA);
      if (int st = take_status(c)) return fail(st);
      // the lower triangle, as the CUDA-core kernel forms it
      for (int i = 0; i < P; i++)
        for (int j = 0; j <= i; j++) {
          G[i * P + j] = cplx(h[2 * (i * kMaxP + j)], h[2 * (i * kMaxP + j) + 1]);
          G[j * P + i] = std::conj(G[i * P + j]);
        }
    } else {
      k_bdots<P><<<grid, kDotThreads, 0, s>>>(n2, ptrs(X), ptrs(Y), partial, counter, dres);
      if (cudaGetLastError() != cudaSuccess) return fail(TBGPU_E_CUDA);
      double h[2 * K];
      if (cudaMemcpyAsync(h, dres, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return fail(TBGPU_E_CUDA);
      int t = 0;
      for (int i = 0; i < P; i++)
        for (int j = 0; j <= i; j++, t++) {
          G[i * P + j] = cplx(h[2 * t], h[2 * t + 1]);
          G[j * P + i] = std::conj(G[i * P + j]);
        }
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
  // one block step (single_iteration); the current block ends up in Qo
  auto step = [&](Mat &B, Mat &Al) -> int {
    if (it != 0 && qr(B)) return rc;
    // R_i = H Q_i, the block at once
    if (launch_spmm(c, P, reinterpret_cast<const double *>(Q), 2 * n2,
                    reinterpret_cast<double *>(R), 2 * n2, 0.0, s))
      return fail(TBGPU_E_CUDA);
    if (it != 0) {  // R -= Qold B^H
      Mat M(size_t(P) * P);
      for (int k = 0; k < P; k++)
        for (int i = 0; i < P; i++) M[k * P + i] = -std::conj(B[i * P + k]);
      if (combine(Qo, M, R, 1.0, R)) return rc;
    }
    if (dots(Q, R, Al)) return rc;  // Al[i][j] = Q_i^H R_j
    {                               // R -= Q A, A[k][i] = Q_k^H R_i
      Mat M(size_t(P) * P);
      for (int k = 0; k < P; k++)
        for (int i = 0; i < P; i++) M[k * P + i] = -Al[k * P + i];
      if (combine(Q, M, R, 1.0, R)) return rc;
    }
    std::swap(Q, Qo);
    return TBGPU_OK;
  };
  // start block: R = r0, Q = qr(R)
  auto restart = [&]() -> int {
    if (cudaMemcpyAsync(R, r0_dev, vbytes * P, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return fail(TBGPU_E_CUDA);
    Mat B0;
    return qr(B0);
  };
  Mat B, Al;
  if (!rc) restart();
  bool converged = false;
  while (!rc) {
    if (step(B, Al)) break;
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
  values.assign(conv1.begin(), conv1.end());
  values.insert(values.end(), conv2.begin(), conv2.end());
  std::sort(values.begin(), values.end());
  const int it0_steps = it;
  // ---- eigenvectors: Ritz vectors of the band matrix, second pass ---------
  // (eigenvectorsBlockLanczos, lanczos_blk.c:1857-2145: the recurrence is
  // repeated from the start block, which the deterministic kernels reproduce
  // bit for bit, and every block is accumulated with its rows of the band
  // matrix's eigenvectors)
  const int nvec = V_dev ? std::min(int(values.size()), std::max(maxvec, 0)) : 0;
  double2 *Cand = nullptr;
  if (!rc && nvec > 0) {
    // Clusters of equal values (within 100x the tolerance, e.g. Kramers
    // pairs).  Without reorthogonalisation the band matrix also carries
    // copies ("ghosts") of converged values whose Ritz vectors repeat true
    // ones, so every band eigenvector of a cluster's window is rebuilt and
    // the cluster's vectors are the orthonormal directions of largest
    // weight among those candidates (the reference instead Gram-Schmidts
    // the rebuilt vectors of close values, lanczos_blk.c:2117-2128).
    struct Cluster {
      int e0, r;                 // first value index, members
      std::vector<std::vector<cplx>> y;  // band eigenvectors (candidates)
      int c0;                    // first candidate index
    };
    std::vector<Cluster> cl;
    for (int e = 0; e < nvec;) {
      int f = e + 1;
      while (f < nvec && values[f] - values[f - 1] < 100.0 * A.tol) f++;
      cl.push_back({e, f - e, {}, 0});
      e = f;
    }
    int ncand = 0;
    for (auto &C : cl) {
      const double lo = values[C.e0] - 100.0 * A.tol, hi = values[C.e0 + C.r - 1] + 100.0 * A.tol;
      std::vector<double> wv;
      band_eigenvalues(tsize, P, band.data(), lo, hi, A.tol, wv);
      if (int(wv.size()) < C.r) wv.assign(values.begin() + C.e0, values.begin() + C.e0 + C.r);
      if (wv.size() > 8) wv.resize(8);
      for (size_t k = 0; k < wv.size() && !rc; k++) {
        std::vector<cplx> y;
        if (!band_eigvec(tsize, P, band, wv[k], C.y, 977ULL + 31ULL * ncand + k, y))
          rc = TBGPU_E_NUMERIC;
        else
          C.y.push_back(y);
      }
      C.c0 = ncand;
      ncand += int(C.y.size());
    }
    if (!rc && cudaMalloc(&Cand, vbytes * ncand) != cudaSuccess) rc = TBGPU_E_NOMEM;
    if (!rc && cudaMemsetAsync(Cand, 0, vbytes * ncand, s) != cudaSuccess) rc = TBGPU_E_CUDA;
    std::vector<const std::vector<cplx> *> Y;
    for (auto &C : cl)
      for (auto &y : C.y) Y.push_back(&y);
    if (!rc) {
      it = 0;
      restart();
    }
    const int nsteps = it0_steps;
    for (int k = 0; k < nsteps && !rc; k++) {
      if (step(B, Al)) break;
      ++it;
      // Cand_j += sum_i Qo_i * Y_j[k*P + i], in groups of up to P candidates
      for (int e0 = 0; e0 < ncand && !rc; e0 += P) {
        const int ne = std::min(P, ncand - e0);
        SmallMat sm{};
        for (int i = 0; i < P; i++)
          for (int e = 0; e < ne; e++) {
            const cplx v = (*Y[e0 + e])[size_t(k) * P + i];
            sm.m[i][e] = make_double2(v.real(), v.imag());
          }
        BlockOut vo{};
        BlockPtrs vi{};
        for (int e = 0; e < ne; e++) {
          vo.v[e] = Cand + size_t(e0 + e) * n2;
          vi.v[e] = Cand + size_t(e0 + e) * n2;
        }
        k_bcombine<P><<<grid, 256, 0, s>>>(n2, P, ptrs(Qo), sm, ne, vo, 1.0, vi);
        if (cudaGetLastError() != cudaSuccess) rc = TBGPU_E_CUDA;
      }
    }
    // each cluster: Gram matrix of its candidates, keep the r directions of
    // largest weight, orthonormal, as the cluster's eigenvectors
    for (auto &C : cl) {
      if (rc) break;
      const int m = int(C.y.size());
      BlockPtrs cp{};
      for (int j = 0; j < 8; j++) cp.v[j] = Cand + size_t(C.c0 + std::min(j, m - 1)) * n2;
      constexpr int K8 = 8 * 9 / 2;
      double *part8 = nullptr, *res8 = nullptr;
      if (cudaMalloc(&part8, sizeof(double) * 2 * K8 * grid) != cudaSuccess ||
          cudaMalloc(&res8, sizeof(double) * 2 * K8) != cudaSuccess) {
        cudaFree(part8);
        rc = TBGPU_E_NOMEM;
        break;
      }
      k_bdots<8><<<grid, kDotThreads, 0, s>>>(n2, cp, cp, part8, counter, res8);
      double h[2 * K8];
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(h, res8, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        rc = TBGPU_E_CUDA;
      cudaFree(part8);
      cudaFree(res8);
      if (rc) break;
      Mat G(size_t(m) * m);
      int t = 0;
      for (int i = 0; i < 8; i++)
        for (int j = 0; j <= i; j++, t++)
          if (i < m && j < m) {
            G[i * m + j] = cplx(h[2 * t], h[2 * t + 1]);
            G[j * m + i] = std::conj(G[i * m + j]);
          }
      std::vector<double> gw;
      std::vector<std::vector<cplx>> gu;
      herm_eig_desc(m, G, gw, gu);
      const int keep = std::min(C.r, int(gu.size()));
      if (keep < C.r || gw[keep - 1] <= 0.0) {
        rc = TBGPU_E_NUMERIC;
        break;
      }
      SmallMat sm{};
      for (int j = 0; j < m; j++)
        for (int e = 0; e < keep; e++) {
          const cplx v = gu[e][j] / std::sqrt(gw[e]);
          sm.m[j][e] = make_double2(v.real(), v.imag());
        }
      BlockOut vo{};
      for (int e = 0; e < keep; e++)
        vo.v[e] = reinterpret_cast<double2 *>(V_dev) + size_t(C.e0 + e) * n2;
      k_bcombine<8><<<grid, 256, 0, s>>>(n2, m, cp, sm, keep, vo, 0.0, cp);
      if (cudaGetLastError() != cudaSuccess) rc = TBGPU_E_CUDA;
    }
    it = nsteps;
  }
  cudaFree(Cand);
  (void)converged;
  cudaStreamSynchronize(s);
  cudaFree(tc_part); cudaFree(tc_out);
  cudaFree(Q); cudaFree(Qo); cudaFree(R); cudaFree(partial); cudaFree(dres); cudaFree(counter);
  if (rc) return set_error(rc);
  found1_out = int(conv1.size());
  found2_out = int(conv2.size());
  iters_out = it;
  return TBGPU_OK;
}

int solve_block(Ctx &c, const BlkArgs &A, const double *r0_dev, std::vector<double> &values,
                int &f1, int &f2, int &iters, double *V_dev, int maxvec) {
  switch (A.p) {
    case 1: return blk_run<1>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 2: return blk_run<2>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 3: return blk_run<3>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 4: return blk_run<4>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 5: return blk_run<5>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 6: return blk_run<6>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 7: return blk_run<7>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    case 8: return blk_run<8>(c, A, r0_dev, values, f1, f2, iters, V_dev, maxvec);
    default: return set_error(TBGPU_E_ARG);
  }
}

// Double-precision Rayleigh-Ritz refinement of Ritz vectors (the final
// pass of the mixed-precision solves).  Vector e lives at V + e*stride
// (double complex); nseg disjoint segments [off, off + len) of the vectors are
// independent problems (one per dot of a batched solve; one segment of the
// whole vector otherwise), and H never couples two segments.  For groups of
// up to 8 vectors: W = H V with the double-precision recompute product (all
// segments at once), then per segment S = V^H V, G = V^H W, G y = lambda S y
// on the host (Cholesky S = U^H U, Hermitian eigenproblem of U^-H G U^-1);
// V <- V Y with S-orthonormal columns, values <- lambda (ascending), and the
// residual ||H v - lambda v|| and the change of each eigenvalue.  values,
// resid, delta are [nseg][nvec]; seg_nvec (or NULL: nvec each) gives the
// number of vectors a segment holds.
int refine_ritz(Ctx &c, double *V_dev, int nvec, long stride, int nseg, const long *seg_off,
                const long *seg_len, double *values, double *resid, double *delta,
                cudaStream_t s, const int *seg_nvec) {
  if (nvec <= 0 || nseg <= 0) return TBGPU_OK;
  if (!c.d_onsite || c.rc_warps <= 0) return set_error(TBGPU_E_STATE);
  const long dim = c.natoms * c.nb;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  long maxlen = 0;
  for (int q = 0; q < nseg; q++) maxlen = std::max(maxlen, seg_len[q]);
  const unsigned gmax =
      unsigned(std::max<long>(1, std::min<long>((maxlen + 255) / 256, long(sms) * 8)));
  constexpr int K8 = 8 * 9 / 2;
  const int mg = std::min(nvec, 8);
  double2 *W = nullptr, *T = nullptr;
  double *part = nullptr, *res = nullptr;
  unsigned *counter = nullptr;
  int rc = TBGPU_OK;
  if (cudaMalloc(&W, sizeof(double2) * dim * mg) != cudaSuccess ||
      cudaMalloc(&T, sizeof(double2) * dim * mg) != cudaSuccess ||
      cudaMalloc(&part, sizeof(double) * 2 * K8 * gmax) != cudaSuccess ||
      cudaMalloc(&res, sizeof(double) * 2 * K8 * 3) != cudaSuccess ||
      cudaMalloc(&counter, sizeof(unsigned)) != cudaSuccess)
    rc = TBGPU_E_NOMEM;
  if (!rc && cudaMemsetAsync(counter, 0, sizeof(unsigned), s) != cudaSuccess) rc = TBGPU_E_CUDA;
  double2 *V = reinterpret_cast<double2 *>(V_dev);
  // vectors j < m of a set with vector stride vs, offset off
  auto ptrs = [&](double2 *base, long vs, long off, int m) {
    BlockPtrs b{};
    for (int j = 0; j < 8; j++) b.v[j] = base + size_t(std::min(j, m - 1)) * vs + off;
    return b;
  };
  auto outs = [&](double2 *base, long vs, long off, int m) {
    BlockOut b{};
    for (int j = 0; j < m; j++) b.v[j] = base + size_t(j) * vs + off;
    return b;
  };
  // lower triangle of X^H Y as an m x m Hermitian matrix
  auto to_mat = [&](const double *h, int m) {
    Mat G(size_t(m) * m);
    int t = 0;
    for (int i = 0; i < 8; i++)
      for (int j = 0; j <= i; j++, t++)
        if (i < m && j < m) {
          G[i * m + j] = cplx(h[2 * t], h[2 * t + 1]);
          G[j * m + i] = std::conj(G[i * m + j]);
        }
    return G;
  };
  for (int g0 = 0; g0 < nvec && !rc; g0 += 8) {
    const int m_all = std::min(8, nvec - g0);
    double2 *Vg = V + size_t(g0) * stride;
    for (int i = 0; i < m_all && !rc; i++)
      rc = launch_spmv_recompute(c, reinterpret_cast<const double *>(Vg + size_t(i) * stride),
                                 reinterpret_cast<double *>(W + size_t(i) * dim), 0.0, nullptr,
                                 0, nullptr, 0, s);
    for (int q = 0; q < nseg && !rc; q++) {
      const long off = seg_off[q], n2 = seg_len[q];
      // this segment's vectors of the group (segments may hold fewer)
      const int m = std::min(m_all, (seg_nvec ? seg_nvec[q] : nvec) - g0);
      if (n2 <= 0 || m <= 0) continue;
      const unsigned grid =
          unsigned(std::max<long>(1, std::min<long>((n2 + 255) / 256, long(sms) * 8)));
      k_bdots<8><<<grid, kDotThreads, 0, s>>>(n2, ptrs(Vg, stride, off, m),
                                              ptrs(Vg, stride, off, m), part, counter, res);
      k_bdots<8><<<grid, kDotThreads, 0, s>>>(n2, ptrs(Vg, stride, off, m),
                                              ptrs(W, dim, off, m), part, counter, res + 2 * K8);
      double h[4 * K8];
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = TBGPU_E_CUDA;
        break;
      }
      const Mat S = to_mat(h, m), G = to_mat(h + 2 * K8, m);
      // Y (columns: refined vectors in the basis V) and lambda, ascending
      Mat Y(size_t(m) * m, cplx(0.0, 0.0));
      std::vector<double> lam(m);
      Mat U;
      if (cholesky_upper(m, S, U)) {
        const Mat Ui = upper_inverse(m, U);
        Mat UiH(size_t(m) * m);
        for (int i = 0; i < m; i++)
          for (int j = 0; j < m; j++) UiH[i * m + j] = std::conj(Ui[j * m + i]);
        const Mat Gp = matmul(m, matmul(m, UiH, G), Ui);
        std::vector<double> w;
        std::vector<std::vector<cplx>> Z;
        herm_eig_desc(m, Gp, w, Z);
        if (int(Z.size()) != m) {
          rc = TBGPU_E_NUMERIC;
          break;
        }
        for (int e = 0; e < m; e++) {  // herm_eig_desc is descending
          const int src = m - 1 - e;
          lam[e] = w[src];
          for (int i = 0; i < m; i++) {
            cplx v(0.0, 0.0);
            for (int k = 0; k < m; k++) v += Ui[i * m + k] * Z[src][k];
            Y[i * m + e] = v;
          }
        }
      } else {  // dependent vectors: plain Rayleigh quotients, one by one
        for (int e = 0; e < m; e++) {
          const double nn = S[e * m + e].real();
          if (!(nn > 0.0)) {
            rc = TBGPU_E_NUMERIC;
            break;
          }
          lam[e] = G[e * m + e].real() / nn;
          Y[e * m + e] = 1.0 / std::sqrt(nn);
        }
        if (rc) break;
      }
      SmallMat My{}, Ml{};
      for (int k = 0; k < m; k++)
        for (int e = 0; e < m; e++)
          My.m[k][e] = make_double2(Y[k * m + e].real(), Y[k * m + e].imag());
      for (int e = 0; e < m; e++) Ml.m[e][e] = make_double2(-lam[e], 0.0);
      // T = W Y; V = V Y (in place through T's second half is not possible:
      // the refined vectors go to T, the residuals to W, both segment-local)
      k_bcombine<8><<<grid, 256, 0, s>>>(n2, m, ptrs(W, dim, off, m), My, m,
                                         outs(T, dim, off, m), 0.0, ptrs(T, dim, off, m));
      k_bcombine<8><<<grid, 256, 0, s>>>(n2, m, ptrs(Vg, stride, off, m), My, m,
                                         outs(W, dim, off, m), 0.0, ptrs(W, dim, off, m));
      // W now holds V Y; T = T - W diag(lambda) are the residuals
      k_bcombine<8><<<grid, 256, 0, s>>>(n2, m, ptrs(W, dim, off, m), Ml, m,
                                         outs(T, dim, off, m), 1.0, ptrs(T, dim, off, m));
      k_bdots<8><<<grid, kDotThreads, 0, s>>>(n2, ptrs(T, dim, off, m), ptrs(T, dim, off, m),
                                              part, counter, res + 4 * K8);
      double hr[2 * K8];
      bool ok = cudaGetLastError() == cudaSuccess;
      for (int e = 0; e < m && ok; e++)
        ok = cudaMemcpyAsync(Vg + size_t(e) * stride + off, W + size_t(e) * dim + off,
                             sizeof(double2) * n2, cudaMemcpyDeviceToDevice, s) == cudaSuccess;
      if (!ok ||
          cudaMemcpyAsync(hr, res + 4 * K8, sizeof(hr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = TBGPU_E_CUDA;
        break;
      }
      for (int e = 0; e < m; e++) {
        const int t = e * (e + 1) / 2 + e;  // diagonal entry (e, e)
        const size_t at = size_t(q) * nvec + g0 + e;
        if (resid) resid[at] = std::sqrt(std::max(hr[2 * t], 0.0));
        if (delta) delta[at] = lam[e] - values[at];
        values[at] = lam[e];
      }
    }
  }
  cudaStreamSynchronize(s);
  cudaFree(W);
  cudaFree(T);
  cudaFree(part);
  cudaFree(res);
  cudaFree(counter);
  return rc ? set_error(rc) : TBGPU_OK;
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_eigensolve_blk_lanczos_dev(
    tbgpu_ctx *ctx, int ConvCheckStartIter, int ConvCheckSkipRate, int imax, int requested1,
    int requested2, double emin1, double emax1, double emin2, double emax2, double tolerance,
    int p, int max_no_success, const double *r0_dev, double *values, int *found_vb,
    int *found_cb, int *iterations, double *vectors_dev, int max_vectors) {
  if (!ctx || !r0_dev || !values || p < 1 || p > kMaxP || imax < 2 || ConvCheckSkipRate < 1 ||
      requested1 < 0 || requested2 < 0 || tolerance <= 0.0 || max_vectors < 0 ||
      misaligned16(r0_dev) || misaligned16(vectors_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  set_error(TBGPU_OK);
  BlkArgs A{ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2, p,
            max_no_success > 0 ? max_no_success : 1 << 30,
            emin1, emax1, emin2, emax2, tolerance};
  std::vector<double> vals;
  int f1 = 0, f2 = 0, it = 0;
  int rc = solve_block(c, A, r0_dev, vals, f1, f2, it, vectors_dev, max_vectors);
  if (rc) return rc;
  rc = take_status(c);  // a bounded device-side wait that ran out in a product
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
    int *found_cb, int *iterations, tbgpu_dcomplex *vectors, int max_vectors) {
  if (!ctx || !r0 || p < 1 || p > kMaxP || max_vectors < 0) return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t vb = sizeof(double2) * size_t(c.natoms) * c.nb;
  const int nv = vectors ? std::min(max_vectors, requested1 + requested2) : 0;
  double *d = nullptr, *dv = nullptr;
  if (cudaMalloc(&d, vb * p) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  if (nv > 0 && cudaMalloc(&dv, vb * nv) != cudaSuccess) {
    cudaFree(d);
    return set_error(TBGPU_E_NOMEM);
  }
  int rc = TBGPU_OK;
  if (cudaMemcpyAsync(d, r0, vb * p, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
    rc = set_error(TBGPU_E_CUDA);
  if (!rc)
    rc = tbgpu_eigensolve_blk_lanczos_dev(ctx, ConvCheckStartIter, ConvCheckSkipRate, imax,
                                          requested1, requested2, emin1, emax1, emin2, emax2,
                                          tolerance, p, max_no_success, d, values, found_vb,
                                          found_cb, iterations, dv, nv);
  if (rc > 0 && nv > 0) {
    const int got = std::min(rc, nv);
    if (cudaMemcpyAsync(vectors, dv, vb * got, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
      rc = set_error(TBGPU_E_CUDA);
  }
  cudaStreamSynchronize(c.stream);
  cudaFree(d);
  cudaFree(dv);
  return rc;
}
