// Momentum (optical) matrix elements of a set of eigenstates: the reference's
// MOMENTUM_MATRIX block (nemo3d/src/base/eigsys3d_par.c:410-640, the same
// code for Px, Py and Pz), with its output layout (pXmatrix) and transition
// table (TransProbX).
//
// The reference forms, per final state f and direction d, H psi_f, x H psi_f,
// x psi_f and H x psi_f (and the same for the Kramers partner psi'_f), then
// for every initial state temp1 = <a|x H b>, temp2 = <a|H x b> and
// p = i (temp2 - temp1): four H*x per final state and direction.  Here, with
// H Hermitian, temp2 = <H a|x b>, so
//   p_ab^d = i sum_j x_d(j) [conj((H a)_j) b_j - conj(a_j) (H b)_j],
// which needs H*x only once per state and partner (2n products for all three
// directions) and one fused pass over the vectors: per atom the bracket is
// summed over its orbitals once and weighted by the atom's three strained
// coordinates (getPosition_strained, nemo3d/src/base/geo_struct.c:2109-2131).
#include <algorithm>
#include <vector>

#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

constexpr int kSet = 16;        // vectors per side of one pass
constexpr int kRow = kSet + 1;  // padded shared-memory row (conflict-free staging)
constexpr int kTile = 2;        // atoms staged per step
constexpr int kThreads = kSet * kSet;  // one thread per (a, b) pair

struct VecSet {
  const double2 *v[kSet];
  const double2 *hv[kSet];
};

// Kramers partner psi' (eigsys3d_par.c:461-475): up <- -conj(down),
// down <- conj(up), per atom; psi, phi are [n][natoms*2*norb]
__global__ void k_kramers(long total, long natoms, int norb, const double2 *__restrict__ psi,
                          double2 *__restrict__ phi) {
  const int nb = 2 * norb;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long per = natoms * norb;
    const long k = e / per, r = e - k * per;
    const long a = r / norb;
    const int o = int(r - a * norb);
    const long base = (k * natoms + a) * nb;
    const double2 up = psi[base + o], dn = psi[base + norb + o];
    phi[base + o] = make_double2(-dn.x, dn.y);
    phi[base + norb + o] = make_double2(up.x, -up.y);
  }
}

// Per-block partial sums of S_ab^d = sum_j x_d(j) [conj((HA_a)_j) B_b,j -
// conj(A_a,j) (HB_b)_j] for a < na, b < nbv; thread (a, b) owns the three
// complex sums of its pair.  Vectors are staged kTile atoms at a time into
// shared memory as [set][atom][orbital][vector] so that the 16 b-values of a
// warp read one contiguous row.
template <int NB>
__global__ void __launch_bounds__(kThreads)
    k_momentum(long natoms, int na, VecSet A, int nbv, VecSet B,
               const int *__restrict__ atom_site, const double *__restrict__ dsp, int ny,
               int nz, double lx, double ly, double lz, double *__restrict__ partial) {
  extern __shared__ double2 sm[];  // [4][kTile][NB][kRow]
  __shared__ double pos[kTile][3];
  const int t = threadIdx.x;
  const int a = t / kSet, b = t - a * kSet;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  constexpr int PER = kSet * kTile * NB;
  for (long a0 = long(blockIdx.x) * kTile; a0 < natoms; a0 += long(gridDim.x) * kTile) {
    __syncthreads();  // the previous tile is consumed
    for (int e = t; e < 4 * PER; e += kThreads) {
      const int which = e / PER;  // 0: A, 1: H A, 2: B, 3: H B
      int r = e - which * PER;
      const int vec = r / (kTile * NB);
      r -= vec * (kTile * NB);
      const int ta = r / NB, o = r - ta * NB;
      const long atom = a0 + ta;
      double2 v = make_double2(0.0, 0.0);
      if (vec < (which < 2 ? na : nbv) && atom < natoms) {
        const double2 *src = which == 0 ? A.v[vec] : which == 1 ? A.hv[vec]
                           : which == 2 ? B.v[vec] : B.hv[vec];
        v = src[atom * NB + o];
      }
      sm[((which * kTile + ta) * NB + o) * kRow + vec] = v;
    }
    if (t < kTile) {
      const long atom = a0 + t;
      double p[3] = {0.0, 0.0, 0.0};
      if (atom < natoms) {
        const long s = atom_site[atom];
        const int m = int(s & 7);
        const long cell = s >> 3;
        const long k = cell % nz, j = (cell / nz) % ny, i = cell / (long(nz) * ny);
        const double lat[3] = {lx, ly, lz};
        const long ijk[3] = {i, j, k};
        for (int d = 0; d < 3; d++) {
          p[d] = lat[d] * (double(ijk[d]) + c_site_pos[m][d]);
          if (dsp) p[d] += dsp[s * 3 + d];
        }
      }
      pos[t][0] = p[0];
      pos[t][1] = p[1];
      pos[t][2] = p[2];
    }
    __syncthreads();
#pragma unroll
    for (int ta = 0; ta < kTile; ta++) {
      double mr = 0.0, mi = 0.0;
      const double2 *XA = sm + ((0 * kTile + ta) * NB) * kRow + a;
      const double2 *HA = sm + ((1 * kTile + ta) * NB) * kRow + a;
      const double2 *XB = sm + ((2 * kTile + ta) * NB) * kRow + b;
      const double2 *HB = sm + ((3 * kTile + ta) * NB) * kRow + b;
#pragma unroll 4
      for (int o = 0; o < NB; o++) {
        const double2 xa = XA[o * kRow], ha = HA[o * kRow];
        const double2 xb = XB[o * kRow], hb = HB[o * kRow];
        mr += (ha.x * xb.x + ha.y * xb.y) - (xa.x * hb.x + xa.y * hb.y);
        mi += (ha.x * xb.y - ha.y * xb.x) - (xa.x * hb.y - xa.y * hb.x);
      }
#pragma unroll
      for (int d = 0; d < 3; d++) {
        acc[2 * d] += pos[ta][d] * mr;
        acc[2 * d + 1] += pos[ta][d] * mi;
      }
    }
  }
  double *out = partial + (size_t(blockIdx.x) * kThreads + t) * 6;
#pragma unroll
  for (int k = 0; k < 6; k++) out[k] = acc[k];
}

// out[t][k] = sum over blocks, in block order (deterministic)
__global__ void k_momentum_sum(int nblocks, const double *__restrict__ partial,
                               double *__restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kThreads * 6) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; b++) s += partial[size_t(b) * kThreads * 6 + e];
  out[e] = s;
}

template <int NB>
int launch_momentum(Ctx &c, int grid, int na, const VecSet &A, int nbv, const VecSet &B,
                    double *partial, double *out, cudaStream_t s) {
  const size_t smem = sizeof(double2) * 4 * kTile * NB * kRow;
  static std::atomic<unsigned long long> attr_done{0};
  if (ensure_smem_attr(attr_done, c.device, k_momentum<NB>, int(smem))) return TBGPU_E_CUDA;
  k_momentum<NB><<<grid, kThreads, smem, s>>>(c.natoms, na, A, nbv, B, c.d_atom_site, c.d_dsp,
                                              c.ny, c.nz, c.lattice[0], c.lattice[1],
                                              c.lattice[2], partial);
  k_momentum_sum<<<(kThreads * 6 + 255) / 256, 256, 0, s>>>(grid, partial, out);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// double-precision H*x: the recompute product when the context keeps a float
// store for a mixed-precision solve, the context's own product otherwise
int hx_fp64(Ctx &c, const double2 *x, double2 *y, cudaStream_t s) {
  const double *X = reinterpret_cast<const double *>(x);
  double *Y = reinterpret_cast<double *>(y);
  if (c.lanczos_f32) return launch_spmv_recompute(c, X, Y, 0.0, nullptr, 0, nullptr, 0, s);
  return launch_spmv(c, X, Y, 0.0, nullptr, 0, nullptr, 0, s);
}

}  // namespace

int momentum_matrix(Ctx &c, int n, const double *psi_dev, const double *E, double *P,
                    double *trans) {
  if (n < 1 || !psi_dev || (trans && !E)) return set_error(TBGPU_E_ARG);
  if (!c.built) return set_error(TBGPU_E_STATE);
  if (c.nspin != 2 || c.bloch) return set_error(TBGPU_E_UNSUPPORTED);
  const long dim = c.natoms * c.nb;
  const size_t vb = sizeof(double2) * dim;
  cudaStream_t s = c.stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  const int grid = std::max(1, int(std::min<long>(long(sms) * 4, (c.natoms + kTile - 1) / kTile)));
  double2 *phi = nullptr, *Hpsi = nullptr, *Hphi = nullptr;
  double *partial = nullptr, *dout = nullptr;
  int rc = TBGPU_OK;
  if (cudaMalloc(&phi, vb * n) != cudaSuccess || cudaMalloc(&Hpsi, vb * n) != cudaSuccess ||
      cudaMalloc(&Hphi, vb * n) != cudaSuccess ||
      cudaMalloc(&partial, sizeof(double) * size_t(grid) * kThreads * 6) != cudaSuccess ||
      cudaMalloc(&dout, sizeof(double) * kThreads * 6) != cudaSuccess)
    rc = TBGPU_E_NOMEM;
  const double2 *psi = reinterpret_cast<const double2 *>(psi_dev);
  if (!rc) {
    const long total = long(n) * c.natoms * c.norb;
    k_kramers<<<unsigned(std::min<long>((total + 255) / 256, long(sms) * 16)), 256, 0, s>>>(
        total, c.natoms, c.norb, psi, phi);
    if (cudaGetLastError() != cudaSuccess) rc = TBGPU_E_CUDA;
  }
  for (int k = 0; k < n && !rc; k++) {
    rc = hx_fp64(c, psi + size_t(k) * dim, Hpsi + size_t(k) * dim, s);
    if (!rc) rc = hx_fp64(c, phi + size_t(k) * dim, Hphi + size_t(k) * dim, s);
  }
  // U = (psi_0..psi_{n-1}, psi'_0..psi'_{n-1}); S[u][v][d] complex
  const int nu = 2 * n;
  std::vector<double> S(size_t(nu) * nu * 6, 0.0);
  auto uvec = [&](int u) -> const double2 * {
    return u < n ? psi + size_t(u) * dim : phi + size_t(u - n) * dim;
  };
  auto uhv = [&](int u) -> const double2 * {
    return u < n ? Hpsi + size_t(u) * dim : Hphi + size_t(u - n) * dim;
  };
  for (int u0 = 0; u0 < nu && !rc; u0 += kSet)
    for (int v0 = 0; v0 < nu && !rc; v0 += kSet) {
      const int na = std::min(kSet, nu - u0), nbv = std::min(kSet, nu - v0);
      VecSet A{}, B{};
      for (int i = 0; i < kSet; i++) {
        A.v[i] = uvec(u0 + std::min(i, na - 1));
        A.hv[i] = uhv(u0 + std::min(i, na - 1));
        B.v[i] = uvec(v0 + std::min(i, nbv - 1));
        B.hv[i] = uhv(v0 + std::min(i, nbv - 1));
      }
      if (c.norb == 10) rc = launch_momentum<20>(c, grid, na, A, nbv, B, partial, dout, s);
      else rc = launch_momentum<10>(c, grid, na, A, nbv, B, partial, dout, s);
      std::vector<double> h(kThreads * 6);
      if (!rc && (cudaMemcpyAsync(h.data(), dout, sizeof(double) * h.size(),
                                  cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                  cudaStreamSynchronize(s) != cudaSuccess))
        rc = TBGPU_E_CUDA;
      for (int i = 0; i < na && !rc; i++)
        for (int j = 0; j < nbv; j++)
          for (int k = 0; k < 6; k++)
            S[(size_t(u0 + i) * nu + (v0 + j)) * 6 + k] = h[size_t(i * kSet + j) * 6 + k];
    }
  cudaStreamSynchronize(s);
  cudaFree(phi);
  cudaFree(Hpsi);
  cudaFree(Hphi);
  cudaFree(partial);
  cudaFree(dout);
  if (rc) return set_error(rc);
  // pXmatrix layout: [d][i][8f + 2c] = label, [8f + 2c + 1] = p, for the
  // pairs c = (psi_i, psi_f), (psi_i, psi'_f), (psi'_i, psi_f), (psi'_i, psi'_f);
  // p = i S = (-Im S, Re S)
  const int pairs[4][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}};
  long nt = 0;
  for (int d = 0; d < 3; d++) {
    nt = 0;
    for (int f = 0; f < n; f++)
      for (int i = 0; i < n; i++) {
        double rate = 0.0;
        for (int cc = 0; cc < 4; cc++) {
          const int u = i + n * pairs[cc][0], v = f + n * pairs[cc][1];
          const double sr = S[(size_t(u) * nu + v) * 6 + 2 * d];
          const double si = S[(size_t(u) * nu + v) * 6 + 2 * d + 1];
          const double pr = -si, pi = sr;
          rate += pr * pr + pi * pi;
          if (P) {
            double *row = P + ((size_t(d) * n + i) * 8 * n + 8 * f + 2 * cc) * 2;
            row[0] = (pairs[cc][0] ? -1.0 : 1.0) * (i + 1);
            row[1] = (pairs[cc][1] ? -1.0 : 1.0) * (f + 1);
            row[2] = pr;
            row[3] = pi;
          }
        }
        if (trans && i > f) {
          double *tr = trans + (size_t(d) * (size_t(n) * (n - 1) / 2) + nt) * 4;
          tr[0] = i + 1;
          tr[1] = f + 1;
          tr[2] = E[i] - E[f];
          tr[3] = rate;
          nt++;
        }
      }
  }
  return TBGPU_OK;
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_momentum_matrix(tbgpu_ctx *ctx, int n, const double *psi_dev,
                                     const double *E, double *P, double *trans) {
  if (!ctx || misaligned16(psi_dev)) return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  const int rc = momentum_matrix(c, n, psi_dev, E, P, trans);
  if (rc) return rc;
  return take_status(c);  // a bounded device-side wait that ran out in a product
}
