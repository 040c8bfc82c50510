// Keating valence-force-field strain relaxation on the GPU: the reference's
// min_estrain with StrainModel = VFF_keating (nemo3d/src/base/strain3d.c:
// 157-480), its energy and gradient calc_estrain (strain3d.c:1361-2080), the
// boundary conditions of calc_estrain_macopt (strain3d.c:816-1340) and the
// conjugate-gradient minimiser macoptII_par (NEMO_3D/eigen/src/macopt_par.c:
// 121-475, defaults of macopt_defaults, eigen/src/macopt.c:418-454).
//
// Energy: per atom m and present neighbours n, p, with nnv = a_latt*eta +
// (u_n - u_m), nnv0 = alat(m, n)*eta (eta: the neighbour's cell offset plus
// the in-cell position difference),
//   0.5*alpha/|nnv0|^2 * (|nnv|^2 - |nnv0|^2)^2                (each bond from
//                                                               both ends)
//   sqrt(beta_n beta_p)/sqrt(|nnv0_p|^2 |nnv0_n|^2) * (nnv_n.nnv_p - nnv0_n.nnv0_p)^2.
// The gradient is the reference's: the bond-stretching term moves only the
// vertex atom of each (atom, bond) term, so the gradient is that of
// (stretching/2 + bending); the minimiser, which uses gradients only, relaxes
// that function, and the energy reported is the reference's full sum.
//
// GPU layout: k_vff_vertex, one thread per atom, evaluates the atom's terms
// and writes its own gradient part and, per neighbour slot, the part that
// belongs to that neighbour (bond bending moves the arms); k_vff_gather sums,
// per atom, its own part and the parts its neighbours hold for it (through
// the fixed reverse-slot table), so every sum has a fixed order and no
// atomics are involved.  The line search and the CG recurrence run on the
// host from reduced scalars, exactly as macopt orders them.
#include <algorithm>
#include <cmath>
#include <vector>

#include "reduce.cuh"
#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads)
    k_vff_vertex(long natoms, const int *__restrict__ atom_site, const int4 *__restrict__ nbr,
                 const unsigned char *__restrict__ type, const double *__restrict__ vff, int ns,
                 double lx, double ly, double lz, const double *__restrict__ u,
                 double *__restrict__ own, double *__restrict__ arm, double *partial,
                 unsigned *counter, double *energy, int *status) {
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double e = 0.0;
  if (a < natoms) {
    const long s = atom_site[a];
    const int m = int(s & 7);
    const int tm = type[s];
    const int4 v4 = nbr[a];
    const int nb[4] = {v4.x, v4.y, v4.z, v4.w};
    const double lat[3] = {lx, ly, lz};
    double nnv[4][3], nnv0[4][3], al[4], be[4], d0sq[4];
    bool st[4];
    const double ua[3] = {u[a * 3], u[a * 3 + 1], u[a * 3 + 2]};
#pragma unroll
    for (int n = 0; n < 4; n++) {
      st[n] = nb[n] >= 0;
      if (!st[n]) continue;
      const long sn = atom_site[nb[n]];
      const int tn = type[sn];
      const int mn = c_nnmap[m][n][3];
      const double *vp = vff + (long(tm < ns ? tm : 0) * ns + (tn < ns ? tn : 0)) * 3;
      if (tm >= ns || tn >= ns || !(vp[0] > 0.0)) {
        atomicExch(status, TBGPU_E_MATERIAL);
        st[n] = false;
        continue;
      }
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const double disp = u[long(nb[n]) * 3 + q] - ua[q];
        const double r1 = double(c_nnmap[m][n][q]) + (c_site_pos[mn][q] - c_site_pos[m][q]);
        nnv[n][q] = lat[q] * r1 + disp;
        nnv0[n][q] = vp[0] * r1;
      }
      al[n] = vp[1];
      be[n] = vp[2];
      d0sq[n] = nnv0[n][0] * nnv0[n][0] + nnv0[n][1] * nnv0[n][1] + nnv0[n][2] * nnv0[n][2];
    }
    double go[3] = {0.0, 0.0, 0.0};
    double ga[4][3];
#pragma unroll
    for (int n = 0; n < 4; n++) ga[n][0] = ga[n][1] = ga[n][2] = 0.0;
#pragma unroll
    for (int n = 0; n < 4; n++) {
      if (!st[n]) continue;
      const double dssq = nnv[n][0] * nnv[n][0] + nnv[n][1] * nnv[n][1] + nnv[n][2] * nnv[n][2];
      const double bldc = 0.5 * al[n] / d0sq[n];
      const double bldl = dssq - d0sq[n];
      e += bldc * bldl * bldl;
      const double r1 = 4 * bldc * bldl;
#pragma unroll
      for (int q = 0; q < 3; q++) go[q] -= r1 * nnv[n][q];
#pragma unroll
      for (int p = n + 1; p < 4; p++) {
        if (!st[p]) continue;
        const double d0dot = nnv0[n][0] * nnv0[p][0] + nnv0[n][1] * nnv0[p][1] +
                             nnv0[n][2] * nnv0[p][2];
        const double dsdot = nnv[n][0] * nnv[p][0] + nnv[n][1] * nnv[p][1] + nnv[n][2] * nnv[p][2];
        const double bbdc = sqrt(be[n] * be[p]) / sqrt(d0sq[p] * d0sq[n]);
        const double bbdl = dsdot - d0dot;
        const double bb_mul = bbdc * bbdl;
        e += bb_mul * bbdl;
        const double bb2 = 2 * bb_mul;
#pragma unroll
        for (int q = 0; q < 3; q++) {
          ga[n][q] += nnv[p][q] * bb2;
          ga[p][q] += nnv[n][q] * bb2;
          go[q] -= (nnv[p][q] + nnv[n][q]) * bb2;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 3; q++) own[a * 3 + q] = go[q];
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int q = 0; q < 3; q++) arm[(a * 4 + n) * 3 + q] = ga[n][q];
  }
  if (energy) grid_reduce<kThreads>(e, partial, counter, energy, 0, false);
}

// g[a] = own[a] + sum over neighbours b of the part b holds for a; zero for
// atoms the boundary condition keeps fixed
__global__ void k_vff_gather(long natoms, const int4 *__restrict__ nbr,
                             const unsigned char *__restrict__ site_m,
                             const double *__restrict__ own, const double *__restrict__ arm,
                             const unsigned char *__restrict__ free_mask, double *__restrict__ g) {
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  double v[3] = {own[a * 3], own[a * 3 + 1], own[a * 3 + 2]};
  const int m = site_m[a];
  const int4 v4 = nbr[a];
  const int nb[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
  for (int n = 0; n < 4; n++) {
    if (nb[n] < 0) continue;
    const double *src = arm + (long(nb[n]) * 4 + c_rev_slot[m][n]) * 3;
#pragma unroll
    for (int q = 0; q < 3; q++) v[q] += src[q];
  }
  const bool f = free_mask ? free_mask[a] != 0 : true;
#pragma unroll
  for (int q = 0; q < 3; q++) g[a * 3 + q] = f ? v[q] : 0.0;
}

// boundary conditions of calc_estrain_macopt: 0 AllFree, 1 FixOne,
// 2 FixSurfaceAll, 3 FixZmin (two lowest cell layers, isInZ_min), 4
// FixInterior
__global__ void k_vff_mask(long natoms, const int *__restrict__ atom_site,
                           const unsigned char *__restrict__ surface, int nz, int bc,
                           unsigned char *__restrict__ mask) {
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const long cell = atom_site[a] >> 3;
  const int k = int(cell % nz);
  bool f = true;
  if (bc == 1) f = a != 0;
  else if (bc == 2) f = !surface[a];
  else if (bc == 3) f = k > 1;
  else if (bc == 4) f = surface[a] != 0;
  mask[a] = f ? 1 : 0;
}

__global__ void k_site_to_atom(long natoms, const int *__restrict__ atom_site,
                               const double *__restrict__ dsp, double *__restrict__ u) {
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const long s = atom_site[a];
  for (int q = 0; q < 3; q++) u[a * 3 + q] = dsp ? dsp[s * 3 + q] : 0.0;
}

__global__ void k_atom_to_site(long natoms, const int *__restrict__ atom_site,
                               const double *__restrict__ u, double *__restrict__ dsp) {
  const long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const long s = atom_site[a];
  for (int q = 0; q < 3; q++) dsp[s * 3 + q] = u[a * 3 + q];
}

// --- vector kernels of the minimiser (n = 3 natoms doubles) ---------------
__global__ void k_line(long n, const double *__restrict__ u, double y,
                       const double *__restrict__ xi, double *__restrict__ pt) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x)
    pt[j] = u[j] + y * xi[j];
}

// out = sum (a + b) . c   (b may be null)
__global__ void __launch_bounds__(kThreads)
    k_dot(long n, const double *__restrict__ a, const double *__restrict__ b,
          const double *__restrict__ c, double *partial, unsigned *counter, double *out,
          int idx) {
  double s = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x)
    s += (a[j] + (b ? b[j] : 0.0)) * c[j];
  grid_reduce<kThreads>(s, partial, counter, out, idx, false);
}

// u += m xi (sum |m xi|), xi = s gy + t gx
__global__ void __launch_bounds__(kThreads)
    k_vff_step(long n, double *__restrict__ u, double *__restrict__ xi,
               const double *__restrict__ gx, const double *__restrict__ gy, double m,
               double s, double t, double *partial, unsigned *counter, double *out) {
  double st = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x) {
    const double d = m * xi[j];
    u[j] += d;
    st += fabs(d);
    xi[j] = s * gy[j] + t * gx[j];
  }
  grid_reduce<kThreads>(st, partial, counter, out, 0, false);
}

// g = -xi; xi = h = g + gam h; out = -sum xi.g
__global__ void __launch_bounds__(kThreads)
    k_vff_cg(long n, double *__restrict__ g, double *__restrict__ xi, double *__restrict__ h,
             double gam, double *partial, unsigned *counter, double *out) {
  double s = 0.0;
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x) {
    const double gj = -xi[j];
    g[j] = gj;
    const double x = gj + gam * h[j];
    xi[j] = h[j] = x;
    s -= x * gj;
  }
  grid_reduce<kThreads>(s, partial, counter, out, 0, false);
}

// macopt_restart: (g = -xi unless keep_g); xi = h = g
__global__ void k_vff_restart(long n, int keep_g, double *__restrict__ g,
                              double *__restrict__ xi, double *__restrict__ h) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x) {
    const double gj = keep_g ? g[j] : -xi[j];
    g[j] = gj;
    xi[j] = h[j] = gj;
  }
}

struct Vff {
  Ctx &c;
  long natoms = 0, n = 0;
  unsigned grid_a = 1, grid_v = 1;
  double *vff = nullptr, *own = nullptr, *arm = nullptr, *u = nullptr;
  unsigned char *mask = nullptr;
  double *red = nullptr;  // device scalars
  double *host = nullptr; // pinned readback
  unsigned *counter = nullptr;
  double *partial = nullptr;
  int rc = TBGPU_OK;
  explicit Vff(Ctx &ctx) : c(ctx) {}
  ~Vff() {
    cudaStreamSynchronize(c.stream);
    cudaFree(vff); cudaFree(own); cudaFree(arm); cudaFree(u); cudaFree(mask);
    cudaFree(red); cudaFree(counter); cudaFree(partial);
    if (host) cudaFreeHost(host);
  }
  int init(const double *vff_host) {
    natoms = c.natoms;
    n = 3 * natoms;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    grid_a = unsigned((natoms + kThreads - 1) / kThreads);
    grid_v = unsigned(std::max<long>(1, std::min<long>((n + kThreads - 1) / kThreads, sms * 8L)));
    const unsigned pmax = std::max(grid_a, grid_v);
    const size_t nv = size_t(c.nspecies) * c.nspecies * 3;
    if (cudaMalloc(&vff, sizeof(double) * nv) != cudaSuccess ||
        cudaMalloc(&own, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&arm, sizeof(double) * 4 * n) != cudaSuccess ||
        cudaMalloc(&u, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&mask, natoms) != cudaSuccess ||
        cudaMalloc(&red, sizeof(double) * 4) != cudaSuccess ||
        cudaMalloc(&counter, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&partial, sizeof(double) * pmax) != cudaSuccess ||
        cudaMallocHost(&host, sizeof(double) * 4) != cudaSuccess)
      return set_error(TBGPU_E_NOMEM);
    TB_CUDA(cudaMemcpyAsync(vff, vff_host, sizeof(double) * nv, cudaMemcpyHostToDevice, c.stream));
    TB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), c.stream));
    return TBGPU_OK;
  }
  // g = gradient at x (free atoms only when masked); energy to red[0] if asked
  int grad(const double *x, double *g, bool masked, bool with_energy) {
    k_vff_vertex<<<grid_a, kThreads, 0, c.stream>>>(
        natoms, c.d_atom_site, c.d_nbr, c.d_type, vff, c.nspecies, c.lattice[0], c.lattice[1],
        c.lattice[2], x, own, arm, partial, counter, with_energy ? red : nullptr, c.d_status);
    k_vff_gather<<<grid_a, kThreads, 0, c.stream>>>(natoms, c.d_nbr, c.d_site_m, own, arm,
                                                     masked ? mask : nullptr, g);
    TB_CUDA(cudaGetLastError());
    return TBGPU_OK;
  }
  // the device scalar red[i] on the host
  int read(int i, double &out) {
    TB_CUDA(cudaMemcpyAsync(host, red + i, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    TB_CUDA(cudaStreamSynchronize(c.stream));
    out = host[0];
    return std::isfinite(out) ? TBGPU_OK : set_error(TBGPU_E_NUMERIC);
  }
  int dot(const double *a, const double *b, const double *cc, double &out) {
    k_dot<<<grid_v, kThreads, 0, c.stream>>>(n, a, b, cc, partial, counter, red, 1);
    TB_CUDA(cudaGetLastError());
    return read(1, out);
  }
};

int ensure_topology(Ctx &c) {
  if (c.topo_built) return TBGPU_OK;
  int rc = build_topology(c);
  if (rc == TBGPU_OK) c.topo_built = true;
  return rc;
}

int vff_status(Ctx &c) {
  int st = 0;
  TB_CUDA(cudaMemcpyAsync(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  if (st) {
    cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream);
    return set_error(st);
  }
  return TBGPU_OK;
}

}  // namespace

int vff_energy(Ctx &c, const double *vff_host, double *energy, double *grad_sites) {
  if (!vff_host) return set_error(TBGPU_E_ARG);
  if (c.built) return set_error(TBGPU_E_STATE);
  int rc = ensure_topology(c);
  if (rc) return rc;
  Vff V(c);
  if ((rc = V.init(vff_host))) return rc;
  k_site_to_atom<<<V.grid_a, kThreads, 0, c.stream>>>(V.natoms, c.d_atom_site, c.d_dsp, V.u);
  double *g = nullptr;
  if (cudaMalloc(&g, sizeof(double) * V.n) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  rc = V.grad(V.u, g, false, true);
  double e = 0.0;
  if (!rc) rc = V.read(0, e);
  if (!rc) rc = vff_status(c);
  if (!rc && grad_sites) {
    double *gs = nullptr;
    if (cudaMalloc(&gs, sizeof(double) * 3 * c.nsites) != cudaSuccess) rc = set_error(TBGPU_E_NOMEM);
    if (!rc && (cudaMemsetAsync(gs, 0, sizeof(double) * 3 * c.nsites, c.stream) != cudaSuccess))
      rc = set_error(TBGPU_E_CUDA);
    if (!rc) {
      k_atom_to_site<<<V.grid_a, kThreads, 0, c.stream>>>(V.natoms, c.d_atom_site, g, gs);
      if (cudaMemcpyAsync(grad_sites, gs, sizeof(double) * 3 * c.nsites, cudaMemcpyDeviceToHost,
                          c.stream) != cudaSuccess ||
          cudaStreamSynchronize(c.stream) != cudaSuccess)
        rc = set_error(TBGPU_E_CUDA);
    }
    cudaFree(gs);
  }
  cudaFree(g);
  if (!rc && energy) *energy = e;
  return rc;
}

int vff_relax(Ctx &c, const double *vff_host, int bc, int itmax, double tol,
              int end_if_small_step, double *energy, int *iterations, double *dsp_sites) {
  if (!vff_host || bc < 0 || bc > 4 || itmax < 1 || !(tol >= 0.0)) return set_error(TBGPU_E_ARG);
  if (c.built) return set_error(TBGPU_E_STATE);
  int rc = ensure_topology(c);
  if (rc) return rc;
  if (!c.d_dsp) {
    TB_CUDA(cudaMalloc(&c.d_dsp, sizeof(double) * 3 * c.nsites));
    TB_CUDA(cudaMemsetAsync(c.d_dsp, 0, sizeof(double) * 3 * c.nsites, c.stream));
  }
  Vff V(c);
  if ((rc = V.init(vff_host))) return rc;
  const long n = V.n;
  double *g = nullptr, *h = nullptr, *xi = nullptr, *pt = nullptr, *gx = nullptr, *gy = nullptr;
  double *all = nullptr;
  if (cudaMalloc(&all, sizeof(double) * 6 * n) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  g = all; h = all + n; xi = all + 2 * n; pt = all + 3 * n; gx = all + 4 * n; gy = all + 5 * n;
  k_vff_mask<<<V.grid_a, kThreads, 0, c.stream>>>(V.natoms, c.d_atom_site, c.d_surface, c.nz, bc,
                                                   V.mask);
  k_site_to_atom<<<V.grid_a, kThreads, 0, c.stream>>>(V.natoms, c.d_atom_site, c.d_dsp, V.u);
  double *u = V.u;
  const int end_if_small_grad = 1 - end_if_small_step;
  int rich = 1, restart = 0, its = 0;
  double lastx = 0.01, gtyp = 0.0;
  const double dn = double(n);
  // s = gy . xi at pt = u + y xi
  auto macprod = [&](double y, double *gout, double &res) -> int {
    k_line<<<V.grid_v, kThreads, 0, c.stream>>>(n, u, y, xi, pt);
    int r = V.grad(pt, gout, true, false);
    if (r) return r;
    return V.dot(gout, nullptr, xi, res);
  };
  rc = V.grad(u, xi, true, false);
  if (!rc) {
    k_vff_restart<<<V.grid_v, kThreads, 0, c.stream>>>(n, 0, g, xi, h);
    for (its = 1; its <= itmax && !rc; ++its) {
      double gg = 0.0;
      if ((rc = V.dot(g, nullptr, g, gg))) break;
      gtyp = std::sqrt(gg / dn);
      if ((end_if_small_grad && gg <= tol) || gg <= 1e-28) break;
      // maclinmin
      double x = lastx / gtyp, y = 0.0, s = 0.0, t = 0.0;
      double *ga = gx, *gb = gy;
      int lits = 1;
      if ((rc = macprod(x, ga, s))) break;
      if (s < 0) {
        do {
          y = x * 2.0;
          if ((rc = macprod(y, gb, t))) break;
          if (t >= 0.0) break;
          x = y; s = t; std::swap(ga, gb);
          ++lits;
        } while (lits <= 20);
      } else if (s > 0) {
        do {
          y = x * 0.5;
          if ((rc = macprod(y, gb, t))) break;
          if (t <= 0.0) break;
          x = y; s = t; std::swap(ga, gb);
          ++lits;
        } while (lits <= 20);
      } else {
        t = 1.0;
        y = x;
      }
      if (rc) break;
      if (lits > 20) {
        double tmpd = 0.0;
        if ((rc = macprod(0.0, gb, tmpd))) break;
        if (tmpd > 0 && rich == 0) rich = 1;
        if (tmpd > 0) restart = 1;
      }
      s = std::fabs(s);
      t = std::fabs(t);
      double m = s + t;
      s /= m;
      t /= m;
      m = s * y + t * x;
      double step = 0.0;
      k_vff_step<<<V.grid_v, kThreads, 0, c.stream>>>(n, u, xi, ga, gb, m, s, t, V.partial,
                                                        V.counter, V.red + 2);
      if ((rc = V.read(2, step))) break;
      lastx = m * 1.25 * gtyp;
      step /= dn;
      if (((end_if_small_step && step <= tol) || step <= 0.0) && restart == 0) break;
      if (rich || restart)
        if ((rc = V.grad(u, xi, true, false))) break;
      if (restart) {
        lastx = 0.01;
        k_vff_restart<<<V.grid_v, kThreads, 0, c.stream>>>(n, restart == 2, g, xi, h);
        restart = 0;
      } else {
        double dgg = 0.0, tmpd = 0.0;
        if ((rc = V.dot(xi, g, xi, dgg))) break;
        const double gam = dgg / gg;
        k_vff_cg<<<V.grid_v, kThreads, 0, c.stream>>>(n, g, xi, h, gam, V.partial, V.counter,
                                                        V.red + 3);
        if ((rc = V.read(3, tmpd))) break;
        if (tmpd > 0.0) {
          rich = 1;
          lastx = 0.01;
          k_vff_restart<<<V.grid_v, kThreads, 0, c.stream>>>(n, 1, g, xi, h);
        }
      }
    }
  }
  double e = 0.0;
  if (!rc) rc = V.grad(u, gx, false, true);
  if (!rc) rc = V.read(0, e);
  if (!rc) rc = vff_status(c);
  if (!rc) {
    k_atom_to_site<<<V.grid_a, kThreads, 0, c.stream>>>(V.natoms, c.d_atom_site, u, c.d_dsp);
    if (dsp_sites &&
        (cudaMemcpyAsync(dsp_sites, c.d_dsp, sizeof(double) * 3 * c.nsites,
                         cudaMemcpyDeviceToHost, c.stream) != cudaSuccess))
      rc = set_error(TBGPU_E_CUDA);
    if (cudaStreamSynchronize(c.stream) != cudaSuccess && !rc) rc = set_error(TBGPU_E_CUDA);
  }
  cudaFree(all);
  if (rc) return rc;
  if (energy) *energy = e;
  if (iterations) *iterations = std::min(its, itmax);
  return TBGPU_OK;
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_vff_energy(tbgpu_ctx *ctx, const double *vff, double *energy,
                                double *grad) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  return vff_energy(*reinterpret_cast<Ctx *>(ctx), vff, energy, grad);
}

extern "C" int tbgpu_vff_relax(tbgpu_ctx *ctx, const double *vff, int bc, int max_iter,
                               double tol, int end_if_small_step, double *energy,
                               int *iterations, double *dsp) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  return vff_relax(*reinterpret_cast<Ctx *>(ctx), vff, bc, max_iter, tol, end_if_small_step,
                   energy, iterations, dsp);
}
