// Zincblende topology on the GPU: which sites hold atoms, the atom numbering,
// the four-neighbour table and the surface flags.
//
// Restates, for a dense cell grid:
//   remove_few_bonded_atoms(0)          nemo3d/src/base/geo_struct.c:1527-1579
//   get_total_hamiltonian_dimension_and_offsets
//                                       nemo3d/src/base/ham3d_final.c:547-568
//   FindSurfaceAtoms (bit 0, isOnSurface) nemo3d/src/base/geo_struct.c:1374-1463
// Atoms are numbered in site order (cell-major, k fastest, then in-cell site),
// which is the reference's vector layout.
#include <algorithm>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "tbgpu_internal.cuh"
#include "zincblende.cuh"

namespace tbgpu {

struct Grid {
  int nx, ny, nz, px, py, pz;
};

// neighbour site of site s along slot n; -1 outside a closed boundary.
// *wrapped is set when a periodic image is crossed; w (optional) receives the
// image crossed along each axis (-1, 0, +1).
__device__ __forceinline__ long nbr_site(const Grid g, long s, int n, bool *wrapped,
                                         int *w = nullptr) {
  const int m = int(s & 7);
  long cell = s >> 3;
  int k = int(cell % g.nz);
  int j = int((cell / g.nz) % g.ny);
  int i = int(cell / ((long)g.nz * g.ny));
  int c[3] = {i + c_nnmap[m][n][0], j + c_nnmap[m][n][1], k + c_nnmap[m][n][2]};
  const int dim[3] = {g.nx, g.ny, g.nz};
  const int per[3] = {g.px, g.py, g.pz};
  *wrapped = false;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (w) w[d] = 0;
    if (c[d] < 0 || c[d] >= dim[d]) {
      if (!per[d]) return -1;
      *wrapped = true;
      if (w) w[d] = c[d] < 0 ? -1 : 1;
      c[d] = (c[d] + dim[d]) % dim[d];
    }
  }
  return ((((long)c[0] * g.ny + c[1]) * g.nz + c[2]) << 3) + c_nnmap[m][n][3];
}

// 1 for a site that holds an atom bonded to at least one in-domain atom
// (periodic images are not counted here, as in remove_few_bonded_atoms).
__global__ void k_mark(Grid g, long nsites, const unsigned char *type, int *flag) {
  long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  int f = 0;
  if (type[s]) {
    for (int n = 0; n < 4; n++) {
      bool w;
      long t = nbr_site(g, s, n, &w);
      if (t >= 0 && !w && type[t]) { f = 1; break; }
    }
  }
  flag[s] = f;
}

__global__ void k_finalize(Grid g, long nsites, const int *flag, const int *index,
                           int *site_index, int *atom_site, int4 *nbr,
                           unsigned char *site_m, unsigned char *surface) {
  long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  if (!flag[s]) {
    site_index[s] = -1;
    return;
  }
  const int a = index[s];
  site_index[s] = a;
  atom_site[a] = int(s);
  site_m[a] = (unsigned char)(s & 7);
  int b[4], cnt = 0;
  for (int n = 0; n < 4; n++) {
    bool w;
    long t = nbr_site(g, s, n, &w);
    b[n] = (t >= 0 && flag[t]) ? index[t] : -1;
    cnt += b[n] >= 0;
  }
  nbr[a] = make_int4(b[0], b[1], b[2], b[3]);
  surface[a] = (unsigned char)(cnt != 4);
}

// Phase of H[a][b] for every bond: the conjugate of the Bloch factor of the
// periodic image crossed from a to b, exp(i*ph) with ph = -pi*(w.k -
// 2*int(0.5*w.k)) (geo_struct::phasePeriodic, nemo3d/src/base/geo_struct.h:
// 811-826, applied in Hmult_stored.c:386-437); 1 inside the domain.
__global__ void k_phase(Grid g, long natoms, const int *atom_site, const int4 *nbr,
                        double k0, double k1, double k2, double2 *phase) {
  long a = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const long s = atom_site[a];
  const int4 v = nbr[a];
  const int b[4] = {v.x, v.y, v.z, v.w};
  for (int n = 0; n < 4; n++) {
    double2 p = make_double2(1.0, 0.0);
    bool wrapped;
    int w[3];
    nbr_site(g, s, n, &wrapped, w);
    if (b[n] >= 0 && wrapped) {
      double ph = w[0] * k0 + w[1] * k1 + w[2] * k2;
      ph = -M_PI * (ph - 2 * (int)(0.5 * ph));
      double sn, cs;
      sincos(ph, &sn, &cs);
      p = make_double2(cs, -sn);
    }
    phase[a * 4 + n] = p;
  }
}

int build_phases(Ctx &c) {
  if (!c.d_phase) TB_CUDA(cudaMalloc(&c.d_phase, sizeof(double2) * 4 * c.natoms));
  Grid g{c.nx, c.ny, c.nz, c.periodic[0], c.periodic[1], c.periodic[2]};
  const int threads = 256;
  const unsigned blocks = unsigned((c.natoms + threads - 1) / threads);
  k_phase<<<blocks, threads, 0, c.stream>>>(g, c.natoms, c.d_atom_site, c.d_nbr, c.kvec[0],
                                            c.kvec[1], c.kvec[2], c.d_phase);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// Work order of the warp-staged H*x kernel.  Atoms are numbered in site
// order, so the atoms of a k-pencil of cells (i, j, 0..nz-1) are one
// contiguous run.  Visiting pencils j-block by j-block (kPencilBlock pencils
// wide, i slower than j inside a block) keeps the atoms that share a bond,
// and with it the x segments and bond blocks read twice, within a few
// thousand atoms of each other in processing order, so the second read hits
// L2; in plain atom order the i-direction neighbours are a whole y-z plane
// apart.
#ifndef TBGPU_PENCIL_BLOCK
#define TBGPU_PENCIL_BLOCK 8
#endif
constexpr int kPencilBlock = TBGPU_PENCIL_BLOCK;
constexpr int kGroupAtoms = 3;

static int build_work_order(Ctx &c, const int *index) {
  const long npen = long(c.nx) * c.ny;
  const size_t pitch = size_t(c.nz) * 8 * sizeof(int);
  std::vector<int> start(npen + 1);
  TB_CUDA(cudaMemcpy2DAsync(start.data(), sizeof(int), index, pitch, sizeof(int), npen,
                            cudaMemcpyDeviceToHost, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  start[npen] = int(c.natoms);
  std::vector<int2> groups;
  groups.reserve(c.natoms / kGroupAtoms + npen + 1);
  for (int jb = 0; jb < c.ny; jb += kPencilBlock)
    for (int i = 0; i < c.nx; i++)
      for (int j = jb; j < jb + kPencilBlock && j < c.ny; j++) {
        const long p = long(i) * c.ny + j;
        for (int a = start[p]; a < start[p + 1]; a += kGroupAtoms)
          groups.push_back(make_int2(a, std::min(kGroupAtoms, start[p + 1] - a)));
      }
  c.ngroups = long(groups.size());
  TB_CUDA(cudaMalloc(&c.d_groups, sizeof(int2) * groups.size()));
  TB_CUDA(cudaMemcpyAsync(c.d_groups, groups.data(), sizeof(int2) * groups.size(),
                          cudaMemcpyHostToDevice, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  return TBGPU_OK;
}

int build_topology(Ctx &c) {
  Grid g{c.nx, c.ny, c.nz, c.periodic[0], c.periodic[1], c.periodic[2]};
  const long ns = c.nsites;
  int *flag = nullptr, *index = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  const int threads = 256;
  const unsigned blocks = unsigned((ns + threads - 1) / threads);
  int rc = TBGPU_OK;
  if (cudaMallocAsync(&flag, sizeof(int) * (ns + 1), c.stream) != cudaSuccess ||
      cudaMallocAsync(&index, sizeof(int) * (ns + 1), c.stream) != cudaSuccess)
    return set_error(TBGPU_E_NOMEM);
  TB_CUDA(cudaMemsetAsync(flag + ns, 0, sizeof(int), c.stream));
  k_mark<<<blocks, threads, 0, c.stream>>>(g, ns, c.d_type, flag);
  TB_CUDA(cudaGetLastError());
  // exclusive scan over ns+1 entries: index[ns] is the atom count
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, index, ns + 1, c.stream);
  TB_CUDA(cudaMallocAsync(&tmp, tmp_bytes, c.stream));
  TB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, index, ns + 1, c.stream));
  int natoms = 0;
  TB_CUDA(cudaMemcpyAsync(&natoms, index + ns, sizeof(int), cudaMemcpyDeviceToHost,
                          c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  c.natoms = natoms;
  if (natoms <= 0) rc = set_error(TBGPU_E_ARG);
  if (rc == TBGPU_OK) {
    TB_CUDA(cudaMalloc(&c.d_site_index, sizeof(int) * ns));
    TB_CUDA(cudaMalloc(&c.d_atom_site, sizeof(int) * natoms));
    TB_CUDA(cudaMalloc(&c.d_nbr, sizeof(int4) * natoms));
    TB_CUDA(cudaMalloc(&c.d_site_m, natoms));
    TB_CUDA(cudaMalloc(&c.d_surface, natoms));
    k_finalize<<<blocks, threads, 0, c.stream>>>(g, ns, flag, index, c.d_site_index,
                                                 c.d_atom_site, c.d_nbr, c.d_site_m,
                                                 c.d_surface);
    TB_CUDA(cudaGetLastError());
    rc = build_work_order(c, index);
  }
  cudaFreeAsync(tmp, c.stream);
  cudaFreeAsync(flag, c.stream);
  cudaFreeAsync(index, c.stream);
  return rc;
}

}  // namespace tbgpu
