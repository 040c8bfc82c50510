// Internal definitions shared by the libtbgpu.so translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <complex>
#include <cstdint>
#include <vector>

#include "../../include/tbgpu.h"

namespace tbgpu {

// The reference's sqrt(3) (nemo3d/src/ham/mb_ham_spds_micro.c:42).  Kept so
// that Hamiltonian entries agree with the reference to 1e-12.
constexpr double kSqr3 = 1.73205080757;

constexpr int kNPV = 35;
constexpr int kNPAR = TBGPU_NPAR;

// parameter-vector indices (nemo3d/src/ham/mb_ham_spds_micro.h:100-264)
enum : int {
  pE_sa = 0, pE_pa = 1, pE_sc = 2, pE_pc = 3, pE_sta = 4, pE_stc = 5,
  pE_da = 6, pE_dc = 7, pE_La = 8, pE_Lc = 9, pA0 = 31
};
enum : int {
  eta_ssts = 0, eta_ststs, eta_sss, eta_sps, eta_pps, eta_ppp, eta_sds,
  eta_stps, eta_pds, eta_pdp, eta_const, eta_dds, eta_ddp, eta_ddd, eta_stds,
  eta_cat_shift, eta_an_shift
};

// per-atom on-site record (doubles): [0,nb) diagonal, [nb] spin-orbit
// lambda, [nb+1] passivated flag, [nb+2, nb+8) dangling-bond sp3 couplings
// (s-x, s-y, s-z, x-y, x-z, y-z); padded to a multiple of 8 doubles.
__host__ __device__ constexpr int onsite_len(int nb) { return ((nb + 8 + 7) / 8) * 8; }

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
};

struct Ctx {
  // model
  int band_model = 0, norb = 0, nspin = 0, nb = 0, ons = 0;
  int include_strain = 1, passivate = 1;
  double dangling_shift = 0.0;
  int nspecies = 0;
  // geometry
  int nx = 0, ny = 0, nz = 0;
  int periodic[3] = {0, 0, 0};
  double lattice[3] = {0, 0, 0};
  long nsites = 0;
  long natoms = 0;
  bool built = false;
  bool topo_built = false;  // topology done (by the build or a strain relaxation)
  int device = 0;
  int sms = 0;                      // multiprocessors of the context's device
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // device arrays
  unsigned char *d_type = nullptr;  // [nsites]
  double *d_dsp = nullptr;          // [nsites*3] or null
  double *d_par = nullptr;          // [ns*ns*NPAR]
  unsigned char *d_par_ok = nullptr;
  int *d_site_index = nullptr;      // [nsites] atom index or -1
  int *d_atom_site = nullptr;       // [natoms]
  int4 *d_nbr = nullptr;            // [natoms]
  unsigned char *d_site_m = nullptr;// [natoms] in-cell site 0..7
  unsigned char *d_surface = nullptr;
  double *d_onsite = nullptr;       // [natoms*ons]
  double *d_blocks = nullptr;       // [natoms*4*norb*norb], cation atoms
  // single-precision store (the reference's HamMemorySave build): the same
  // arrays in float, and d_onsite / d_blocks released after assembly
  bool ham_fp32 = false;
  // blocks recomputed inside every H*x instead of stored (HamCompute=Recompute)
  bool recompute = false;
  // recompute work order: eight cations per warp, then eight anions per
  // warp, padded with -1 (rc_cat_warps warps of cations, rc_warps in all)
  int *d_rc_order = nullptr;
  long rc_cat_warps = 0, rc_warps = 0;
  // mixed-precision Lanczos: complex-float vectors over the single-precision
  // store, then a double-precision Rayleigh-Ritz refinement of the Ritz
  // vectors through the recompute product (the double on-site records and
  // the recompute work order are kept for it)
  bool lanczos_f32 = false;
  // per atom, 1 = left out of the products (set only while a batched solve
  // runs, for the dots that have converged); null otherwise
  const unsigned char *d_skip = nullptr;
  std::vector<double> state_resid, state_delta;  // per state of the last solve
  float *d_onsite32 = nullptr;
  float *d_blocks32 = nullptr;
  // H*x work order: groups of up to 3 consecutive atoms of one k-pencil of
  // cells, pencils visited in j-blocks (first atom, atom count)
  int2 *d_groups = nullptr;
  long ngroups = 0;
  // unit table of H*x variant 3 (units of two cells of one pencil; built on
  // first use): nunits descriptors of unit_stride ints, stage capacities
  int *d_units = nullptr;
  long nunits = 0;
  int unit_stride = 0, unit_cap_nb = 0, unit_cap_nx = 0;
  // reduction scratch (per-block partials + completion counter)
  double *d_partial = nullptr;
  unsigned int *d_counter = nullptr;
  int partial_cap = 0;
  int *d_status = nullptr;          // device error word
  // Lanczos state
  std::vector<double> alpha, beta;  // host copy of the last tridiagonal
  // stats
  tbgpu_stats stats{};
  bool profiling = false;
  int spmv_variant = 0;
  // Bloch phases of bonds that cross a periodic boundary (off: Gamma point)
  bool bloch = false;
  double kvec[3] = {0, 0, 0};
  double2 *d_phase = nullptr;       // [natoms*4] phase of H[a][nbr], or null
  // scratch for the host-pointer matvec
  double *d_x = nullptr, *d_y = nullptr;
  // start vector set by tbgpu_set_start_vector (used when a solve gets none)
  double *d_start = nullptr;
  // task list of the lane-per-(atom, spin) H*x kernel (spmv_lane.cu; built on
  // first use): lane_ntasks tasks of lane_apw atom indices (-1 padded)
  int *d_lane_tasks = nullptr;
  long lane_ntasks = 0;
  int lane_apw = 0;
  int lane_jblock = 0;   // pencils per j-block of its work order (0: 8)
  // the pencil layout of the stored Hamiltonian (spmv_pen.cu; built on first
  // use): bond blocks as column pairs, on-site records, site mask; scratch
  // for products on vectors in the reference's order
  void *d_pen_blk = nullptr, *d_pen_ons = nullptr;
  unsigned char *d_pen_ok = nullptr;
  bool pen_fp32 = false;
  void *d_pen_scratch = nullptr;
  size_t pen_scratch_bytes = 0;
  // eigenvector pass of the Lanczos solve: 0 = the reference's second run of
  // the recurrence from the start vector; 1 = regeneration of vec_segment-
  // iteration segments from checkpoints saved by the first pass,
  // vec_columns segments at a time (lane kernel products, update fused)
  int vec_pass = 0, vec_columns = 4, vec_segment = 256;
  // block Lanczos dots: 0 = double-precision CUDA-core kernel, 1 = the
  // tensor-core (tcgen05 kind::i8 slice) kernel
  int block_dots = 0;
  // mixed-precision recurrence: floor of the bound on the last components of
  // a tridiagonal eigenvector that accepts its Ritz value (0: the caller's
  // tolerance, as in double precision)
  double mixed_accept = 0.0;
  // folded-spectrum operator F = factor (H - s2)(H - s1) + offset of
  // matvect_mult2 (nemo3d/src/base/h_cvectr_mult.c:156-198; its constants
  // by default); fold on: the Lanczos solves run on F
  bool fold = false;
  double fold_s1 = 1.48 - 0.1, fold_s2 = 1.48 + 0.1, fold_factor = -10.0, fold_offset = 0.0;
  std::vector<double> fold_energy;  // <v, H v> of the last folded solve's vectors
  double *d_fold_tmp = nullptr;     // scratch of the host-pointer folded matvec
};

// the stored Hamiltonian in its element type
template <typename HT> inline const HT *ham_blocks(const Ctx &c);
template <> inline const double *ham_blocks<double>(const Ctx &c) { return c.d_blocks; }
template <> inline const float *ham_blocks<float>(const Ctx &c) { return c.d_blocks32; }
template <typename HT> inline const HT *ham_onsite(const Ctx &c);
template <> inline const double *ham_onsite<double>(const Ctx &c) { return c.d_onsite; }
template <> inline const float *ham_onsite<float>(const Ctx &c) { return c.d_onsite32; }

// error helpers
int set_error(int code);
// The status word of the context's kernels (a device-side wait that ran
// out, a bad species id): read after the context's stream drained, cleared,
// and returned as the call's status (TBGPU_OK when clear).
int take_status(Ctx &c);
// the solver's per-device memory pool (memory kept mapped between solves;
// nullptr if it could not be made) and its reserved but unused bytes
cudaMemPool_t solver_pool(int device);
size_t solver_pool_spare(int device);
template <typename T>
inline cudaError_t solver_alloc(int device, T **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = solver_pool(device);
  void *q = nullptr;
  const cudaError_t e =
      pool ? cudaMallocFromPoolAsync(&q, bytes, pool, s) : cudaMallocAsync(&q, bytes, s);
  *p = static_cast<T *>(q);
  return e;
}

// Dynamic shared memory above 48 KB is allowed per kernel and per device
// context.  `done` (one per kernel instance) records the devices already
// set; devices past 63 set it on every launch.  Setting it twice from two
// host threads is harmless.
template <typename K>
inline int ensure_smem_attr(std::atomic<unsigned long long> &done, int device, K *func,
                            int bytes) {
  const unsigned long long bit = (device >= 0 && device < 64) ? 1ull << device : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return TBGPU_OK;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
      cudaSuccess)
    return set_error(TBGPU_E_CUDA);
  done.fetch_or(bit, std::memory_order_acq_rel);
  return TBGPU_OK;
}
// device vectors must start on a 16-byte boundary (the kernels move them in
// 16-byte pieces); null passes
inline bool misaligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) != 0; }
#define TB_CUDA(call)                                              \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ::tbgpu::set_error(TBGPU_E_CUDA); \
  } while (0)

// spmm_async.cu: y + v*ystride = (H - shift)(x + v*xstride) for v < p <= 8
int launch_spmm(Ctx &c, int p, const double *x, long xstride, double *y, long ystride,
                double shift, cudaStream_t s);

// band_eig.cu: eigenvalues in (vl, vu] of a Hermitian band matrix (lower
// band storage, ldab = kd + 1), ascending
int band_eigenvalues(int n, int kd, const std::complex<double> *ab, double vl, double vu,
                     double abstol, std::vector<double> &w);

// topology.cu
int build_topology(Ctx &c);
int build_phases(Ctx &c);  // fills d_phase for c.kvec
// build.cu
int assemble(Ctx &c);
int compute_blocks(Ctx &c, double *blocks);
// recompute.cu
int build_recompute_order(Ctx &c);
int launch_spmv_recompute_f32(Ctx &c, const float *x, float *y, double shift,
                              const double *xnorm, int xidx, double *alpha_out, int aidx,
                              cudaStream_t s);
int launch_spmv_recompute(Ctx &c, const double *x, double *y, double shift,
                          const double *xnorm, int xidx, double *alpha_out, int aidx,
                          cudaStream_t s);
// spmv.cu
int launch_spmv(Ctx &c, const double *x, double *y, double shift,
                const double *xscale_dev, int scale_index, double *alpha_out,
                int alpha_index, cudaStream_t s);
int launch_spmv_f32(Ctx &c, const float *x, float *y, double shift, const double *xscale_dev,
                    int scale_index, double *alpha_out, int alpha_index, cudaStream_t s);
// spmv_async.cu
int launch_spmv_async(Ctx &c, const double *x, double *y, double shift,
                      const double *xscale_dev, int scale_index, double *alpha_out,
                      int alpha_index, cudaStream_t s);
int launch_spmv_async_f32(Ctx &c, const float *x, float *y, double shift,
                          const double *xscale_dev, int scale_index, double *alpha_out,
                          int alpha_index, cudaStream_t s);
// spmv_lane.cu: lane per (atom, spin), 10-orbital models, stored blocks,
// Gamma point (variant 5)
// columns one regenerating pass can take: 4 complex-float or 2 complex-double
constexpr int lane_max_cols(bool f32) { return f32 ? 4 : 2; }
bool lane_supported(const Ctx &c);
int launch_spmv_lane(Ctx &c, const double *x, double *y, double shift,
                     const double *xscale_dev, int scale_index, double *alpha_out,
                     int alpha_index, cudaStream_t s);
int launch_spmv_lane_f32(Ctx &c, const float *x, float *y, double shift,
                         const double *xscale_dev, int scale_index, double *alpha_out,
                         int alpha_index, cudaStream_t s);
// p Lanczos segments advanced by one step in one pass, the update fused:
// y[j] = next r of the segment whose current r is x[j] at iteration it[j]
template <typename VT>
int launch_lane_regen(Ctx &c, int p, const VT *const *x, VT *const *y, const VT *const *rp,
                      const int *it, const double *bet, const double *alpha, cudaStream_t s);
// spmv_pen.cu: pencil-interleaved layout (variant 6), 10-orbital models,
// stored blocks, Gamma point, no skip mask
bool pen_supported(const Ctx &c);
bool pen_staged(const Ctx &c);
long pen_length(const Ctx &c);  // complex entries of a pencil-layout vector
int launch_spmv_pen(Ctx &c, const double *x, double *y, double shift, const double *xscale_dev,
                    int scale_index, double *alpha_out, int alpha_index, cudaStream_t s);
int launch_spmv_pen_f32(Ctx &c, const float *x, float *y, double shift,
                        const double *xscale_dev, int scale_index, double *alpha_out,
                        int alpha_index, cudaStream_t s);
// on vectors already in the pencil layout (the solver's)
template <typename VT>
int launch_spmv_pen_internal(Ctx &c, const VT *x, VT *y, double shift, const double *xnorm,
                             int xidx, double *alpha_out, int aidx, cudaStream_t s);
// reference order <-> pencil layout (to_pen: out is zeroed first)
template <typename VT>
int pen_permute(Ctx &c, const VT *in, VT *out, bool to_pen, cudaStream_t s);
template <typename VT>
int launch_pen_regen(Ctx &c, int p, const VT *const *x, VT *const *y, const VT *const *rp,
                     const int *it, const double *bet, const double *alpha, cudaStream_t s);
// bdots_tc.cu: G (2*8*8 doubles, device, row-major 8 x 8 complex) = X^H Y of
// blocks of p <= 8 vectors on tcgen05 (int8 slices, exact int32 sums,
// double scaling); partial >= grid * 256 doubles, counter zeroed
int launch_bdots_tc(Ctx &c, int p, const double2 *const *x, const double2 *const *y, long n2,
                    double *partial, unsigned int *counter, int grid, double *G_dev,
                    cudaStream_t s);
int bdots_tc_grid(const Ctx &c, long n2);
// spmv_tile.cu: variant 3 (falls back to launch_spmv_async where it does not apply)
int launch_spmv_tile(Ctx &c, const double *x, double *y, double shift,
                     const double *xscale_dev, int scale_index, double *alpha_out,
                     int alpha_index, cudaStream_t s);
// caller-provided reduction scratch (noalloc.cu)
int launch_spmv_scratch(Ctx &c, const double *x, double *y, double shift, double *partial,
                        unsigned int *counter, int cap, double *dot_out, cudaStream_t s);
int launch_spmv_async_scratch(Ctx &c, const double *x, double *y, double shift,
                              double *partial, unsigned int *counter, int cap, double *dot_out,
                              cudaStream_t s);
// lanczos.cu
int ensure_partials(Ctx &c, int nblocks);
// y = F x (the folded operator) on double vectors in the reference's order
int fold_product(Ctx &c, const double *x, double *y, double *tmp, cudaStream_t s);
struct SolveArgs {
  int conv_start, conv_skip, imax, req1, req2;
  double emin1, emax1, emin2, emax2, tol;
  // restoreState: eigenvectors of restore_n values from a given tridiagonal
  // matrix of restore_its iterations (alpha[its], beta[its]), no first pass
  int restore_its = 0, restore_n = 0;
  const double *restore_alpha = nullptr, *restore_beta = nullptr,
               *restore_values = nullptr;
};
int solve(Ctx &c, const SolveArgs &A, const double *r0_dev, double *values, int *conv_iters,
          int *iterations, double *V_dev, int maxvec);
// lanczos.cu host pieces shared with the batched solve
struct Rng {  // uniform [0,1] starts for inverse iteration
  unsigned long long s;
  double next() {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return double(s >> 11) * (1.0 / 9007199254740992.0);
  }
};
bool inverse_iteration(int m, const double *d, const double *e, double lambda, Rng &rng,
                       std::vector<double> &x);
void check_window(int it, const double *al, const double *be, double emin, double emax,
                  double tol, double res, std::vector<double> &conv, std::vector<int> &conv_it,
                  unsigned long long seed);
// blk_lanczos.cu: double-precision Rayleigh-Ritz of nvec eigenvectors
// (vector e at V_dev + 2*e*stride doubles) over nseg independent segments
// [seg_off, seg_off + seg_len); values/resid/delta are [nseg][nvec]
int refine_ritz(Ctx &c, double *V_dev, int nvec, long stride, int nseg, const long *seg_off,
                const long *seg_len, double *values, double *resid, double *delta,
                cudaStream_t s, const int *seg_nvec = nullptr);

}  // namespace tbgpu
