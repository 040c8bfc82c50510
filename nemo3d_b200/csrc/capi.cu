// C ABI entry points of libtbgpu.so (declared in include/tbgpu.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "stage.cuh"
#include "tbgpu_internal.cuh"

namespace tbgpu {

static thread_local int g_last_error = TBGPU_OK;

int set_error(int code) {
  g_last_error = code;
  return code;
}

int take_status(Ctx &c) {
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return set_error(TBGPU_E_CUDA);
  int st = 0;
  if (cudaMemcpy(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(TBGPU_E_CUDA);
  if (!st) return TBGPU_OK;
  if (cudaMemset(c.d_status, 0, sizeof(int)) != cudaSuccess) return set_error(TBGPU_E_CUDA);
  return set_error(st);
}

// The solver's per-solve buffers (Lanczos rings, checkpoints, segment rings)
// come from one memory pool per device that keeps its memory mapped between
// solves: through a pool that returns memory at every synchronisation, the
// tens of gigabytes a large solve takes and gives back cost up to seconds of
// host time per solve, long enough to drain the work queued on the GPU.
namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices];
bool g_pool_made[kMaxPoolDevices];
bool g_pool_failed[kMaxPoolDevices];
}  // namespace

cudaMemPool_t solver_pool(int device) {
  if (device < 0 || device >= kMaxPoolDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_pool_made[device]) return g_pool[device];
  if (g_pool_failed[device]) return nullptr;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  unsigned long long keep = ~0ull;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess ||
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
    cudaGetLastError();
    if (pool) cudaMemPoolDestroy(pool);
    g_pool_failed[device] = true;  // the solver falls back to the default pool
    return nullptr;
  }
  g_pool[device] = pool;
  g_pool_made[device] = true;
  return pool;
}

size_t solver_pool_spare(int device) {
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (device < 0 || device >= kMaxPoolDevices || !g_pool_made[device]) return 0;
    pool = g_pool[device];
  }
  unsigned long long reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? size_t(reserved - used) : 0;
}


static int model_dims(int bm, int *norb, int *nspin) {
  switch (bm) {
    case TBGPU_SP3S: *norb = 5; *nspin = 1; return TBGPU_OK;
    case TBGPU_SP3S_SO: *norb = 5; *nspin = 2; return TBGPU_OK;
    case TBGPU_SP3D5S: *norb = 10; *nspin = 1; return TBGPU_OK;
    case TBGPU_SP3D5S_SO: *norb = 10; *nspin = 2; return TBGPU_OK;
    default: return TBGPU_E_ARG;
  }
}

static void free_ctx(Ctx *c) {
  if (!c) return;
  void *ptrs[] = {c->d_type, c->d_dsp, c->d_par, c->d_par_ok, c->d_site_index, c->d_atom_site,
                  c->d_nbr, c->d_site_m, c->d_surface, c->d_onsite, c->d_blocks, c->d_partial,
                  c->d_counter, c->d_status, c->d_x, c->d_y, c->d_phase, c->d_groups,
                  c->d_blocks32, c->d_onsite32, c->d_rc_order, c->d_units, c->d_start,
                  c->d_lane_tasks, c->d_pen_blk, c->d_pen_ons, c->d_pen_ok,
                  c->d_pen_scratch, c->d_fold_tmp};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

static int create(const tbgpu_geom *g, const tbgpu_model *m, bool dev, tbgpu_ctx **out) {
  if (!g || !m || !out || !g->type || !m->par || !m->par_ok) return set_error(TBGPU_E_ARG);
  *out = nullptr;
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || m->nspecies <= 0 || m->nspecies > 255)
    return set_error(TBGPU_E_ARG);
  Ctx *c = new (std::nothrow) Ctx();
  if (!c) return set_error(TBGPU_E_NOMEM);
  if (model_dims(m->band_model, &c->norb, &c->nspin)) {
    delete c;
    return set_error(TBGPU_E_ARG);
  }
  c->band_model = m->band_model;
  c->nb = c->norb * c->nspin;
  c->ons = onsite_len(c->nb);
  c->include_strain = m->include_strain;
  c->passivate = m->passivate;
  c->dangling_shift = m->dangling_shift;
  c->nspecies = m->nspecies;
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz;
  for (int d = 0; d < 3; d++) {
    c->periodic[d] = g->periodic[d] ? 1 : 0;
    c->lattice[d] = g->lattice[d];
  }
  c->nsites = long(g->nx) * g->ny * g->nz * 8;
  cudaGetDevice(&c->device);
  if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
      c->sms < 1) {
    delete c;
    return set_error(TBGPU_E_CUDA);
  }
  auto fail = [&](int code) {
    free_ctx(c);
    return set_error(code);
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(TBGPU_E_CUDA);
  c->own_stream = true;
  const size_t ns = size_t(c->nsites);
  const size_t npar = size_t(m->nspecies) * m->nspecies;
  if (cudaMalloc(&c->d_type, ns) != cudaSuccess) return fail(TBGPU_E_NOMEM);
  if (g->dsp && cudaMalloc(&c->d_dsp, ns * 3 * sizeof(double)) != cudaSuccess)
    return fail(TBGPU_E_NOMEM);
  if (cudaMalloc(&c->d_par, npar * kNPAR * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_par_ok, npar) != cudaSuccess ||
      cudaMalloc(&c->d_counter, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess)
    return fail(TBGPU_E_NOMEM);
  if (!dev) {  // species ids index the parameter table
    for (size_t i = 0; i < ns; i++)
      if (g->type[i] >= m->nspecies) return fail(TBGPU_E_ARG);
  }
  const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (cudaMemcpy(c->d_type, g->type, ns, kind) != cudaSuccess) return fail(TBGPU_E_CUDA);
  if (g->dsp && cudaMemcpy(c->d_dsp, g->dsp, ns * 3 * sizeof(double), kind) != cudaSuccess)
    return fail(TBGPU_E_CUDA);
  if (cudaMemcpy(c->d_par, m->par, npar * kNPAR * sizeof(double), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(c->d_par_ok, m->par_ok, npar, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(c->d_counter, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess)
    return fail(TBGPU_E_CUDA);
  *out = reinterpret_cast<tbgpu_ctx *>(c);
  return TBGPU_OK;
}

static Ctx *C(tbgpu_ctx *p) { return reinterpret_cast<Ctx *>(p); }
static const Ctx *C(const tbgpu_ctx *p) { return reinterpret_cast<const Ctx *>(p); }

}  // namespace tbgpu

using namespace tbgpu;

extern "C" {

int tbgpu_ctx_create(const tbgpu_geom *geom, const tbgpu_model *model, tbgpu_ctx **out) {
  return create(geom, model, false, out);
}

int tbgpu_ctx_create_dev(const tbgpu_geom *geom, const tbgpu_model *model, tbgpu_ctx **out) {
  return create(geom, model, true, out);
}

int tbgpu_ctx_destroy(tbgpu_ctx *ctx) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  Ctx *c = C(ctx);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_ctx(c);
  return TBGPU_OK;
}

int tbgpu_set_stream(tbgpu_ctx *ctx, void *stream) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  Ctx *c = C(ctx);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  c->own_stream = false;
  return TBGPU_OK;
}

int tbgpu_build_hamiltonian(tbgpu_ctx *ctx) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (c.built) return set_error(TBGPU_E_STATE);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c.stream);
  int rc = TBGPU_OK;
  if (!c.topo_built) {
    rc = build_topology(c);
    if (rc == TBGPU_OK) c.topo_built = true;
  }
  if (rc == TBGPU_OK) rc = assemble(c);
  if (rc == TBGPU_OK) rc = ensure_partials(c, int(c.natoms / 8 + 65536));
  cudaEventRecord(e1, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess && rc == TBGPU_OK) rc = set_error(TBGPU_E_CUDA);
  int st = 0;
  if (rc == TBGPU_OK && cudaMemcpy(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = set_error(TBGPU_E_CUDA);
  if (rc == TBGPU_OK && st != 0) rc = set_error(st);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  c.stats.build_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == TBGPU_OK) c.built = true;
  return rc;
}

long tbgpu_num_atoms(const tbgpu_ctx *ctx) { return ctx ? C(ctx)->natoms : -1; }

long tbgpu_dimension(const tbgpu_ctx *ctx) {
  return ctx ? C(ctx)->natoms * C(ctx)->nb : -1;
}

int tbgpu_hx_dev(tbgpu_ctx *ctx, double shift, const double *x_dev, double *y_dev) {
  if (!ctx || !x_dev || !y_dev || misaligned16(x_dev) || misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  return launch_spmv(c, x_dev, y_dev, shift, nullptr, 0, nullptr, 0, c.stream);
}

void tbgpu_matvect_mult_dev(const int **argList, double *y_dev, const double *x_dev) {
  set_error(TBGPU_OK);  // void entry point: status is read back via tbgpu_last_error
  if (!argList || !argList[0]) {
    set_error(TBGPU_E_ARG);
    return;
  }
  const double shift = argList[1] ? *reinterpret_cast<const double *>(argList[1]) : 0.0;
  tbgpu_hx_dev(reinterpret_cast<tbgpu_ctx *>(const_cast<int *>(argList[0])), shift, x_dev, y_dev);
}

int tbgpu_set_start_vector(tbgpu_ctx *ctx, const tbgpu_dcomplex *r_0) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!r_0) {
    if (c.d_start) cudaFree(c.d_start);
    c.d_start = nullptr;
    return TBGPU_OK;
  }
  if (!c.topo_built) return set_error(TBGPU_E_STATE);  // the dimension is known after the build
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  if (!c.d_start && cudaMalloc(&c.d_start, bytes) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  TB_CUDA(cudaMemcpyAsync(c.d_start, r_0, bytes, cudaMemcpyHostToDevice, c.stream));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  return TBGPU_OK;
}

int tbgpu_hx_dev_f32(tbgpu_ctx *ctx, double shift, const float *x_dev, float *y_dev) {
  if (!ctx || !x_dev || !y_dev || misaligned16(x_dev) || misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  return launch_spmv_f32(c, x_dev, y_dev, shift, nullptr, 0, nullptr, 0, c.stream);
}

void tbgpu_matvect_mult(const int **argList, tbgpu_dcomplex *y, const tbgpu_dcomplex *x) {
  set_error(TBGPU_OK);  // void entry point: status is read back via tbgpu_last_error
  if (!argList || !argList[0] || !x || !y) {
    set_error(TBGPU_E_ARG);
    return;
  }
  Ctx &c = *reinterpret_cast<Ctx *>(const_cast<int *>(argList[0]));
  const double shift = argList[1] ? *reinterpret_cast<const double *>(argList[1]) : 0.0;
  if (!c.built) {
    set_error(TBGPU_E_STATE);
    return;
  }
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  if (!c.d_x) {
    if (cudaMalloc(&c.d_x, bytes) != cudaSuccess || cudaMalloc(&c.d_y, bytes) != cudaSuccess) {
      set_error(TBGPU_E_NOMEM);
      return;
    }
  }
  if (cudaMemcpyAsync(c.d_x, x, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess) {
    set_error(TBGPU_E_CUDA);
    return;
  }
  if (launch_spmv(c, c.d_x, c.d_y, shift, nullptr, 0, nullptr, 0, c.stream)) return;
  if (cudaMemcpyAsync(y, c.d_y, bytes, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) {
    set_error(TBGPU_E_CUDA);
    return;
  }
  take_status(c);
}

namespace tbgpu {
namespace {
// One warp waits, with the bounded poll loop of the library's device-side
// waits, on an mbarrier that expects two arrivals and gets one: the wait
// runs out and the status word says so.
__global__ void k_selftest_wait(long polls, int *status) {
  __shared__ unsigned long long bar;
  const uint32_t mb = stage::smem_addr(&bar);
  if (threadIdx.x == 0) {
    stage::mbar_init(mb, 2);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (threadIdx.x == 0) stage::mbar_arrive(mb);
  bool done = false;
  for (long p = 0; p < polls && !done; p++) done = stage::mbar_try_wait(mb, 0);
  if (!__any_sync(0xffffffffu, done) && threadIdx.x == 0) atomicExch(status, TBGPU_E_TIMEOUT);
}
}  // namespace
}  // namespace tbgpu

int tbgpu_selftest_bounded_wait(tbgpu_ctx *ctx, long polls) {
  if (!ctx || polls < 1 || polls > (1L << 24)) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  k_selftest_wait<<<1, 32, 0, c.stream>>>(polls, c.d_status);
  TB_CUDA(cudaGetLastError());
  return take_status(c);
}

int tbgpu_eigensolve_lanczos_dev(tbgpu_ctx *ctx, int ConvCheckStartIter, int ConvCheckSkipRate,
                                 int imax, int requested1, int requested2, double emin1,
                                 double emax1, double emin2, double emax2, double tolerance,
                                 const double *r0_dev, double *values, int *conv_iterations,
                                 int *iterations, double *vectors_dev, int max_vectors) {
  if (!ctx || misaligned16(r0_dev) || misaligned16(vectors_dev)) return set_error(TBGPU_E_ARG);
  if (!r0_dev) r0_dev = C(ctx)->d_start;  // the vector set by tbgpu_set_start_vector
  if (!r0_dev) return set_error(TBGPU_E_ARG);
  SolveArgs A{ConvCheckStartIter, ConvCheckSkipRate, imax, requested1, requested2,
              emin1, emax1, emin2, emax2, tolerance};
  const int ne = solve(*C(ctx), A, r0_dev, values, conv_iterations, iterations, vectors_dev,
                       max_vectors);
  if (ne < 0) return ne;
  const int st = take_status(*C(ctx));
  return st ? st : ne;
}

int tbgpu_eigensolve_lanczos(tbgpu_ctx *ctx, int ConvCheckStartIter, int ConvCheckSkipRate,
                             int imax, int requested1, int requested2, double emin1,
                             double emax1, double emin2, double emax2, double tolerance,
                             const tbgpu_dcomplex *r_0, double *values, int *conv_iterations,
                             int *iterations, tbgpu_dcomplex *vectors, int max_vectors) {
  if (!ctx || (!r_0 && !C(ctx)->d_start)) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  // the device copies come from the solver's pool (kept mapped between
  // solves) and go back to it in stream order
  cudaStream_t s = c.stream;
  double *r0 = nullptr, *V = nullptr;
  const int nv = (vectors && max_vectors > 0) ? max_vectors : 0;
  if (nv && solver_alloc(c.device, &V, bytes * nv, s) != cudaSuccess) {
    cudaGetLastError();
    return set_error(TBGPU_E_NOMEM);
  }
  if (r_0 && solver_alloc(c.device, &r0, bytes, s) != cudaSuccess) {
    cudaGetLastError();
    if (V) cudaFreeAsync(V, s);
    return set_error(TBGPU_E_NOMEM);
  }
  int ne = TBGPU_OK;
  if (r_0 && cudaMemcpyAsync(r0, r_0, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
    ne = set_error(TBGPU_E_CUDA);
  // without r_0: the vector set by tbgpu_set_start_vector
  if (ne == TBGPU_OK)
    ne = tbgpu_eigensolve_lanczos_dev(ctx, ConvCheckStartIter, ConvCheckSkipRate, imax,
                                      requested1, requested2, emin1, emax1, emin2, emax2,
                                      tolerance, r0, values, conv_iterations, iterations, V, nv);
  if (ne > 0 && nv) {
    const int got = ne < nv ? ne : nv;
    if (cudaMemcpyAsync(vectors, V, bytes * got, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      ne = set_error(TBGPU_E_CUDA);
  }
  if (r0) cudaFreeAsync(r0, s);
  if (V) cudaFreeAsync(V, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && ne >= 0) ne = set_error(TBGPU_E_CUDA);
  return ne;
}

int tbgpu_eigenvectors_from_tridiagonal(tbgpu_ctx *ctx, int iterations, const double *alpha,
                                        const double *beta, int nvalues, const double *values,
                                        const tbgpu_dcomplex *r_0, tbgpu_dcomplex *vectors,
                                        int max_vectors) {
  if (!ctx || iterations < 2 || !alpha || !beta || nvalues < 1 || !values || !r_0 || !vectors ||
      max_vectors < 1)
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  const int nv = nvalues < max_vectors ? nvalues : max_vectors;
  double *r0 = nullptr, *V = nullptr;
  if (cudaMalloc(&r0, bytes) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
  if (cudaMalloc(&V, bytes * nv) != cudaSuccess) {
    cudaFree(r0);
    return set_error(TBGPU_E_NOMEM);
  }
  int rc = cudaMemcpyAsync(r0, r_0, bytes, cudaMemcpyHostToDevice, c.stream) == cudaSuccess
               ? TBGPU_OK
               : set_error(TBGPU_E_CUDA);
  std::vector<double> vals(values, values + nvalues), out(nvalues);
  std::sort(vals.begin(), vals.end());
  if (rc == TBGPU_OK) {
    SolveArgs A{0, 1, iterations + 1, 0, 0, 0.0, 0.0, 0.0, 0.0, 1e-7};
    A.restore_its = iterations;
    A.restore_n = nvalues;
    A.restore_alpha = alpha;
    A.restore_beta = beta;
    A.restore_values = vals.data();
    rc = solve(c, A, r0, out.data(), nullptr, nullptr, V, nv);
    if (rc > 0) {
      const int st = take_status(c);
      if (st) rc = st;
    }
  }
  if (rc > 0 && (cudaMemcpyAsync(vectors, V, bytes * nv, cudaMemcpyDeviceToHost, c.stream) !=
                     cudaSuccess ||
                 cudaStreamSynchronize(c.stream) != cudaSuccess))
    rc = set_error(TBGPU_E_CUDA);
  cudaFree(r0);
  cudaFree(V);
  return rc > 0 ? nv : rc;
}

int tbgpu_get_tridiagonal(const tbgpu_ctx *ctx, double *alpha, double *beta, int cap) {
  if (!ctx || !alpha || !beta) return set_error(TBGPU_E_ARG);
  const Ctx &c = *C(ctx);
  const int n = int(c.alpha.size()) < cap ? int(c.alpha.size()) : cap;
  for (int i = 0; i < n; i++) {
    alpha[i] = c.alpha[i];
    beta[i] = c.beta[i];
  }
  return n;
}

int tbgpu_export_pattern(const tbgpu_ctx *ctx, int *atom_site, int *nbr, unsigned char *surface) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  const Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t n = size_t(c.natoms);
  if ((atom_site && cudaMemcpy(atom_site, c.d_atom_site, n * sizeof(int), cudaMemcpyDeviceToHost)) ||
      (nbr && cudaMemcpy(nbr, c.d_nbr, n * sizeof(int4), cudaMemcpyDeviceToHost)) ||
      (surface && cudaMemcpy(surface, c.d_surface, n, cudaMemcpyDeviceToHost)))
    return set_error(TBGPU_E_CUDA);
  return TBGPU_OK;
}

int tbgpu_export_hamiltonian(const tbgpu_ctx *ctx, double *onsite, double *blocks) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  const Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t n = size_t(c.natoms);
  const int nb = c.nb, norb = c.norb;
  // the single-precision store is exported widened to double
  auto fetch = [&](double *dst, const double *src64, const float *src32, size_t count) -> bool {
    if (!c.ham_fp32)
      return cudaMemcpy(dst, src64, count * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
    std::vector<float> tmp(count);
    if (cudaMemcpy(tmp.data(), src32, count * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      return false;
    for (size_t i = 0; i < count; i++) dst[i] = tmp[i];
    return true;
  };
  if (blocks && c.recompute) {  // not stored: compute them for the export
    double *tmp = nullptr;
    const size_t cnt = n * 4 * norb * norb;
    if (cudaMalloc(&tmp, cnt * sizeof(double)) != cudaSuccess) return set_error(TBGPU_E_NOMEM);
    int rc = compute_blocks(const_cast<Ctx &>(c), tmp);
    if (!rc && (cudaStreamSynchronize(c.stream) != cudaSuccess ||
                cudaMemcpy(blocks, tmp, cnt * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
      rc = set_error(TBGPU_E_CUDA);
    cudaFree(tmp);
    if (rc) return rc;
  } else if (blocks && !fetch(blocks, c.d_blocks, c.d_blocks32, n * 4 * norb * norb)) {
    return set_error(TBGPU_E_CUDA);
  }
  if (!onsite) return TBGPU_OK;
  std::vector<double> rec(n * c.ons);
  if (!fetch(rec.data(), c.d_onsite, c.d_onsite32, rec.size())) return set_error(TBGPU_E_CUDA);
  std::memset(onsite, 0, sizeof(double) * n * nb * nb * 2);
  for (size_t a = 0; a < n; a++) {
    const double *r = rec.data() + a * c.ons;
    double *h = onsite + a * nb * nb * 2;
    auto re = [&](int i, int j) -> double & { return h[(i * nb + j) * 2]; };
    auto im = [&](int i, int j) -> double & { return h[(i * nb + j) * 2 + 1]; };
    for (int i = 0; i < nb; i++) re(i, i) = r[i];
    for (int sp = 0; sp < c.nspin; sp++) {
      const int o = sp * norb;
      re(o + 1, o + 2) += r[nb + 2]; re(o + 2, o + 1) += r[nb + 2];
      re(o + 1, o + 3) += r[nb + 3]; re(o + 3, o + 1) += r[nb + 3];
      re(o + 1, o + 4) += r[nb + 4]; re(o + 4, o + 1) += r[nb + 4];
      re(o + 2, o + 3) += r[nb + 5]; re(o + 3, o + 2) += r[nb + 5];
      re(o + 2, o + 4) += r[nb + 6]; re(o + 4, o + 2) += r[nb + 6];
      re(o + 3, o + 4) += r[nb + 7]; re(o + 4, o + 3) += r[nb + 7];
    }
    if (c.nspin == 2) {  // spin-orbit (mb_ham_spds_so.h)
      const double L = r[nb];
      const int u = 0, d = norb;
      im(u + 2, u + 3) += -L; im(u + 3, u + 2) += L;
      im(d + 2, d + 3) += L;  im(d + 3, d + 2) += -L;
      re(u + 2, d + 4) += L;  im(u + 3, d + 4) += -L;
      re(u + 4, d + 2) += -L; im(u + 4, d + 3) += L;
      re(d + 2, u + 4) += -L; im(d + 3, u + 4) += -L;
      re(d + 4, u + 2) += L;  im(d + 4, u + 3) += L;
    }
  }
  return TBGPU_OK;
}

int tbgpu_set_spmv_variant(tbgpu_ctx *ctx, int variant) {
  if (!ctx || variant < 0 || variant > 9) return set_error(TBGPU_E_ARG);
  C(ctx)->spmv_variant = variant;
  return TBGPU_OK;
}

// The variants that launch distinct kernels for this context: all seven for
// the 10-orbital models with the double store at the Gamma point; the
// warp-staged, the lane-gather, the lane-per-(atom, spin) and the pencil
// kernel with the float store; one kernel otherwise (5-orbital models, Bloch
// phases, recompute storage).
static int distinct_variants(const Ctx &c, int *v) {
  if (c.recompute) {
    v[0] = 0;
    return 1;
  }
  int n = 0;
  if (c.norb != 10 || c.bloch) {  // the lane-gather kernel at three block sizes
    v[n++] = 0;
  } else if (c.ham_fp32) {
    v[n++] = 0;
    v[n++] = 1;
    v[n++] = 5;
    v[n++] = 6;
    // the staged pencil kernel where it applies (otherwise 7 runs 6's)
    if (c.nspin == 2 && c.nz % 16 == 0 && !c.periodic[2]) v[n++] = 7;
  } else {
    for (int i = 0; i < 7; i++) v[n++] = i;
  }
  v[n++] = 8;
  v[n++] = 9;
  return n;
}

// Times the context's distinct H*x variants (the product with the fused
// alpha dot, as the Lanczos recurrence launches it; CUDA events on the
// context stream, two untimed launches first) and keeps the fastest (ties:
// the lower number).
int tbgpu_autotune_spmv(tbgpu_ctx *ctx, int reps, int *variant_out, double *ms_out) {
  if (!ctx || reps < 1 || reps > 1000) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  set_error(TBGPU_OK);
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  double *x = nullptr, *y = nullptr, *dot = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = TBGPU_OK;
  const int keep = c.spmv_variant;
  int best = keep;
  float best_ms = 0.0f;
  if (cudaMalloc(&x, bytes) != cudaSuccess || cudaMalloc(&y, bytes) != cudaSuccess ||
      cudaMalloc(&dot, sizeof(double)) != cudaSuccess) {
    rc = TBGPU_E_NOMEM;
  } else if (cudaMemsetAsync(x, 0, bytes, c.stream) != cudaSuccess ||
             cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = TBGPU_E_CUDA;
  }
  int cand[12];
  const int ncand = distinct_variants(c, cand);
  for (int ci = 0; ci < ncand && rc == TBGPU_OK; ci++) {
    const int v = cand[ci];
    c.spmv_variant = v;
    for (int r = 0; r < reps + 2 && rc == TBGPU_OK; r++) {
      if (r == 2 && cudaEventRecord(e0, c.stream) != cudaSuccess) rc = TBGPU_E_CUDA;
      if (rc == TBGPU_OK) rc = launch_spmv(c, x, y, 0.0, nullptr, 0, dot, 0, c.stream);
    }
    float ms = 0.0f;
    if (rc == TBGPU_OK && (cudaEventRecord(e1, c.stream) != cudaSuccess ||
                           cudaEventSynchronize(e1) != cudaSuccess ||
                           cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      rc = TBGPU_E_CUDA;
    ms /= float(reps);
    if (rc == TBGPU_OK && (ci == 0 || ms < best_ms)) {
      best = v;
      best_ms = ms;
    }
  }
  c.spmv_variant = rc == TBGPU_OK ? best : keep;
  if (c.spmv_variant != 3 && c.d_units) {  // the unit table only serves variant 3
    cudaFree(c.d_units);
    c.d_units = nullptr;
    c.nunits = 0;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(x);
  cudaFree(y);
  cudaFree(dot);
  if (rc) return set_error(rc);
  if (variant_out) *variant_out = best;
  if (ms_out) *ms_out = double(best_ms);
  return TBGPU_OK;
}

int tbgpu_set_ham_precision(tbgpu_ctx *ctx, int bits) {
  if (!ctx || (bits != 32 && bits != 64)) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (c.built) return set_error(TBGPU_E_STATE);
  c.ham_fp32 = bits == 32;
  return TBGPU_OK;
}

int tbgpu_set_ham_storage(tbgpu_ctx *ctx, int recompute) {
  if (!ctx || (recompute != 0 && recompute != 1)) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (c.built) return set_error(TBGPU_E_STATE);
  c.recompute = recompute == 1;
  return TBGPU_OK;
}

int tbgpu_set_lanczos_precision(tbgpu_ctx *ctx, int bits) {
  if (!ctx || (bits != 32 && bits != 64)) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (c.built) return set_error(TBGPU_E_STATE);
  c.lanczos_f32 = bits == 32;
  return TBGPU_OK;
}

int tbgpu_get_state_errors(const tbgpu_ctx *ctx, int cap, double *residual, double *delta) {
  if (!ctx || cap < 0) return set_error(TBGPU_E_ARG);
  const Ctx &c = *reinterpret_cast<const Ctx *>(ctx);
  const int n = std::min(cap, int(c.state_resid.size()));
  for (int i = 0; i < n; i++) {
    if (residual) residual[i] = c.state_resid[i];
    if (delta) delta[i] = c.state_delta[i];
  }
  return n;
}

int tbgpu_set_bloch_k(tbgpu_ctx *ctx, const double *k) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  for (int d = 0; d < 3; d++) c.kvec[d] = k ? k[d] : 0.0;
  const bool periodic = c.periodic[0] || c.periodic[1] || c.periodic[2];
  const bool nonzero = c.kvec[0] != 0.0 || c.kvec[1] != 0.0 || c.kvec[2] != 0.0;
  c.bloch = false;
  if (!periodic || !nonzero) return TBGPU_OK;  // Gamma point: no phases
  int rc = build_phases(c);
  if (rc) return rc;
  c.bloch = true;
  return TBGPU_OK;
}

int tbgpu_set_profiling(tbgpu_ctx *ctx, int on) {
  if (!ctx) return set_error(TBGPU_E_ARG);
  C(ctx)->profiling = on != 0;
  return TBGPU_OK;
}

int tbgpu_get_stats(const tbgpu_ctx *ctx, tbgpu_stats *out) {
  if (!ctx || !out) return set_error(TBGPU_E_ARG);
  *out = C(ctx)->stats;
  return TBGPU_OK;
}

int tbgpu_set_fold(tbgpu_ctx *ctx, int on, double shift1, double shift2, double factor,
                   double offset) {
  if (!ctx || (on != 0 && on != 1) || !std::isfinite(shift1) || !std::isfinite(shift2) ||
      !std::isfinite(factor) || !std::isfinite(offset) || factor == 0.0)
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  c.fold = on != 0;
  c.fold_s1 = shift1;
  c.fold_s2 = shift2;
  c.fold_factor = factor;
  c.fold_offset = offset;
  return TBGPU_OK;
}

int tbgpu_hx_fold_dev(tbgpu_ctx *ctx, const double *x_dev, double *y_dev) {
  if (!ctx || !x_dev || !y_dev || x_dev == y_dev || misaligned16(x_dev) || misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  if (!c.d_fold_tmp && cudaMalloc(&c.d_fold_tmp, bytes) != cudaSuccess)
    return set_error(TBGPU_E_NOMEM);
  return fold_product(c, x_dev, y_dev, c.d_fold_tmp, c.stream);
}

void tbgpu_matvect_mult2(const int **argList, tbgpu_dcomplex *y, const tbgpu_dcomplex *x) {
  set_error(TBGPU_OK);  // void entry point: status is read back via tbgpu_last_error
  if (!argList || !argList[0] || !x || !y) {
    set_error(TBGPU_E_ARG);
    return;
  }
  Ctx &c = *reinterpret_cast<Ctx *>(const_cast<int *>(argList[0]));
  if (!c.built) {
    set_error(TBGPU_E_STATE);
    return;
  }
  const size_t bytes = sizeof(double) * 2 * size_t(c.natoms) * c.nb;
  if ((!c.d_x && (cudaMalloc(&c.d_x, bytes) != cudaSuccess ||
                  cudaMalloc(&c.d_y, bytes) != cudaSuccess)) ||
      (!c.d_fold_tmp && cudaMalloc(&c.d_fold_tmp, bytes) != cudaSuccess)) {
    set_error(TBGPU_E_NOMEM);
    return;
  }
  if (cudaMemcpyAsync(c.d_x, x, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess) {
    set_error(TBGPU_E_CUDA);
    return;
  }
  if (fold_product(c, c.d_x, c.d_y, c.d_fold_tmp, c.stream)) return;
  if (cudaMemcpyAsync(y, c.d_y, bytes, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) {
    set_error(TBGPU_E_CUDA);
    return;
  }
  take_status(c);
}

int tbgpu_get_fold_energies(const tbgpu_ctx *ctx, int cap, double *energies) {
  if (!ctx || cap < 0 || (cap > 0 && !energies)) return set_error(TBGPU_E_ARG);
  const Ctx &c = *C(ctx);
  const int n = int(c.fold_energy.size());
  for (int i = 0; i < n && i < cap; i++) energies[i] = c.fold_energy[i];
  return n;
}

int tbgpu_set_eigenvector_pass(tbgpu_ctx *ctx, int mode, int columns, int segment) {
  if (!ctx || mode < 0 || mode > 1 || columns < 1 || columns > lane_max_cols(true) ||
      segment < 16 || segment > (1 << 20))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *C(ctx);
  c.vec_pass = mode;
  c.vec_columns = columns;
  c.vec_segment = segment;
  return TBGPU_OK;
}

int tbgpu_release_solver_memory(void) {
  int rc = TBGPU_OK;
  for (int d = 0; d < kMaxPoolDevices; d++) {
    cudaMemPool_t pool = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_pool_mu);
      if (g_pool_made[d]) pool = g_pool[d];
    }
    if (pool && cudaMemPoolTrimTo(pool, 0) != cudaSuccess) rc = set_error(TBGPU_E_CUDA);
  }
  return rc;
}

int tbgpu_set_mixed_acceptance(tbgpu_ctx *ctx, double floor) {
  if (!ctx || !(floor < 1.0) || !(floor > -HUGE_VAL)) return set_error(TBGPU_E_ARG);
  if (floor < 0.0) floor = -1.0;  // the automatic floor
  C(ctx)->mixed_accept = floor;
  return TBGPU_OK;
}

int tbgpu_set_block_dots(tbgpu_ctx *ctx, int mode) {
  if (!ctx || mode < 0 || mode > 1) return set_error(TBGPU_E_ARG);
  C(ctx)->block_dots = mode;
  return TBGPU_OK;
}

int tbgpu_last_error(void) { return g_last_error; }

const char *tbgpu_error_string(int code) {
  switch (code) {
    case TBGPU_OK: return "ok";
    case TBGPU_E_ARG: return "invalid argument";
    case TBGPU_E_CUDA: return "CUDA call failed";
    case TBGPU_E_NOMEM: return "device allocation failed";
    case TBGPU_E_MATERIAL: return "no material parameter set for a bond";
    case TBGPU_E_STATE: return "call out of order";
    case TBGPU_E_UNSUPPORTED: return "unsupported option";
    case TBGPU_E_NUMERIC: return "numerical breakdown";
    case TBGPU_E_TIMEOUT: return "a bounded device-side wait ran out";
    default: return "unknown error";
  }
}

}  // extern "C"
