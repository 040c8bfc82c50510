// tbgpu_hx_dot_noalloc: H*x with the fused dot product, allocating nothing.
//
// The regular entry points reduce the dot product through scratch that the
// context allocates with cudaMalloc the first time it is needed.  Some
// callers cannot have the library allocate at that point: applications that
// have handed the whole device memory to their own pool allocator (the
// Hamiltonian of a dot of tens of millions of atoms fills most of the HBM),
// and eigensolver loops that call H*x thousands of times and cannot accept
// the implicit device-wide synchronisation of cudaMalloc/cudaFree inside the
// loop.  This entry point
// takes the reduction scratch from a fixed array in this file instead.
//
// The scratch: kMaxBlocks (2048) block partials plus a completion counter,
// 16,640 bytes held on every device that loads the library, until the
// process exits.  A launch that would need more than 2048 blocks is refused
// with TBGPU_E_ARG: the 10-orbital models launch one block per SM at the
// Gamma point (one block per 24 atoms, at most 49,152 atoms, with a Bloch
// vector set); the 5-orbital models launch one block per 48 atoms, so at
// most 98,304 atoms.
//
// The array is shared by every call and keeps the last call's contents; the
// counter is cleared before each launch.  Calls that overlap on the GPU (from
// different streams or host threads) race on it and must be serialised by
// the caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current); that first call should
// come before any stream capture.
#include <mutex>

#include "tbgpu_internal.cuh"

namespace tbgpu {
namespace {

constexpr int kMaxBlocks = 2048;
constexpr int kMaxDevices = 64;

// [0, kMaxBlocks): block partials; the next 8 bytes: the completion counter
static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks + 32];

std::mutex g_setup_mutex;
double *g_scratch_dev[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (looked up once).
int scratch_address(int device, double **out) {
  if (device < 0 || device >= kMaxDevices) return set_error(TBGPU_E_ARG);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
      return set_error(TBGPU_E_CUDA);
    g_scratch_dev[device] = static_cast<double *>(p);
  }
  *out = g_scratch_dev[device];
  return TBGPU_OK;
}

}  // namespace
}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_hx_dot_noalloc(tbgpu_ctx *ctx, double shift, const double *x_dev,
                                    double *y_dev, double *dot_dev) {
  if (!ctx || !x_dev || !y_dev || !dot_dev || misaligned16(x_dev) || misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return set_error(TBGPU_E_CUDA);
  if (cur != c.device) return set_error(TBGPU_E_ARG);  // the context's device must be current
  double *scratch = nullptr;
  int rc = scratch_address(c.device, &scratch);
  if (rc) return rc;
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kMaxBlocks);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), c.stream) != cudaSuccess)
    return set_error(TBGPU_E_CUDA);
  return launch_spmv_scratch(c, x_dev, y_dev, shift, scratch, counter, kMaxBlocks, dot_dev,
                             c.stream);
}
