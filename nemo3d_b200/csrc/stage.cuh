// Shared-memory staging helpers of the warp-staged H*x kernels
// (spmv_async.cu, spmm_async.cu): 16-byte cp.async copies, and the group
// metadata of the context's work order (up to three consecutive atoms of
// one k-pencil of cells per group).
#pragma once

#include <cstdint>

#include "tbgpu_internal.cuh"

namespace tbgpu {
namespace stage {

constexpr int kAPW = 3;  // atoms per warp (one lane per orbital, 10 orbitals)

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
// 16-byte copy that reads `bytes` (16 or 0) from global memory and fills the
// rest of the chunk with zeros: a missing neighbour costs no branch
__device__ __forceinline__ void cp16z(void *dst, const void *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 1-D bulk copies (cp.async.bulk, no multicast) complete on an mbarrier in
// the copying CTA's shared memory; waits on it are bounded.  A kernel whose
// wait runs out reports TBGPU_E_TIMEOUT, waits once more (bounded) and stops
// issuing copies; if the second wait also runs out, the CTA may end with
// that copy still in flight into its shared memory -- the one exit whose
// state is not guaranteed, and the status word says it happened.
constexpr long kWaitLimit = 1L << 20;  // mbarrier polls before giving up

__device__ __forceinline__ void mbar_init(uint32_t mb, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mb) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mb) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mb, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mb, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(mb), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase of the given parity; false when it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mb, uint32_t parity) {
  for (long polls = 0; polls < kWaitLimit; polls++)
    if (mbar_try_wait(mb, parity)) return true;
  return false;
}
// 1-D bulk copy global -> shared with completion on mbarrier mb (addresses
// and size multiples of 16 bytes)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t mb) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(mb)
      : "memory");
}

struct Meta {
  int nb[kAPW][4];
  int m[kAPW];  // -1: no atom
  int a0;       // first atom of the group
};

// Group g of the work order: up to three consecutive atoms of one pencil.
// skip (or null): per atom, 1 for atoms left out of the product (the atoms of
// a converged dot in a batched solve; a group lies in one dot).
__device__ __forceinline__ Meta load_meta(long g, long ngroups, const int2 *__restrict__ groups,
                                          const int4 *__restrict__ nbr,
                                          const unsigned char *__restrict__ site_m,
                                          const unsigned char *__restrict__ skip = nullptr) {
  Meta M;
  int2 e = make_int2(0, 0);
  if (g < ngroups) e = __ldg(groups + g);
  if (skip && g < ngroups && __ldg(skip + e.x)) e.y = 0;
  M.a0 = e.x;
#pragma unroll
  for (int i = 0; i < kAPW; i++) {
    const long a = long(e.x) + i;
    if (i < e.y) {
      const int4 v = __ldg(nbr + a);
      M.nb[i][0] = v.x; M.nb[i][1] = v.y; M.nb[i][2] = v.z; M.nb[i][3] = v.w;
      M.m[i] = __ldg(site_m + a);
    } else {
      M.nb[i][0] = M.nb[i][1] = M.nb[i][2] = M.nb[i][3] = -1;
      M.m[i] = -1;
    }
  }
  return M;
}

}  // namespace stage
}  // namespace tbgpu
