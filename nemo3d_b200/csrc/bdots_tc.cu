// Block dots G = X^H Y of two blocks of p <= 8 complex double vectors on the
// 5th-generation tensor cores (tcgen05), to double precision.
//
// The block Lanczos recurrence needs these p x p inner products every block
// step (lanczos_blk.c:150-219, 273-357: the block QR and Q^H W); the scalar
// kernel (k_bdots, blk_lanczos.cu) streams both blocks once and sums in
// double.  Here the same products run as an integer GEMM on tcgen05.mma
// kind::i8, exact in its int32 accumulator, and are scaled back in double:
//
//  * a CTA takes chunks of 256 vector entries.  Every real or imaginary part
//    of a vector (16 rows: re and im of 8 vectors, zero-padded) gets a shared
//    exponent per chunk (its largest |entry| = f * 2^e, 1/2 <= f < 1), and
//    each entry's mantissa m = x * 2^-e is cut into 8 signed 7-bit slices,
//    m = sum_s q_s 2^(-7(s+1)) + r, |q_s| <= 127, |r| < 2^-56 (all slices of
//    an entry carry its sign);
//  * the slices of X are the rows of A (8 slices x 16 rows = M = 128), those
//    of Y the rows of B (N = 128), K = the chunk's entries; one
//    M=128 x N=128 x K=32 MMA per 32 entries, 8 per chunk, accumulating every
//    slice product q_a q_b in TMEM (|sum| < 2^22, exact in int32);
//  * the four warps read the accumulator back (tcgen05.ld, one TMEM lane per
//    thread = one A row) and add, in double, the slice pairs with
//    s_a + s_b <= 7 scaled by 2^(e_a + e_b - 7(s_a + s_b + 2)).  Per entry
//    the 56-bit truncation costs < 2^-55 and the dropped pairs < 2^-53.2 of
//    2^(e_a + e_b) < 4 max|x| max|y| over the chunk: below 2^-50 of that
//    product of maxima, against a double dot's 2^-53 of each product plus
//    its sums' rounding (the double sums here round as the scalar kernel's);
//  * at the end each CTA sums its eight slice rows per output, writes its
//    16 x 16 real partial products, and the last CTA to finish adds all
//    partials in CTA order (deterministic) and forms
//    G_ij = (re re + im im) + i (re im - im re).
//
// Operands are written to shared memory by the threads in the K-major,
// no-swizzle canonical layout of 8-row x 16-byte core matrices (core matrix
// (row group g, K chunk c) at ((c * G) + g) * 128 bytes, G row groups), which
// the MMA's shared-memory descriptors describe (leading byte offset: the next
// 16-byte K chunk, G * 128; stride byte offset: the next 8-row group, 128).
// One thread issues the MMAs and commits them to an mbarrier; the wait on it
// is bounded: a wait that runs out reports TBGPU_E_TIMEOUT in the status
// word, waits once more, and the CTA stops, frees its TMEM and returns.
#include <algorithm>
#include <atomic>
#include <cstdint>

#include "tbgpu_internal.cuh"
#include "stage.cuh"

namespace tbgpu {

namespace {

constexpr int kTcP = 8;           // vectors per block (fewer are zero-padded)
constexpr int kSlices = 8;        // 7-bit slices of a 56-bit mantissa
constexpr int kRowsPerSlice = 16; // re and im rows of 8 vectors
constexpr int kM = kSlices * kRowsPerSlice;  // 128: A rows, TMEM lanes
constexpr int kN = kSlices * kRowsPerSlice;  // 128: B rows, accumulator columns
constexpr int kKC = 256;          // vector entries (K bytes) per chunk
constexpr int kThreads = 128;
constexpr int kGA = kM / 8, kGB = kN / 8;   // 8-row groups of A and B
constexpr int kBytesA = kM * kKC, kBytesB = kN * kKC;
constexpr int kTmemCols = 128;    // power of two >= kN
constexpr int kMaxSum = kSlices - 1;  // slice pairs kept: s_a + s_b <= 7

// byte offset of (row r, K byte k) in a canonical K-major no-swizzle tile
__device__ __forceinline__ uint32_t core_off(int r, int k, int G) {
  return uint32_t(((k >> 4) * G + (r >> 3)) * 128 + (r & 7) * 16 + (k & 15));
}

// shared-memory matrix descriptor: start address, leading byte offset (next
// 16-byte K chunk), stride byte offset (next 8-row group), version 1 (sm_100
// descriptors), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int G) {
  uint64_t d = uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(((G * 128) >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((128 >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// instruction descriptor of kind::i8: D s32, A and B signed 8-bit, both
// K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kN >> 3) << 17) |
                            (uint32_t(kM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

struct TcBlocks {
  const double2 *x[kTcP];
  const double2 *y[kTcP];
};

// 8 slices of the mantissas x * 2^-e of 16 consecutive entries, packed 16
// bytes per slice
__device__ __forceinline__ void slice16(const double (&v)[16], int e, uint4 (&out)[kSlices]) {
  uint32_t w[kSlices][4];
#pragma unroll
  for (int s = 0; s < kSlices; s++)
#pragma unroll
    for (int q = 0; q < 4; q++) w[s][q] = 0u;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    double m = ldexp(v[k], -e);  // |m| < 1, exact
#pragma unroll
    for (int s = 0; s < kSlices; s++) {
      const double t = m * 128.0;  // exact
      const double q = trunc(t);   // |q| <= 127
      m = t - q;                   // exact
      w[s][k >> 2] |= (uint32_t(int32_t(q)) & 0xFFu) << (8 * (k & 3));
    }
  }
#pragma unroll
  for (int s = 0; s < kSlices; s++) out[s] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}

// exponent e with max|v| = f 2^e, f in [0.5, 1); 0 for an all-zero part
__device__ __forceinline__ int part_exponent(double amax) {
  int e = 0;
  if (amax > 0.0) frexp(amax, &e);
  return e;
}

__global__ void __launch_bounds__(kThreads, 1)
    k_bdots_tc(long n2, int p, TcBlocks B, double *partial, unsigned int *counter,
               double *out, int *status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sA = smem;                 // kBytesA
  unsigned char *sB = smem + kBytesA;       // kBytesB
  __shared__ int eA[kRowsPerSlice], eB[kRowsPerSlice];
  __shared__ double red[4][kRowsPerSlice * kRowsPerSlice];
  __shared__ uint32_t tmem_base;
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ bool last;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t mb = stage::smem_addr(&mbar);
  // row of A (TMEM lane) this thread drains: slice, part, vector
  const int row = tid, s_a = row / kRowsPerSlice, rest = row % kRowsPerSlice;

  if (tid == 0) {
    stage::mbar_init(mb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     stage::smem_addr(&tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  double acc[kRowsPerSlice];  // this row's sums over the B rows (part, vector)
#pragma unroll
  for (int c = 0; c < kRowsPerSlice; c++) acc[c] = 0.0;

  // the loader: thread t takes vector t/16 of both blocks, entries 16*(t%16)..+15
  const int lv = tid / 16, lk = (tid % 16) * 16;
  const long nchunk = (n2 + kKC - 1) / kKC;
  uint32_t phase = 0;
  for (long ch = blockIdx.x; ch < nchunk; ch += gridDim.x) {
    const long base = ch * kKC + lk;
    double xr[16], xi[16], yr[16], yi[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
      if (lv < p && base + k < n2) {
        a = __ldg(B.x[lv] + base + k);
        b = __ldg(B.y[lv] + base + k);
      }
      xr[k] = a.x; xi[k] = a.y; yr[k] = b.x; yi[k] = b.y;
    }
    // per-part exponents over the chunk: 16 threads share a vector
    double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
      m0 = fmax(m0, fabs(xr[k])); m1 = fmax(m1, fabs(xi[k]));
      m2 = fmax(m2, fabs(yr[k])); m3 = fmax(m3, fabs(yi[k]));
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
      m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
    }
    const int exr = part_exponent(m0), exi = part_exponent(m1);
    const int eyr = part_exponent(m2), eyi = part_exponent(m3);
    if ((tid & 15) == 0) {
      eA[lv] = exr; eA[8 + lv] = exi;
      eB[lv] = eyr; eB[8 + lv] = eyi;
    }
    // slices into the canonical layout: row (slice s, part, vector)
    {
      uint4 sl[kSlices];
      slice16(xr, exr, sl);
#pragma unroll
      for (int s = 0; s < kSlices; s++)
        *reinterpret_cast<uint4 *>(sA + core_off(s * kRowsPerSlice + lv, lk, kGA)) = sl[s];
      slice16(xi, exi, sl);
#pragma unroll
      for (int s = 0; s < kSlices; s++)
        *reinterpret_cast<uint4 *>(sA + core_off(s * kRowsPerSlice + 8 + lv, lk, kGA)) = sl[s];
      slice16(yr, eyr, sl);
#pragma unroll
      for (int s = 0; s < kSlices; s++)
        *reinterpret_cast<uint4 *>(sB + core_off(s * kRowsPerSlice + lv, lk, kGB)) = sl[s];
      slice16(yi, eyi, sl);
#pragma unroll
      for (int s = 0; s < kSlices; s++)
        *reinterpret_cast<uint4 *>(sB + core_off(s * kRowsPerSlice + 8 + lv, lk, kGB)) = sl[s];
    }
    // the writes reach the tensor cores' (async) proxy; then one thread
    // issues the chunk's MMAs
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = stage::smem_addr(sA), b0 = stage::smem_addr(sB);
#pragma unroll
      for (int kk = 0; kk < kKC / 32; kk++)
        mma_i8(tmem, smem_desc(a0 + uint32_t(2 * kk * kGA * 128), kGA),
               smem_desc(b0 + uint32_t(2 * kk * kGB * 128), kGB), kk > 0 ? 1u : 0u);
      mma_commit(mb);
    }
    // bounded wait for the MMAs
    const bool done = stage::mbar_wait(mb, phase);
    if (!__syncthreads_and(done)) {
      if (tid == 0) {
        if (status) atomicExch(status, TBGPU_E_TIMEOUT);
      }
      stage::mbar_wait(mb, phase);  // once more for the MMAs in flight
      __syncthreads();
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // drain: this thread's TMEM lane (row) over the 128 columns, four
    // slices of B at a time
    const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
    const int ea = eA[rest];
#pragma unroll
    for (int h = 0; h < kSlices; h += 4) {
      uint32_t d[4][16];
#pragma unroll
      for (int q = 0; q < 4; q++) tmem_ld16(trow + uint32_t((h + q) * 16), d[q]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int s_b = h + q;
        if (s_a + s_b > kMaxSum) continue;
#pragma unroll
        for (int c = 0; c < kRowsPerSlice; c++)
          acc[c] += double(int32_t(d[q][c])) * ldexp(1.0, ea + eB[c] - 7 * (s_a + s_b + 2));
      }
    }
    // TMEM and shared memory are reused by the next chunk
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }

  // sum the eight slice rows of every (part, vector): lanes 16 apart in a
  // warp, then the four warps through shared memory
#pragma unroll
  for (int c = 0; c < kRowsPerSlice; c++) {
    double v = acc[c];
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    if (lane < 16) red[warp][lane * kRowsPerSlice + c] = v;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
  // this CTA's 16 x 16 real partial products, then the last CTA's sum
  for (int i = tid; i < kRowsPerSlice * kRowsPerSlice; i += kThreads)
    partial[size_t(blockIdx.x) * 256 + i] = red[0][i] + red[1][i] + red[2][i] + red[3][i];
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double tot[256];
  for (int i = tid; i < 256; i += kThreads) {
    double v = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) v += __ldcg(partial + size_t(b) * 256 + i);
    tot[i] = v;
  }
  __syncthreads();
  // G_ij = (xr.yr + xi.yi) + i (xr.yi - xi.yr); row (part, i), column (part, j)
  for (int t = tid; t < kTcP * kTcP; t += kThreads) {
    const int i = t / kTcP, j = t % kTcP;
    const double rr = tot[i * 16 + j], ii = tot[(8 + i) * 16 + 8 + j];
    const double ri = tot[i * 16 + 8 + j], ir = tot[(8 + i) * 16 + j];
    out[2 * t] = rr + ii;
    out[2 * t + 1] = ri - ir;
  }
  if (tid == 0) *counter = 0u;
}

}  // namespace

// G (row-major p x p complex, 2*p*p doubles, device) = X^H Y for blocks of
// p <= 8 vectors of n2 complex entries (x[i], y[j] device pointers), on the
// context's stream.  partial: >= grid*256 doubles, counter zeroed.
int launch_bdots_tc(Ctx &c, int p, const double2 *const *x, const double2 *const *y, long n2,
                    double *partial, unsigned int *counter, int grid, double *G_dev,
                    cudaStream_t s) {
  if (p < 1 || p > kTcP || n2 < 1 || grid < 1) return set_error(TBGPU_E_ARG);
  TcBlocks B{};
  for (int i = 0; i < kTcP; i++) {
    B.x[i] = i < p ? x[i] : x[0];
    B.y[i] = i < p ? y[i] : y[0];
  }
  constexpr int smem = kBytesA + kBytesB;
  static std::atomic<unsigned long long> attr_done{0};
  if (ensure_smem_attr(attr_done, c.device, k_bdots_tc, smem)) return TBGPU_E_CUDA;
  k_bdots_tc<<<grid, kThreads, smem, s>>>(n2, p, B, partial, counter, G_dev, c.d_status);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

// grid of the tensor-core block dots: one CTA per SM (each holds 128 TMEM
// columns and 64 kB of operand tiles), fewer for short vectors
int bdots_tc_grid(const Ctx &c, long n2) {
  const long chunks = (n2 + kKC - 1) / kKC;
  return int(std::max<long>(1, std::min<long>(chunks, long(c.sms))));
}

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_block_dots_dev(tbgpu_ctx *ctx, int p, const double *x_dev,
                                    const double *y_dev, long n2, double *G) {
  if (!ctx || p < 1 || p > kTcP || !x_dev || !y_dev || !G || n2 < 1 || misaligned16(x_dev) ||
      misaligned16(y_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  cudaStream_t s = c.stream;
  const double2 *xp[kTcP], *yp[kTcP];
  for (int i = 0; i < p; i++) {
    xp[i] = reinterpret_cast<const double2 *>(x_dev) + size_t(i) * n2;
    yp[i] = reinterpret_cast<const double2 *>(y_dev) + size_t(i) * n2;
  }
  double *d = nullptr, *part = nullptr;
  unsigned *cnt = nullptr;
  const int grid = bdots_tc_grid(c, n2);
  int rc = TBGPU_OK;
  if (cudaMalloc(&d, sizeof(double) * 2 * kTcP * kTcP) != cudaSuccess ||
      cudaMalloc(&cnt, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&part, sizeof(double) * 256 * size_t(grid)) != cudaSuccess)
    rc = set_error(TBGPU_E_NOMEM);
  if (!rc && cudaMemsetAsync(cnt, 0, sizeof(unsigned), s) != cudaSuccess) rc = set_error(TBGPU_E_CUDA);
  if (!rc) rc = launch_bdots_tc(c, p, xp, yp, n2, part, cnt, grid, d, s);
  double h[2 * kTcP * kTcP];
  if (!rc && (cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
              cudaStreamSynchronize(s) != cudaSuccess))
    rc = set_error(TBGPU_E_CUDA);
  if (!rc) rc = take_status(c);
  if (!rc)
    for (int i = 0; i < p; i++)
      for (int j = 0; j < p; j++) {
        G[2 * (i * p + j)] = h[2 * (i * kTcP + j)];
        G[2 * (i * p + j) + 1] = h[2 * (i * kTcP + j) + 1];
      }
  cudaFree(d);
  cudaFree(cnt);
  cudaFree(part);
  return rc;
}
