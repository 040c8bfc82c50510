// Learned warm start of the Lanczos solve: the kernels of a small 3-D
// convolutional network (training and inference) and the two maps between a
// structure and the network's grid.  No counterpart in the reference, whose
// start vector comes from rand() or a file (eigen/src/lanczos.c:1823-1900);
// this replaces the random start through the same seam (the r_0 argument).
//
//   features      structure -> [3][G^3]: per coarse voxel the In fraction of
//                 the cation sites, the site occupancy and a strain proxy (the
//                 mean displacement length in units of 1 pm)
//   conv3d        3x3x3 convolution, zero padding, stride 1, activations in
//                 float [n][c][G^3], weights bf16 [cout][cin][27] with float
//                 accumulation; forward (optional ReLU on the output),
//                 backward to the input and to the weights and bias (the
//                 ReLU mask taken from the stored activation)
//   loss          mean squared envelope error plus a weighted squared error
//                 of sigma (the grid mean of the last output channel), with
//                 its gradient; or sigma alone for inference
//   adam          Adam step on the float master weights, bf16 copy refreshed
//   start vector  envelopes [k][G^3] and orbital profiles -> r_0: each atom's
//                 orbital o gets a uniform random number times
//                 sqrt(sum_k env_k(voxel)^2 prof_k(sublattice, o) + floor)
//
// Every reduction is deterministic (fixed order, no atomics on floats).
#include <cuda_bf16.h>

#include <cstdint>

#include "tbgpu_internal.cuh"

namespace tbgpu {

namespace {

constexpr int kConvThreads = 128;
constexpr int kCoGroup = 8;    // output (forward) or input (backward) channels per thread
constexpr int kMaxCh = 32;    // channels (the weights of a channel group stay in 48 KB of shared memory)
constexpr int kMaxGrid = 64;

__device__ __forceinline__ float bf(uint16_t w) {
  return __bfloat162float(__ushort_as_bfloat16(w));
}

// voxel of cell index i along an axis of n cells on a grid of G voxels
__host__ __device__ __forceinline__ int voxel_of(int i, int n, int G) {
  return int((long(i) * G) / n);
}
// first cell of voxel v (inverse of voxel_of)
__host__ __device__ __forceinline__ int first_cell(int v, int n, int G) {
  return int((long(v) * n + G - 1) / G);
}

__global__ void k_ws_features(int nx, int ny, int nz, int G, const unsigned char *type,
                              const double *dsp, int in_species, double scale, float *feat) {
  const long G3 = long(G) * G * G;
  const long v = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (v >= G3) return;
  const int vx = int(v / (G * G)), vy = int((v / G) % G), vz = int(v % G);
  const int i0 = first_cell(vx, nx, G), i1 = first_cell(vx + 1, nx, G);
  const int j0 = first_cell(vy, ny, G), j1 = first_cell(vy + 1, ny, G);
  const int k0 = first_cell(vz, nz, G), k1 = first_cell(vz + 1, nz, G);
  int ncat = 0, nin = 0, nocc = 0, nsite = 0;
  double dsum = 0.0;
  for (int i = i0; i < i1; i++)
    for (int j = j0; j < j1; j++)
      for (int k = k0; k < k1; k++)
        for (int m = 0; m < 8; m++) {
          const long s = ((long(i) * ny + j) * nz + k) * 8 + m;
          const int ty = type[s];
          nsite++;
          if (!ty) continue;
          nocc++;
          if (m < 4) {
            ncat++;
            nin += ty == in_species;
          }
          if (dsp) {
            const double dx = dsp[3 * s], dy = dsp[3 * s + 1], dz = dsp[3 * s + 2];
            dsum += sqrt(dx * dx + dy * dy + dz * dz);
          }
        }
  feat[v] = ncat ? float(nin) / float(ncat) : 0.0f;
  feat[G3 + v] = nsite ? float(nocc) / float(nsite) : 0.0f;
  feat[2 * G3 + v] = nocc ? float(dsum / nocc * scale) : 0.0f;
}

// out[n][co][p] = bias[co] + sum_ci sum_t w[co][ci][t] in[n][ci][p + off(t)]
// (thread: one voxel, kCoGroup output channels; the group's weights in
// shared memory as float)
__global__ void __launch_bounds__(kConvThreads)
    k_conv3d_fwd(const float *__restrict__ in, const uint16_t *__restrict__ w,
                 const float *__restrict__ bias, float *__restrict__ out, int cin, int cout,
                 int G, int relu) {
  extern __shared__ float ws[];  // [kCoGroup][cin][27]
  const int G3 = G * G * G;
  const int co0 = blockIdx.y * kCoGroup, n = blockIdx.z;
  const int nco = min(kCoGroup, cout - co0);
  for (int e = threadIdx.x; e < kCoGroup * cin * 27; e += blockDim.x) {
    const int c = e / (cin * 27);
    ws[e] = c < nco ? bf(w[(long(co0) * cin) * 27 + e]) : 0.0f;
  }
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= G3) return;
  const int x = p / (G * G), y = (p / G) % G, z = p % G;
  float acc[kCoGroup];
#pragma unroll
  for (int c = 0; c < kCoGroup; c++) acc[c] = 0.0f;
  for (int ci = 0; ci < cin; ci++) {
    const float *src = in + (long(n) * cin + ci) * G3;
    for (int t = 0; t < 27; t++) {
      const int xx = x + t / 9 - 1, yy = y + (t / 3) % 3 - 1, zz = z + t % 3 - 1;
      if (xx < 0 || xx >= G || yy < 0 || yy >= G || zz < 0 || zz >= G) continue;
      const float v = __ldg(src + (xx * G + yy) * G + zz);
#pragma unroll
      for (int c = 0; c < kCoGroup; c++) acc[c] = fmaf(ws[(c * cin + ci) * 27 + t], v, acc[c]);
    }
  }
  for (int c = 0; c < nco; c++) {
    float o = acc[c] + bias[co0 + c];
    if (relu) o = fmaxf(o, 0.0f);
    out[(long(n) * cout + co0 + c) * G3 + p] = o;
  }
}

// gradient through an optional ReLU: dout where the stored activation is
// positive
__device__ __forceinline__ float grad_at(const float *dout, const float *act, long idx) {
  const float g = __ldg(dout + idx);
  return act ? (__ldg(act + idx) > 0.0f ? g : 0.0f) : g;
}

// din[n][ci][p] = sum_co sum_t w[co][ci][t] g[n][co][p - off(t)]
__global__ void __launch_bounds__(kConvThreads)
    k_conv3d_bwd_data(const float *__restrict__ dout, const float *__restrict__ act,
                      const uint16_t *__restrict__ w, float *__restrict__ din, int cin, int cout,
                      int G) {
  extern __shared__ float ws[];  // [cout][kCoGroup][27]
  const int G3 = G * G * G;
  const int ci0 = blockIdx.y * kCoGroup, n = blockIdx.z;
  const int nci = min(kCoGroup, cin - ci0);
  for (int e = threadIdx.x; e < cout * kCoGroup * 27; e += blockDim.x) {
    const int co = e / (kCoGroup * 27), c = (e / 27) % kCoGroup, t = e % 27;
    ws[e] = c < nci ? bf(w[(long(co) * cin + ci0 + c) * 27 + t]) : 0.0f;
  }
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= G3) return;
  const int x = p / (G * G), y = (p / G) % G, z = p % G;
  float acc[kCoGroup];
#pragma unroll
  for (int c = 0; c < kCoGroup; c++) acc[c] = 0.0f;
  for (int co = 0; co < cout; co++) {
    const long base = (long(n) * cout + co) * G3;
    for (int t = 0; t < 27; t++) {
      const int xx = x - (t / 9 - 1), yy = y - ((t / 3) % 3 - 1), zz = z - (t % 3 - 1);
      if (xx < 0 || xx >= G || yy < 0 || yy >= G || zz < 0 || zz >= G) continue;
      const float g = grad_at(dout, act, base + (xx * G + yy) * G + zz);
#pragma unroll
      for (int c = 0; c < kCoGroup; c++) acc[c] = fmaf(ws[(co * kCoGroup + c) * 27 + t], g, acc[c]);
    }
  }
  for (int c = 0; c < nci; c++) din[(long(n) * cin + ci0 + c) * G3 + p] = acc[c];
}

// dw[co][ci][t] = sum_n sum_p g[n][co][p] in[n][ci][p + off(t)], and
// db[co] = sum_n sum_p g[n][co][p] (by the ci = 0 block); one block per
// (co, ci), block-order reduction
__global__ void __launch_bounds__(256)
    k_conv3d_bwd_weight(const float *__restrict__ in, const float *__restrict__ dout,
                        const float *__restrict__ act, float *__restrict__ dw,
                        float *__restrict__ db, int N, int cin, int cout, int G) {
  __shared__ float red[28][256 / 32];
  const int co = blockIdx.x / cin, ci = blockIdx.x % cin;
  const int G3 = G * G * G;
  float acc[28];
#pragma unroll
  for (int t = 0; t < 28; t++) acc[t] = 0.0f;
  for (int n = 0; n < N; n++) {
    const long gb = (long(n) * cout + co) * G3;
    const float *src = in + (long(n) * cin + ci) * G3;
    for (int p = threadIdx.x; p < G3; p += blockDim.x) {
      const float g = grad_at(dout, act, gb + p);
      if (g == 0.0f) continue;
      const int x = p / (G * G), y = (p / G) % G, z = p % G;
      acc[27] += g;
#pragma unroll
      for (int t = 0; t < 27; t++) {
        const int xx = x + t / 9 - 1, yy = y + (t / 3) % 3 - 1, zz = z + t % 3 - 1;
        if (xx < 0 || xx >= G || yy < 0 || yy >= G || zz < 0 || zz >= G) continue;
        acc[t] = fmaf(g, __ldg(src + (xx * G + yy) * G + zz), acc[t]);
      }
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 28; t++) {
    float v = acc[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[t][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 28) {
    float s = 0.0f;
    for (int i = 0; i < 256 / 32; i++) s += red[threadIdx.x][i];
    if (threadIdx.x < 27)
      dw[(long(co) * cin + ci) * 27 + threadIdx.x] = s;
    else if (ci == 0)
      db[co] = s;
  }
}

// Deterministic sum of v over a 256-thread block (result in every thread).
__device__ __forceinline__ float block_sum(float v, float *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = 0.0f;
  for (int i = 0; i < 8; i++) s += red[i];
  return s;
}

// One block.  sigma_pred[n] = mean_p out[n][K][p].  With targets: loss =
// mean over (n, k < K, p) of (out - env)^2 + w_sigma * mean_n (sigma_pred -
// sigma)^2, dout its gradient.
__global__ void __launch_bounds__(256)
    k_ws_loss(const float *__restrict__ out, const float *__restrict__ env,
              const float *__restrict__ sigma, int N, int K, int G, float w_sigma,
              float *__restrict__ dout, float *__restrict__ sigma_pred, float *__restrict__ loss) {
  __shared__ float red[8];
  const long G3 = long(G) * G * G;
  const float inv_env = 1.0f / float(long(N) * K * G3);
  float l = 0.0f;
  for (int n = 0; n < N; n++) {
    const float *o = out + long(n) * (K + 1) * G3;
    float s = 0.0f;
    for (long p = threadIdx.x; p < G3; p += blockDim.x) s += o[K * G3 + p];
    const float sp = block_sum(s, red) / float(G3);
    if (threadIdx.x == 0 && sigma_pred) sigma_pred[n] = sp;
    if (!env) continue;
    const float ds = 2.0f * w_sigma * (sp - sigma[n]) / float(N);
    if (threadIdx.x == 0) l += w_sigma * (sp - sigma[n]) * (sp - sigma[n]) / float(N);
    float *d = dout + long(n) * (K + 1) * G3;
    const float *t = env + long(n) * K * G3;
    for (long e = threadIdx.x; e < K * G3; e += blockDim.x) {
      const float diff = o[e] - t[e];
      d[e] = 2.0f * diff * inv_env;
      l += diff * diff * inv_env;
    }
    for (long p = threadIdx.x; p < G3; p += blockDim.x) d[K * G3 + p] = ds / float(G3);
  }
  if (env) {
    const float tot = block_sum(l, red);
    if (threadIdx.x == 0) *loss = tot;
  }
}

__global__ void k_ws_adam(float *w, uint16_t *wbf, const float *g, float *m, float *v, long n,
                          float lr_t, float b1, float b2, float eps) {
  const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr_t * mi / (sqrtf(vi) + eps);
  w[i] = wi;
  wbf[i] = __bfloat16_as_ushort(__float2bfloat16_rn(wi));
}

// r0[a][o] = u[a][o] * sqrt(sum_k env_k(voxel(a))^2 prof[k][sub(a)][o] + floor)
__global__ void k_ws_start(long natoms, int nb, int nx, int ny, int nz, int K, int G,
                           const int *__restrict__ atom_site, const float *__restrict__ env,
                           const float *__restrict__ prof, float floor_w,
                           const double2 *__restrict__ u, double2 *__restrict__ r0) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= natoms * nb) return;
  const long a = e / nb;
  const int o = int(e - a * nb);
  const long s = atom_site[a];
  const int m = int(s & 7);
  const long cell = s >> 3;
  const int k = int(cell % nz), j = int((cell / nz) % ny), i = int(cell / (long(nz) * ny));
  const long v = (long(voxel_of(i, nx, G)) * G + voxel_of(j, ny, G)) * G + voxel_of(k, nz, G);
  const long G3 = long(G) * G * G;
  const int sub = m < 4 ? 0 : 1;
  float w2 = floor_w;
  for (int q = 0; q < K; q++) {
    const float ev = env[q * G3 + v];
    w2 += ev * ev * prof[(q * 2 + sub) * nb + o];
  }
  const double f = sqrt(double(w2));
  const double2 uu = u[e];
  r0[e] = make_double2(uu.x * f, uu.y * f);
}

bool conv_args_ok(const void *a, const void *b, const void *c, int n, int cin, int cout, int G) {
  return a && b && c && n >= 1 && cin >= 1 && cin <= kMaxCh && cout >= 1 && cout <= kMaxCh &&
         G >= 1 && G <= kMaxGrid;
}

}  // namespace

}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_ws_features(tbgpu_ctx *ctx, int G, int in_species, float *feat_dev) {
  if (!ctx || !feat_dev || G < 1 || G > kMaxGrid) return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.d_type) return set_error(TBGPU_E_STATE);
  const long G3 = long(G) * G * G;
  // displacement lengths in pm
  k_ws_features<<<unsigned((G3 + 127) / 128), 128, 0, c.stream>>>(
      c.nx, c.ny, c.nz, G, c.d_type, c.d_dsp, in_species, 1000.0, feat_dev);
  TB_CUDA(cudaGetLastError());
  TB_CUDA(cudaStreamSynchronize(c.stream));
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_conv3d_fwd(const float *in_dev, const uint16_t *w_dev,
                                   const float *bias_dev, float *out_dev, int n, int cin,
                                   int cout, int G, int relu) {
  if (!conv_args_ok(in_dev, w_dev, out_dev, n, cin, cout, G) || !bias_dev)
    return set_error(TBGPU_E_ARG);
  const int G3 = G * G * G;
  dim3 grid((G3 + kConvThreads - 1) / kConvThreads, (cout + kCoGroup - 1) / kCoGroup, n);
  const size_t smem = sizeof(float) * kCoGroup * cin * 27;
  k_conv3d_fwd<<<grid, kConvThreads, smem>>>(in_dev, w_dev, bias_dev, out_dev, cin, cout, G, relu);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_conv3d_bwd_data(const float *dout_dev, const float *act_dev,
                                        const uint16_t *w_dev, float *din_dev, int n, int cin,
                                        int cout, int G) {
  if (!conv_args_ok(dout_dev, w_dev, din_dev, n, cin, cout, G)) return set_error(TBGPU_E_ARG);
  const int G3 = G * G * G;
  dim3 grid((G3 + kConvThreads - 1) / kConvThreads, (cin + kCoGroup - 1) / kCoGroup, n);
  const size_t smem = sizeof(float) * cout * kCoGroup * 27;
  k_conv3d_bwd_data<<<grid, kConvThreads, smem>>>(dout_dev, act_dev, w_dev, din_dev, cin, cout, G);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_conv3d_bwd_weight(const float *in_dev, const float *dout_dev,
                                          const float *act_dev, float *dw_dev, float *db_dev,
                                          int n, int cin, int cout, int G) {
  if (!conv_args_ok(in_dev, dout_dev, dw_dev, n, cin, cout, G) || !db_dev)
    return set_error(TBGPU_E_ARG);
  k_conv3d_bwd_weight<<<cout * cin, 256>>>(in_dev, dout_dev, act_dev, dw_dev, db_dev, n, cin,
                                           cout, G);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_loss(const float *out_dev, const float *env_dev, const float *sigma_dev,
                             int n, int k, int G, float w_sigma, float *dout_dev,
                             float *sigma_pred_dev, float *loss_dev) {
  if (!out_dev || n < 1 || k < 0 || k >= kMaxCh || G < 1 || G > kMaxGrid ||
      (env_dev && (!sigma_dev || !dout_dev || !loss_dev)) || (!env_dev && !sigma_pred_dev))
    return set_error(TBGPU_E_ARG);
  k_ws_loss<<<1, 256>>>(out_dev, env_dev, sigma_dev, n, k, G, w_sigma, dout_dev, sigma_pred_dev,
                        loss_dev);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_adam(float *w_dev, uint16_t *wbf_dev, const float *g_dev, float *m_dev,
                             float *v_dev, long n, float lr, float b1, float b2, float eps,
                             int step) {
  if (!w_dev || !wbf_dev || !g_dev || !m_dev || !v_dev || n < 1 || step < 1)
    return set_error(TBGPU_E_ARG);
  const float lr_t = float(lr * sqrt(1.0 - pow(double(b2), step)) / (1.0 - pow(double(b1), step)));
  k_ws_adam<<<unsigned((n + 255) / 256), 256>>>(w_dev, wbf_dev, g_dev, m_dev, v_dev, n, lr_t, b1,
                                                 b2, eps);
  TB_CUDA(cudaGetLastError());
  return TBGPU_OK;
}

extern "C" int tbgpu_ws_start_vector(tbgpu_ctx *ctx, const float *env_dev, const float *prof_dev,
                                     int k, int G, float floor_w, const double *u_dev,
                                     double *r0_dev) {
  if (!ctx || !env_dev || !prof_dev || !u_dev || !r0_dev || k < 1 || k > kMaxCh || G < 1 ||
      G > kMaxGrid || !(floor_w > 0.0f) || misaligned16(u_dev) || misaligned16(r0_dev))
    return set_error(TBGPU_E_ARG);
  Ctx &c = *reinterpret_cast<Ctx *>(ctx);
  if (!c.topo_built) return set_error(TBGPU_E_STATE);
  const long total = c.natoms * c.nb;
  k_ws_start<<<unsigned((total + 255) / 256), 256, 0, c.stream>>>(
      c.natoms, c.nb, c.nx, c.ny, c.nz, k, G, c.d_atom_site, env_dev, prof_dev, floor_w,
      reinterpret_cast<const double2 *>(u_dev), reinterpret_cast<double2 *>(r0_dev));
  TB_CUDA(cudaGetLastError());
  TB_CUDA(cudaStreamSynchronize(c.stream));
  return TBGPU_OK;
}
