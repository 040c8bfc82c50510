// Deterministic grid-wide sum of one double per thread.
#pragma once

namespace tbgpu {

// Deterministic block + grid reduction of one double per thread: every block
// writes its partial, the last block to finish sums the partials in index
// order and writes out[idx].  No block waits on another.
template <int NT>
__device__ __forceinline__ void grid_reduce(double v, double *partial, unsigned int *counter,
                                            double *out, int idx, bool take_sqrt) {
  __shared__ double red[NT / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < NT / 32; i++) t += red[i];
    partial[blockIdx.x] = t;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += NT) t += __ldcg(partial + i);
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) red[w] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < NT / 32; i++) s += red[i];
    out[idx] = take_sqrt ? sqrt(s) : s;
    *counter = 0u;
  }
}

}  // namespace tbgpu
