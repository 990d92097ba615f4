// Deterministic grid reductions: per-block partial sums, finished by the last block to arrive.
// A fixed grid adds the same partials in the same order on every run.
#pragma once

#include "femk_internal.cuh"

namespace femk {

template <int NV, int THREADS = 256>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* partials) {
  __shared__ double red[NV][THREADS / 32];
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) red[j][threadIdx.x >> 5] = v[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = 0.0;
      for (int w = 0; w < THREADS / 32; ++w) t += red[j][w];
      partials[(int64_t)blockIdx.x * NV + j] = t;
    }
  }
}

// Returns true in every thread of the last block to finish; `out` then holds the grid totals.
template <int NV, int THREADS = 256>
__device__ __forceinline__ bool grid_finish(double* partials, uint32_t* ticket, double (&out)[NV]) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double v[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = 0.0;
  // the partials of up to 4*THREADS blocks are loaded before any is added (one round trip)
  for (int b0 = threadIdx.x; b0 < (int)gridDim.x; b0 += 4 * THREADS) {
    double t[4][NV];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int b = b0 + u * THREADS;
#pragma unroll
      for (int j = 0; j < NV; ++j) t[u][j] = b < (int)gridDim.x ? __ldcg(partials + (int64_t)b * NV + j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < NV; ++j) v[j] += t[u][j];
  }
  __shared__ double red[NV][THREADS / 32];
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) red[j][threadIdx.x >> 5] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double t = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) t += red[j][w];
    out[j] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

}  // namespace femk
