// Grid-wide barrier and reductions for persistent (cooperatively launched) solver kernels.
//
// The barrier is a counter plus a generation word in device memory. Every block's thread 0 adds
// one to the counter with acquire-release semantics (releasing its block's writes before the
// barrier; the last arriver acquires everyone else's); the last one resets it and publishes the
// next generation with a release store; the others poll the generation with acquire loads. So
// after the barrier every block sees the other blocks' writes, also through plain loads. Each wait is bounded by a clock64 budget (checked every 256 polls, with the
// timeout word): a block that runs out of budget raises the timeout word and returns false, every
// other waiting block sees the word and returns false too, and the kernel unwinds with
// FEMK_TIMEOUT instead of hanging. A cooperative launch guarantees all blocks are resident, so the
// budget (the plan's barrier_limit_ms, 2 s by default) is never reached in a correct run. Measured
// on B200 with 296 blocks: 2.0 us per barrier (2.96 us with a fence, a relaxed add and 40 ns sleeps
// between polls).
//
// Reductions are redundant instead of serial: every block writes its partial, crosses the
// barrier, and then sums all partials itself in the same fixed order, so each block holds the
// same bit-identical total without a second barrier or a designated finishing block.
#pragma once

#include <stdint.h>

namespace femk {

struct GridBar {
  unsigned int count;
  unsigned int gen;
  unsigned int timeout;
  unsigned int pad;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// All threads of every block call this. `gen` is the caller's generation counter (kept by
// thread 0; starts at 0 for a freshly zeroed GridBar). `limit` bounds the wait in clock64 cycles.
// Returns false once any block timed out. The block numbered `skip` does not arrive at the first
// barrier (gen == 0): that is how a test makes every other block wait out its limit (the plan's
// test_skip_arrival option; -1 in every other launch).
__device__ __forceinline__ bool grid_sync(GridBar* bar, unsigned int& gen, long long limit, int skip = -1) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int target = gen + 1;
    const bool arrive = !(gen == 0u && (int)blockIdx.x == skip);
    unsigned int old = 0;
    if (arrive)
      asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(&bar->count) : "memory");
    if (arrive && old == gridDim.x - 1) {
      bar->count = 0u;  // ordered before the release below; the next arrivals follow its acquire
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&bar->gen), "r"(target) : "memory");
    } else {
      const long long t0 = clock64();
      unsigned int polls = 0;
      while (ld_acquire_u32(&bar->gen) != target) {
        if ((++polls & 255u) == 0u && (ld_acquire_u32(&bar->timeout) != 0u || clock64() - t0 > limit)) {
          atomicExch(&bar->timeout, 1u);
          ok = 0;
          break;
        }
      }
    }
    gen = target;
    ok_s = ok && ld_acquire_u32(&bar->timeout) == 0u;
  }
  __syncthreads();
  return ok_s != 0;
}

// Block sum of NV values; thread 0 stores them to partials[j * gridDim.x + blockIdx.x].
template <int NV, int THREADS>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* __restrict__ partials) {
  __shared__ double red[NV][THREADS / 32];
#pragma unroll
  for (int j = 0; j < NV; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
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
      partials[(int64_t)j * gridDim.x + blockIdx.x] = t;
    }
  }
}

// After a grid_sync: every block sums all partials in the same order (warp 0), result broadcast.
template <int NV>
__device__ __forceinline__ void grid_totals(const double* __restrict__ partials, double (&out)[NV]) {
  __shared__ double tot_s[NV];
  if (threadIdx.x < 32) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = 0.0;
      for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) t += __ldcg(partials + (int64_t)j * gridDim.x + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) tot_s[j] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) out[j] = tot_s[j];
  __syncthreads();
}

}  // namespace femk
