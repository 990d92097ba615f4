// Mixed-precision Jacobi-PCG: FP32 values, vectors and SpMV accumulation in the inner CG; FP64
// solution and FP64 true residual r = b - A x (FP64 values) at every reliable update.
//
// Inner step (FP32):  q = A32 p;  alpha = gamma / <p, q>;  e += alpha p;  r -= alpha q;  z = D^-1 r;
//                     p = z + beta p
// A reliable update is requested when <r, r> fell below delta^2 of its value at the previous
// update, when the FP32 recurrence meets the stop test, or at the iteration cap. The iterations
// left in the current chunk then return at entry, and the chunk ends with
//     x += e;  e = 0;  r64 = b - A64 x;  r = fp32(r64);  z = D^-1 r;  gamma = <r, z>;  p = z + beta p
// which keeps the search direction (FEMK_MIXED_RELIABLE, residual replacement) or restarts it
// with beta = 0 (FEMK_MIXED_RESTART, classic iterative refinement). The solve stops only on the
// FP64 true residual: <r64, r64> <= max(tol^2 <b, b>, atol^2) -- the stop rule of femk_pcg.
//
// The FP32 operator is the plan's sliced-ELL copy: 4 B value + 2 B column offset (int16,
// col - row) per entry when the bandwidth allows it, else 4 B + 4 B. Each chunk (16 iterations,
// 3 kernels each, plus the 3 update kernels) is replayed as one CUDA graph.
//
// No reference counterpart: jNO runs x64 throughout (tests/test_fem_3d.py:37-46).
#include <algorithm>
#include <cmath>

#include "femk_internal.cuh"
#include "femk_spmv.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;

struct MixedState {
  double gamma, rr, rr64, bb, atol2, alpha, beta, rr_since, delta2;
  int32_t iter, maxiter, done, status;
  int32_t need_update;  // 1: update requested this chunk; 2: update done, direction pending
  int32_t hold;         // iterations return at entry until the chunk-end update
  int32_t outer, restart;
  uint32_t ticket;
};

template <int NV>
__device__ __forceinline__ bool reduce_finish(double (&v)[NV], double* partials, uint32_t* ticket, double (&out)[NV]) {
  __shared__ double red[NV][kThreads / 32];
  __shared__ bool last;
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
      for (int w = 0; w < kThreads / 32; ++w) t += red[j][w];
      partials[(int64_t)blockIdx.x * NV + j] = t;
    }
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) s[j] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads)
#pragma unroll
    for (int j = 0; j < NV; ++j) s[j] += __ldcg(partials + (int64_t)b * NV + j);
#pragma unroll
  for (int j = 0; j < NV; ++j) s[j] = warp_sum(s[j]);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) red[j][threadIdx.x >> 5] = s[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[j][w];
    out[j] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

__global__ void k_demote(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void k_fill_f(float* __restrict__ v, int64_t n, float val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = val;
}

__global__ void k_gather32(const int32_t* __restrict__ src, int64_t m, const double* __restrict__ vals,
                           float* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = __ldcs(src + j);
    out[j] = k >= 0 ? (float)__ldcs(vals + k) : 0.f;
  }
}

__device__ __forceinline__ void finish_alpha(MixedState* st, double pq) {
  st->alpha = st->gamma / pq;
  st->need_update = 0;  // a pending direction update was applied before this step
  if (!isfinite(pq)) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(pq > 0.0)) {
    st->status = FEMK_BREAKDOWN;
    st->done = 1;
  }
}

// q = A32 p, <p, q> -> alpha (sliced-ELL operator)
template <typename IDX>
__global__ void __launch_bounds__(kThreads) k_step32_sell(const int64_t* __restrict__ sptr, const IDX* __restrict__ cols,
                                                         const float* __restrict__ vals, int64_t n, int64_t nslices,
                                                         const float* __restrict__ p, float* __restrict__ q,
                                                         double* __restrict__ partials, MixedState* st) {
  if (st->done || st->hold) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  float acc = 0.f;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    if (row >= n) continue;
    const int64_t b0 = __ldg(sptr + sl);
    const int32_t w = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
    const float sv = sell_row(vals, cols, b0 + lane, w, row, GatherX<float>{p});
    q[row] = sv;
    acc = fmaf(__ldg(p + row), sv, acc);
  }
  double v[1] = {(double)acc}, tot[1];
  if (!reduce_finish<1>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  finish_alpha(st, tot[0]);
}

// the same step on the CSR copy (plans without a sliced-ELL layout)
template <int L, int U, typename IDX>
__global__ void __launch_bounds__(kThreads) k_step32(const int32_t* __restrict__ indptr, const IDX* __restrict__ cols,
                                                    const float* __restrict__ vals, int64_t n, const float* __restrict__ p,
                                                    float* __restrict__ q, double* __restrict__ partials, MixedState* st) {
  if (st->done || st->hold) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  float acc = 0.f;
  for (int64_t base = warp * RPW * U; base < n; base += nwarps * RPW * U) {
    float sv[U];
    int64_t rows[U];
    csr_rows<L, U, float, IDX>(indptr, cols, vals, p, n, base, lane, sv, rows);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (rows[u] >= n || sub != 0) continue;
      q[rows[u]] = sv[u];
      acc = fmaf(__ldg(p + rows[u]), sv[u], acc);
    }
  }
  double v[1] = {(double)acc}, tot[1];
  if (!reduce_finish<1>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  finish_alpha(st, tot[0]);
}

// e += alpha p; r -= alpha q; z = D^-1 r; <r, z>, <r, r>; request a reliable update or set beta
__global__ void __launch_bounds__(kThreads) k_update32(int64_t n, float* __restrict__ e, float* __restrict__ r,
                                                      float* __restrict__ z, const float* __restrict__ p,
                                                      const float* __restrict__ q, const float* __restrict__ dinv,
                                                      double* __restrict__ partials, MixedState* st) {
  if (st->done || st->hold) return;
  const float alpha = (float)st->alpha;
  float a0 = 0.f, a1 = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const float pi = p[i];
    e[i] = fmaf(alpha, pi, e[i]);
    const float ri = fmaf(-alpha, q[i], r[i]);
    const float zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    a0 = fmaf(ri, zi, a0);
    a1 = fmaf(ri, ri, a1);
  }
  double v[2] = {(double)a0, (double)a1}, tot[2];
  if (!reduce_finish<2>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  st->iter += 1;
  st->rr = tot[1];
  if (!isfinite(tot[0]) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
    return;
  }
  const bool conv = !(tot[1] > st->atol2);
  const bool drop = tot[1] < st->delta2 * st->rr_since;
  if (conv || drop || st->iter >= st->maxiter) {
    st->need_update = 1;
    st->hold = 1;
  } else {
    st->beta = tot[0] / st->gamma;
    st->gamma = tot[0];
  }
}

// x += e; e = 0 (only at a requested update)
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ e, const MixedState* st) {
  if (st->done || st->need_update != 1) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += (double)e[i];
    e[i] = 0.f;
  }
}

// r64 = b - A64 x; r = fp32(r64); z = D^-1 r; <r, z>, <r64, r64> (+ <b, b> and p = z at init)
template <int L, int U, bool INIT>
__global__ void __launch_bounds__(kThreads) k_true_resid(const int32_t* __restrict__ indptr,
                                                        const int32_t* __restrict__ indices,
                                                        const double* __restrict__ vals, int64_t n,
                                                        const double* __restrict__ x, const double* __restrict__ b,
                                                        const float* __restrict__ dinv, float* __restrict__ r,
                                                        float* __restrict__ z, float* __restrict__ p,
                                                        double* __restrict__ partials, MixedState* st, double tol2,
                                                        double atol2) {
  if (!INIT && (st->done || st->need_update != 1)) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t base = warp * RPW * U; base < n; base += nwarps * RPW * U) {
    double sv[U];
    int64_t rows[U];
    csr_rows<L, U, double, int32_t>(indptr, indices, vals, x, n, base, lane, sv, rows);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t row = rows[u];
      if (row >= n || sub != 0) continue;
      const double bi = b[row];
      const double r64 = bi - sv[u];
      const float rf = (float)r64;
      const float zf = dinv[row] * rf;
      r[row] = rf;
      z[row] = zf;
      if (INIT) p[row] = zf;
      a0 += (double)rf * (double)zf;
      a1 += r64 * r64;
      if (INIT) a2 += bi * bi;
    }
  }
  double v[3] = {a0, a1, a2}, tot[3];
  if (!reduce_finish<3>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  st->outer += 1;
  st->rr64 = tot[1];
  st->rr_since = tot[1];
  if (INIT) {
    st->bb = tot[2];
    st->atol2 = fmax(tol2 * tot[2], atol2);
    st->gamma = tot[0];
    st->iter = 0;
    st->need_update = 0;
    st->hold = 0;
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    st->done = (!(tot[1] > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
    return;
  }
  if (!isfinite(tot[0]) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
    return;
  }
  if (!(tot[1] > st->atol2) || st->iter >= st->maxiter) {
    st->done = 1;
    return;
  }
  st->beta = st->restart ? 0.0 : tot[0] / st->gamma;
  st->gamma = tot[0];
  st->need_update = 2;
  st->hold = 0;
}

// p = z + beta p: every iteration (MODE 0, skipped while held) or after a chunk-end update (MODE 1)
template <int MODE>
__global__ void k_pupdate32(int64_t n, float* __restrict__ p, const float* __restrict__ z, const MixedState* st) {
  if (st->done) return;
  if (MODE == 0 && st->hold) return;
  if (MODE == 1 && st->need_update != 2) return;
  const float beta = (float)st->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fmaf(beta, p[i], z[i]);
}

template <bool INIT>
void launch_true_resid(const femk_plan* p, const double* vals, const double* x, const double* b, const float* dinv,
                       float* r, float* z, float* pv, MixedState* st, double tol2, double atol2, cudaStream_t s) {
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    const int grid = wave_grid(k_true_resid<L, U, INIT>, kThreads, p);
    k_true_resid<L, U, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
        p->indptr, p->indices, vals, p->n, x, b, dinv, r, z, pv, p->partials, st, tol2, atol2);
  });
}

void launch_step32(const femk_plan* p, const float* pv, float* q, MixedState* st, cudaStream_t s) {
  if (p->sell_vals32) {
    if (p->sell_c16) {
      k_step32_sell<int16_t><<<::femk::counted_launch() + wave_grid(k_step32_sell<int16_t>, kThreads, p), kThreads, 0,
                               s>>>(p->sell_ptr, p->sell_c16, p->sell_vals32, p->n, p->n_slices, pv, q, p->partials, st);
    } else {
      k_step32_sell<int32_t><<<::femk::counted_launch() + wave_grid(k_step32_sell<int32_t>, kThreads, p), kThreads, 0,
                               s>>>(p->sell_ptr, p->sell_cols, p->sell_vals32, p->n, p->n_slices, pv, q, p->partials,
                                    st);
    }
    return;
  }
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    if (p->cols16) {
      k_step32<L, U, int16_t><<<::femk::counted_launch() + wave_grid(k_step32<L, U, int16_t>, kThreads, p), kThreads,
                                0, s>>>(p->indptr, p->cols16, p->vals32, p->n, pv, q, p->partials, st);
    } else {
      k_step32<L, U, int32_t><<<::femk::counted_launch() + wave_grid(k_step32<L, U, int32_t>, kThreads, p), kThreads,
                                0, s>>>(p->indptr, p->indices, p->vals32, p->n, pv, q, p->partials, st);
    }
  });
}

struct MixedPtrs {
  float *r, *z, *pv, *q, *e, *d32;
  MixedState* st;
};

MixedPtrs mixed_ptrs(const femk_plan* p) {
  const int64_t n = p->n;
  MixedPtrs m;
  m.r = p->work32;
  m.z = m.r + n;
  m.pv = m.z + n;
  m.q = m.pv + n;
  m.e = m.q + n;
  m.d32 = m.e + n;
  m.st = (MixedState*)p->work64b;
  return m;
}

// one chunk: kChunk inner iterations, then the (conditional) reliable update
int enqueue_mixed_chunk(const femk_plan* p, const double* vals, const double* b, double* x, cudaStream_t s) {
  const MixedPtrs m = mixed_ptrs(p);
  const int64_t n = p->n;
  for (int it = 0; it < kChunk; ++it) {
    launch_step32(p, m.pv, m.q, m.st, s);
    k_update32<<<::femk::counted_launch() + wave_grid(k_update32, kThreads, p), kThreads, 0, s>>>(
        n, m.e, m.r, m.z, m.pv, m.q, m.d32, p->partials, m.st);
    k_pupdate32<0><<<::femk::counted_launch() + wave_grid(k_pupdate32<0>, 256, p), 256, 0, s>>>(n, m.pv, m.z, m.st);
  }
  k_fold<<<::femk::counted_launch() + wave_grid(k_fold, 256, p), 256, 0, s>>>(n, x, m.e, m.st);
  launch_true_resid<false>(p, vals, x, b, m.d32, m.r, m.z, nullptr, m.st, 0.0, 0.0, s);
  k_pupdate32<1><<<::femk::counted_launch() + wave_grid(k_pupdate32<1>, 256, p), 256, 0, s>>>(n, m.pv, m.z, m.st);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int ensure_mixed(femk_plan* p) {
  FEMK_TRY(ensure_workspace(p));
  if (!p->work32) FEMK_CUDA_TRY(cudaMalloc(&p->work32, sizeof(float) * 6 * (p->n + 1)));
  if (p->use_sell && p->sell_src) {
    if (!p->sell_vals32) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals32, sizeof(float) * (p->sell_nnz + 1)));
  } else if (!p->vals32) {
    FEMK_CUDA_TRY(cudaMalloc(&p->vals32, sizeof(float) * (p->nnz + 1)));
  }
  if (!p->work64b) FEMK_CUDA_TRY(cudaMalloc(&p->work64b, sizeof(MixedState) + 64));
  if (!p->mx_stream) {
    FEMK_CUDA_TRY(cudaStreamCreateWithFlags(&p->mx_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 3; ++i) FEMK_CUDA_TRY(cudaEventCreateWithFlags(&p->mx_ev[i], cudaEventDisableTiming));
    FEMK_CUDA_TRY(cudaMallocHost(&p->mx_host, 2 * sizeof(MixedState)));
  }
  return FEMK_OK;
}

int ensure_mixed_graph(femk_plan* p, const double* vals, const double* b, double* x) {
  // every buffer the captured kernels read is allocated by ensure_mixed before this point
  if (!p->work32 || !p->work64b || !(p->sell_vals32 || p->vals32)) {
    set_error("femk_pcg_mixed: workspace missing at graph capture");
    return FEMK_EINVAL;
  }
  const void* key[4] = {vals, b, x, p->sell_vals32 ? (const void*)p->sell_vals32 : (const void*)p->vals32};
  bool same = p->mx_exec != nullptr;
  for (int i = 0; i < 4; ++i) same = same && key[i] == p->mx_key[i];
  if (same) return FEMK_OK;
  // occupancy queries happen before capture begins
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    (void)wave_grid(k_true_resid<L, U, false>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int16_t>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int32_t>, kThreads, p);
  });
  (void)wave_grid(k_step32_sell<int16_t>, kThreads, p);
  (void)wave_grid(k_step32_sell<int32_t>, kThreads, p);
  (void)wave_grid(k_update32, kThreads, p);
  (void)wave_grid(k_pupdate32<0>, 256, p);
  (void)wave_grid(k_pupdate32<1>, 256, p);
  (void)wave_grid(k_fold, 256, p);
  cudaGraph_t g = nullptr;
  set_capturing(true);
  cudaError_t e = cudaStreamBeginCapture(p->mx_stream, cudaStreamCaptureModeThreadLocal);
  int st = e == cudaSuccess ? enqueue_mixed_chunk(p, vals, b, x, p->mx_stream) : FEMK_ECUDA;
  const cudaError_t e2 = cudaStreamEndCapture(p->mx_stream, &g);
  set_capturing(false);
  if (e != cudaSuccess || e2 != cudaSuccess || st != FEMK_OK) {
    if (g) cudaGraphDestroy(g);
    set_error(std::string("femk_pcg_mixed: graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    return st != FEMK_OK ? st : FEMK_ECUDA;
  }
  bool updated = false;
  if (p->mx_exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(p->mx_exec, g, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(p->mx_exec);
      p->mx_exec = nullptr;
    }
  }
  if (!updated) {
    const cudaError_t e3 = cudaGraphInstantiate(&p->mx_exec, g, 0);
    if (e3 != cudaSuccess) {
      cudaGraphDestroy(g);
      p->mx_exec = nullptr;
      set_error(std::string("femk_pcg_mixed: graph instantiation failed: ") + cudaGetErrorString(e3));
      return FEMK_ECUDA;
    }
  }
  cudaGraphDestroy(g);
  for (int i = 0; i < 4; ++i) p->mx_key[i] = key[i];
  p->mx_nodes = 3 * kChunk + 3;
  return FEMK_OK;
}

}  // namespace
}  // namespace femk

using namespace femk;

extern "C" int femk_pcg_mixed(const femk_plan* pc, const double* vals, const double* b, double* x, const double* dinv64,
                              double tol, double atol, int32_t maxiter, int mode, int32_t* inner_out, int32_t* outer_out,
                              double* relres_out, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(pc && vals && b && x && dinv64, "femk_pcg_mixed: NULL argument (a Jacobi inverse is required)");
  FEMK_CHECK_ARG(mode == FEMK_MIXED_RELIABLE || mode == FEMK_MIXED_RESTART, "femk_pcg_mixed: unknown mode");
  femk_plan* p = const_cast<femk_plan*>(pc);
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(ensure_mixed(p));
  const int64_t n = p->n;
  const MixedPtrs m = mixed_ptrs(p);
  cudaStream_t ws = p->mx_stream;
  FEMK_CUDA_TRY(cudaEventRecord(p->mx_ev[2], s));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->mx_ev[2], 0));
  if (p->cg_graph) FEMK_TRY(ensure_mixed_graph(p, vals, b, x));
  const int g1 = p->n_sm * 8;
  if (p->sell_vals32)
    k_gather32<<<::femk::counted_launch() + g1, 256, 0, ws>>>(p->sell_src, p->sell_nnz, vals, p->sell_vals32);
  else
    k_demote<<<::femk::counted_launch() + g1, 256, 0, ws>>>(vals, p->nnz, p->vals32);
  k_demote<<<::femk::counted_launch() + g1, 256, 0, ws>>>(dinv64, n, m.d32);
  k_fill_f<<<::femk::counted_launch() + g1, 256, 0, ws>>>(m.e, n, 0.f);
  MixedState init{};
  init.maxiter = maxiter;
  init.delta2 = mode == FEMK_MIXED_RESTART ? 1e-8 : 1e-2;  // inner reduction per segment: 1e-4 / 0.1
  init.restart = mode == FEMK_MIXED_RESTART ? 1 : 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(m.st, &init, sizeof(MixedState), cudaMemcpyHostToDevice, ws));
  const double tol2 = tol * tol, atol2 = atol * atol;
  launch_true_resid<true>(p, vals, x, b, m.d32, m.r, m.z, m.pv, m.st, tol2, atol2, ws);
  FEMK_CUDA_TRY(cudaGetLastError());
  MixedState* hs = (MixedState*)p->mx_host;
  int64_t enq = 0;
  int chunk = 0;
  bool have_prev = false;
  // a chunk performs at least one inner iteration unless the solve is done, so maxiter + 1 chunks
  // bound the loop
  const int64_t max_chunks = (int64_t)maxiter + 1;
  while (true) {
    if (p->cg_graph) {
      FEMK_CUDA_TRY(cudaGraphLaunch(p->mx_exec, ws));
      count_launches(p->mx_nodes);
    } else {
      FEMK_TRY(enqueue_mixed_chunk(p, vals, b, x, ws));
    }
    ++enq;
    FEMK_CUDA_TRY(cudaMemcpyAsync(hs + (chunk & 1), m.st, sizeof(MixedState), cudaMemcpyDeviceToHost, ws));
    FEMK_CUDA_TRY(cudaEventRecord(p->mx_ev[chunk & 1], ws));
    if (have_prev) {
      FEMK_CUDA_TRY(cudaEventSynchronize(p->mx_ev[(chunk - 1) & 1]));
      if (hs[(chunk - 1) & 1].done) break;
    }
    have_prev = true;
    if (enq >= max_chunks) break;
    ++chunk;
  }
  FEMK_CUDA_TRY(cudaStreamSynchronize(ws));
  MixedState fin{};
  FEMK_CUDA_TRY(cudaMemcpy(&fin, m.st, sizeof(MixedState), cudaMemcpyDeviceToHost));
  FEMK_CUDA_TRY(cudaEventRecord(p->mx_ev[2], ws));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(s, p->mx_ev[2], 0));
  if (inner_out) *inner_out = fin.iter;
  if (outer_out) *outer_out = fin.outer;
  if (relres_out) *relres_out = std::sqrt(fin.rr64) / (std::sqrt(fin.bb) + 1e-30);
  if (fin.status == FEMK_BREAKDOWN) {
    set_error("femk_pcg_mixed: <p, A p> <= 0 in FP32 (operator not SPD at single precision)");
    return FEMK_BREAKDOWN;
  }
  if (fin.status == FEMK_NONFINITE) {
    set_error("femk_pcg_mixed: non-finite value in a reduction");
    return FEMK_NONFINITE;
  }
  if (fin.rr64 > fin.atol2) {
    set_error("femk_pcg_mixed: iteration cap reached above tolerance");
    return FEMK_NOT_CONVERGED;
  }
  return FEMK_OK;
}
