// Mixed-precision Jacobi-PCG: FP32 values, vectors and SpMV accumulation in the inner CG; FP64
// solution and FP64 true residual r = b - A x (FP64 values) at every reliable update.
//
// Inner step (FP32):  q = A32 p;  alpha = gamma / <p, q>;  e += alpha p;  r -= alpha q;  z = D^-1 r
// Reliable update (FP64), when <r, r> fell below delta^2 of its value at the previous update, when
// the FP32 recurrence meets the stop test, or at the iteration cap:
//     x += e;  e = 0;  r64 = b - A64 x;  r = fp32(r64);  z = D^-1 r;  gamma = <r, z>
// then p = z + beta p continues with the same search direction (FEMK_MIXED_RELIABLE) or restarts
// with beta = 0 (FEMK_MIXED_RESTART, classic iterative refinement). The solve stops only on the
// FP64 true residual: <r64, r64> <= max(tol^2 <b, b>, atol^2) -- the stop rule of femk_pcg.
//
// The FP32 matrix stream is 4 B value + 2 B column offset (int16, col - row) per entry when the
// plan's bandwidth allows it, else 4 B + 4 B.
//
// No reference counterpart: jNO runs x64 throughout (tests/test_fem_3d.py:37-46).
#include <algorithm>
#include <cmath>

#include "femk_internal.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;

struct MixedState {
  double gamma, gamma_new, rr, rr64, bb, atol2, alpha, beta, rr_since, delta2;
  int32_t iter, maxiter, done, status, need_update, outer, restart;
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

// FP32 CSR row with int16 (offset from the row) or int32 column indices
template <int L, typename IDX>
__device__ __forceinline__ float row32(const int32_t* __restrict__ indptr, const IDX* __restrict__ cols,
                                       const float* __restrict__ vals, const float* __restrict__ x, int64_t row,
                                       bool valid, int sub) {
  float s = 0.f;
  if (valid) {
    const int32_t beg = __ldg(indptr + row), end = __ldg(indptr + row + 1);
    for (int32_t k = beg + sub; k < end; k += L) {
      const int64_t col = sizeof(IDX) == 2 ? row + (int64_t)__ldcs(cols + k) : (int64_t)__ldcs(cols + k);
      s = fmaf(__ldcs(vals + k), __ldg(x + col), s);
    }
  }
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// q = A32 p, <p, q> -> alpha
template <int L, typename IDX>
__global__ void __launch_bounds__(kThreads) k_step32(const int32_t* __restrict__ indptr, const IDX* __restrict__ cols,
                                                    const float* __restrict__ vals, int64_t n, const float* __restrict__ p,
                                                    float* __restrict__ q, double* __restrict__ partials, MixedState* st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  float acc = 0.f;
  for (int64_t base = warp * RPW; base < n; base += nwarps * RPW) {
    const int64_t row = base + lane / L;
    const bool valid = row < n;
    const float s = row32<L, IDX>(indptr, cols, vals, p, row, valid, sub);
    if (valid && sub == 0) {
      q[row] = s;
      acc = fmaf(__ldg(p + row), s, acc);
    }
  }
  double v[1] = {(double)acc}, tot[1];
  if (!reduce_finish<1>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  st->alpha = st->gamma / tot[0];
  if (!isfinite(tot[0])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(tot[0] > 0.0)) {
    st->status = FEMK_BREAKDOWN;
    st->done = 1;
  }
}

// e += alpha p; r -= alpha q; z = D^-1 r; <r, z>, <r, r>; decide on a reliable update
__global__ void __launch_bounds__(kThreads) k_update32(int64_t n, float* __restrict__ e, float* __restrict__ r,
                                                      float* __restrict__ z, const float* __restrict__ p,
                                                      const float* __restrict__ q, const float* __restrict__ dinv,
                                                      double* __restrict__ partials, MixedState* st) {
  if (st->done) return;
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
    st->need_update = 1;  // beta is formed from the replaced residual
  } else {
    st->beta = tot[0] / st->gamma;
    st->gamma = tot[0];
  }
}

// x += e; e = 0 (only on a reliable update)
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ e, const MixedState* st) {
  if (st->done || !st->need_update) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += (double)e[i];
    e[i] = 0.f;
  }
}

// r64 = b - A64 x; r = fp32(r64); z = D^-1 r; <r, z>, <r64, r64> (+ <b, b> at init)
template <int L, bool INIT>
__global__ void __launch_bounds__(kThreads) k_true_resid(const int32_t* __restrict__ indptr,
                                                        const int32_t* __restrict__ indices,
                                                        const double* __restrict__ vals, int64_t n,
                                                        const double* __restrict__ x, const double* __restrict__ b,
                                                        const float* __restrict__ dinv, float* __restrict__ r,
                                                        float* __restrict__ z, float* __restrict__ p,
                                                        double* __restrict__ partials, MixedState* st, double tol2,
                                                        double atol2) {
  if (!INIT && (st->done || !st->need_update)) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t base = warp * RPW; base < n; base += nwarps * RPW) {
    const int64_t row = base + lane / L;
    const bool valid = row < n;
    double s = 0.0;
    if (valid) {
      const int32_t beg = __ldg(indptr + row), end = __ldg(indptr + row + 1);
      for (int32_t k = beg + sub; k < end; k += L) s += __ldcs(vals + k) * __ldg(x + __ldcs(indices + k));
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (valid && sub == 0) {
      const double bi = b[row];
      const double r64 = bi - s;
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
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    st->done = (!(tot[1] > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
    return;
  }
  st->need_update = 0;
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
}

__global__ void k_pupdate32(int64_t n, float* __restrict__ p, const float* __restrict__ z, const MixedState* st) {
  if (st->done) return;
  const float beta = (float)st->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fmaf(beta, p[i], z[i]);
}

int lanes(const femk_plan* p) {
  const double avg = p->n > 0 ? (double)p->nnz / (double)p->n : 1.0;
  return avg <= 5.0 ? 4 : avg <= 10.0 ? 8 : avg <= 20.0 ? 16 : 32;
}

template <bool INIT>
void launch_true_resid(const femk_plan* p, const double* vals, const double* x, const double* b, const float* dinv,
                       float* r, float* z, float* pv, MixedState* st, double tol2, double atol2, cudaStream_t s) {
  const int grid = p->n_sm * (2048 / kThreads);
  switch (lanes(p)) {
    case 4:
      k_true_resid<4, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, x, b, dinv, r, z, pv, p->partials, st, tol2, atol2);
      break;
    case 8:
      k_true_resid<8, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, x, b, dinv, r, z, pv, p->partials, st, tol2, atol2);
      break;
    case 16:
      k_true_resid<16, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, x, b, dinv, r, z, pv, p->partials, st, tol2, atol2);
      break;
    default:
      k_true_resid<32, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, x, b, dinv, r, z, pv, p->partials, st, tol2, atol2);
  }
}

template <typename IDX>
void launch_step32(const femk_plan* p, const IDX* cols, const float* vals32, const float* pv, float* q, MixedState* st,
                   cudaStream_t s) {
  const int grid = p->n_sm * (2048 / kThreads);
  switch (lanes(p)) {
    case 4:
      k_step32<4, IDX><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, cols, vals32, p->n, pv, q, p->partials, st);
      break;
    case 8:
      k_step32<8, IDX><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, cols, vals32, p->n, pv, q, p->partials, st);
      break;
    case 16:
      k_step32<16, IDX><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, cols, vals32, p->n, pv, q, p->partials, st);
      break;
    default:
      k_step32<32, IDX><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, cols, vals32, p->n, pv, q, p->partials, st);
  }
}

int ensure_mixed(femk_plan* p) {
  FEMK_TRY(ensure_workspace(p));
  if (!p->work32) FEMK_CUDA_TRY(cudaMalloc(&p->work32, sizeof(float) * 6 * (p->n + 1)));
  if (!p->vals32) FEMK_CUDA_TRY(cudaMalloc(&p->vals32, sizeof(float) * (p->nnz + 1)));
  if (!p->work64b) FEMK_CUDA_TRY(cudaMalloc(&p->work64b, sizeof(MixedState) + 64));
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
  float* r = p->work32;
  float* z = r + n;
  float* pv = z + n;
  float* q = pv + n;
  float* e = q + n;
  float* d32 = e + n;
  MixedState* st = (MixedState*)p->work64b;
  const int g1 = p->n_sm * 8;
  k_demote<<<::femk::counted_launch() + g1, 256, 0, s>>>(vals, p->nnz, p->vals32);
  k_demote<<<::femk::counted_launch() + g1, 256, 0, s>>>(dinv64, n, d32);
  k_fill_f<<<::femk::counted_launch() + g1, 256, 0, s>>>(e, n, 0.f);
  MixedState init{};
  init.maxiter = maxiter;
  init.delta2 = mode == FEMK_MIXED_RESTART ? 1e-8 : 1e-2;  // inner reduction per segment: 1e-4 / 0.1
  init.restart = mode == FEMK_MIXED_RESTART ? 1 : 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(MixedState), cudaMemcpyHostToDevice, s));
  const double tol2 = tol * tol, atol2 = atol * atol;
  launch_true_resid<true>(p, vals, x, b, d32, r, z, pv, st, tol2, atol2, s);
  FEMK_CUDA_TRY(cudaGetLastError());
  MixedState* hs = nullptr;
  FEMK_CUDA_TRY(cudaMallocHost(&hs, 2 * sizeof(MixedState)));
  cudaEvent_t ev[2];
  cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  int64_t enq = 0;
  int chunk = 0;
  bool have_prev = false;
  int status = FEMK_OK;
  // every inner iteration may end in a reliable update, so the cap on enqueued steps is maxiter
  while (true) {
    const int64_t todo = std::min<int64_t>(kChunk, (int64_t)maxiter - enq);
    for (int64_t it = 0; it < todo; ++it) {
      if (p->cols16)
        launch_step32<int16_t>(p, p->cols16, p->vals32, pv, q, st, s);
      else
        launch_step32<int32_t>(p, p->indices, p->vals32, pv, q, st, s);
      k_update32<<<::femk::counted_launch() + g1, kThreads, 0, s>>>(n, e, r, z, pv, q, d32, p->partials, st);
      k_fold<<<::femk::counted_launch() + g1, 256, 0, s>>>(n, x, e, st);
      launch_true_resid<false>(p, vals, x, b, d32, r, z, nullptr, st, tol2, atol2, s);
      k_pupdate32<<<::femk::counted_launch() + g1, 256, 0, s>>>(n, pv, z, st);
    }
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_error(std::string("femk_pcg_mixed: ") + cudaGetErrorString(le));
      status = FEMK_ECUDA;
      break;
    }
    enq += todo;
    FEMK_CUDA_TRY(cudaMemcpyAsync(hs + (chunk & 1), st, sizeof(MixedState), cudaMemcpyDeviceToHost, s));
    FEMK_CUDA_TRY(cudaEventRecord(ev[chunk & 1], s));
    if (have_prev) {
      FEMK_CUDA_TRY(cudaEventSynchronize(ev[(chunk - 1) & 1]));
      if (hs[(chunk - 1) & 1].done) break;
    }
    have_prev = true;
    if (enq >= maxiter) break;
    ++chunk;
  }
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  MixedState fin{};
  FEMK_CUDA_TRY(cudaMemcpy(&fin, st, sizeof(MixedState), cudaMemcpyDeviceToHost));
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  cudaFreeHost(hs);
  if (inner_out) *inner_out = fin.iter;
  if (outer_out) *outer_out = fin.outer;
  if (relres_out) *relres_out = std::sqrt(fin.rr64) / (std::sqrt(fin.bb) + 1e-30);
  if (status != FEMK_OK) return status;
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
