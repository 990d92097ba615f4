// Mixed-precision Jacobi-PCG: FP32 values, vectors and SpMV accumulation in the inner CG; FP64
// solution and FP64 true residual r = b - A x (FP64 values) at every reliable update.
//
// The inner iteration is preconditioned CG in the single-reduction form of Chronopoulos and Gear
// (J. Comput. Appl. Math. 25, 1989): with u = D^-1 r, w = A u, s = A p,
//
//   K_A  p = u + beta p;  s = w + beta s;  e += alpha p;  r -= alpha s;  u = D^-1 r
//   K_B  w = A32 u;  gamma' = <r, u>,  delta = <w, u>,  rho = <r, r>       (one grid reduction)
//        beta = gamma' / gamma;  alpha = gamma' / (delta - beta gamma' / alpha)
//
// Both inner products of an iteration come out of the SpMV's epilogue, so an iteration is two
// kernels and one reduction (the textbook form needs three kernels and two reductions; the
// denominator delta - beta gamma' / alpha equals <p, A p> in exact arithmetic).
//
// A reliable update is requested when rho fell below delta2 of its value at the previous update,
// when the FP32 recurrence meets the stop test, or at the iteration cap. The iterations left in the
// chunk then return at entry, and the chunk ends with
//     x += e;  e = 0;  r64 = b - A64 x;  r = fp32(r64);  u = D^-1 r       (k_fold, k_true_resid)
//     w = A32 u and the three products; beta = gamma'/gamma (0 to restart)  (K_B refresh)
// which keeps the search direction (FEMK_MIXED_RELIABLE, residual replacement: p and s = A p are
// unchanged) or restarts it (FEMK_MIXED_RESTART, classic iterative refinement). The solve stops
// only on the FP64 true residual: <r64, r64> <= max(tol^2 <b, b>, atol^2), femk_pcg's stop rule.
//
// The FP32 operator is the plan's sliced-ELL copy: 4 B value + 2 B column offset (int16, col - row)
// per entry when the bandwidth allows it, else 4 B + 4 B. Each chunk (16 iterations of 2 kernels,
// plus the 3 update kernels) is replayed as one CUDA graph.
//
// No reference counterpart: jNO runs x64 throughout (tests/test_fem_3d.py:37-46).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "femk_bulk.cuh"
#include "femk_internal.cuh"
#include "femk_spmv.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;

struct MixedState {
  double gamma;    // <r, u> of the current direction's residual
  double gnew;     // <r, u> after a reliable update, waiting for the refresh step
  double delta;    // <w, u>
  double rr;       // FP32 recurrence <r, r>
  double rr64, bb, atol2, alpha, beta, rr_since, delta2;
  int32_t iter, maxiter, done, status;
  int32_t need_update;  // 1: update requested this chunk; 2: update done, refresh step pending
  int32_t hold;         // inner iterations return at entry until the refresh step
  int32_t outer, restart;
  int32_t fresh;  // 1 until the first direction exists (beta = 0 at the first refresh)
  uint32_t ticket;
};

template <int NV, int THREADS = kThreads>
__device__ __forceinline__ bool reduce_finish(double (&v)[NV], double* partials, uint32_t* ticket, double (&out)[NV]) {
  __shared__ double red[NV][THREADS / 32];
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
      for (int w = 0; w < THREADS / 32; ++w) t += red[j][w];
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
      for (int j = 0; j < NV; ++j) s[j] += t[u][j];
  }
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
    for (int w = 0; w < THREADS / 32; ++w) t += red[j][w];
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

// K_B epilogue state: w[row] = (A u)[row] and the three products of the row
struct StepEpi {
  const float* __restrict__ u;
  const float* __restrict__ r;
  float* __restrict__ w;
  float a[3];  // <w, u>, <r, u>, <r, r>
  __device__ __forceinline__ void operator()(int64_t row, float wv) {
    w[row] = wv;
    const float ui = __ldg(u + row), ri = __ldg(r + row);
    a[0] = fmaf(wv, ui, a[0]);
    a[1] = fmaf(ri, ui, a[1]);
    a[2] = fmaf(ri, ri, a[2]);
  }
};

// Last block of K_B: the new scalars. REFRESH = the step after a reliable update (or the first one).
template <bool REFRESH>
__device__ __forceinline__ void step_finish(MixedState* st, const double (&t)[3]) {
  const double delta = t[0], gnew = REFRESH ? st->gnew : t[1], rho = t[2];
  st->delta = delta;
  st->rr = rho;
  if (!isfinite(delta) || !isfinite(gnew) || !isfinite(rho)) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
    return;
  }
  if (!REFRESH) {
    st->iter += 1;
    const bool conv = !(rho > st->atol2);
    const bool drop = rho < st->delta2 * st->rr_since;
    if (conv || drop || st->iter >= st->maxiter) {  // fold e into x and replace r at the chunk end
      st->need_update = 1;
      st->hold = 1;
      return;
    }
  }
  const double beta = (REFRESH && (st->restart || st->fresh)) ? 0.0 : gnew / st->gamma;
  const double den = beta == 0.0 ? delta : delta - beta * gnew / st->alpha;  // <p, A p> of the new direction
  if (!(den > 0.0)) {
    st->status = isfinite(den) ? FEMK_BREAKDOWN : FEMK_NONFINITE;
    st->done = 1;
    return;
  }
  st->beta = beta;
  st->alpha = gnew / den;
  st->gamma = gnew;
  if (REFRESH) {
    st->need_update = 0;
    st->hold = 0;
    st->fresh = 0;
  }
}

__device__ __forceinline__ bool step_skip(const MixedState* st, bool refresh) {
  return st->done || (refresh ? st->need_update != 2 : st->hold != 0);
}

// K_B on the register-streamed sliced-ELL operator (one thread per row)
template <typename IDX, bool REFRESH>
__global__ void __launch_bounds__(kThreads, 8) k_step32_sell(const int64_t* __restrict__ sptr, const IDX* __restrict__ cols,
                                                         const float* __restrict__ vals, int64_t n, int64_t nslices,
                                                         const float* __restrict__ u, const float* __restrict__ r,
                                                         float* __restrict__ w, double* __restrict__ partials,
                                                         MixedState* st) {
  if (step_skip(st, REFRESH)) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  StepEpi epi{u, r, w, {0.f, 0.f, 0.f}};
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    if (row >= n) continue;
    const int64_t b0 = __ldg(sptr + sl);
    const int32_t wd = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
    epi(row, sell_row<float, IDX, GatherX<float>, 8>(vals + b0 + lane, cols + b0 + lane, wd, (int32_t)row,
                                                     GatherX<float>{u}));
  }
  double v[3] = {(double)epi.a[0], (double)epi.a[1], (double)epi.a[2]}, tot[3];
  if (!reduce_finish<3>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  step_finish<REFRESH>(st, tot);
}

// K_B with the FP32 sliced-ELL stream moved into shared memory by bulk copies (femk_bulk.cuh):
// WPB warps per block, S slices in flight per warp, widths up to WMAX.
template <int WMAX, int S, int WPB, bool REFRESH>
__global__ void __launch_bounds__(WPB * 32) k_step32_bulk(const int64_t* __restrict__ sptr,
                                                         const int16_t* __restrict__ cols,
                                                         const float* __restrict__ vals, int64_t n, int64_t nslices,
                                                         const float* __restrict__ u, const float* __restrict__ r,
                                                         float* __restrict__ w, double* __restrict__ partials,
                                                         MixedState* st, const int64_t* __restrict__ cptr) {
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  constexpr int kWarpBytes = BulkRing<float, int16_t, WMAX, S>::kWarpBytes;
  if (step_skip(st, REFRESH)) return;
  const int wib = threadIdx.x >> 5;
  StepEpi epi{u, r, w, {0.f, 0.f, 0.f}};
  const bool ok = sell_bulk_rows<float, int16_t, WMAX, S>(
      bulk_smem + wib * kWarpBytes, sptr, cols, vals, n, nslices, (int64_t)blockIdx.x * WPB + wib,
      (int64_t)gridDim.x * WPB, GatherX<float>{u}, epi, &st->status, FEMK_TIMEOUT, cptr);
  if (!ok && (threadIdx.x & 31) == 0) st->done = 1;
  double v[3] = {(double)epi.a[0], (double)epi.a[1], (double)epi.a[2]}, tot[3];
  if (!reduce_finish<3, WPB * 32>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  step_finish<REFRESH>(st, tot);
}

// K_B on the CSR copy (plans without a sliced-ELL layout)
template <int L, int U, typename IDX, bool REFRESH>
__global__ void __launch_bounds__(kThreads) k_step32(const int32_t* __restrict__ indptr, const IDX* __restrict__ cols,
                                                    const float* __restrict__ vals, int64_t n,
                                                    const float* __restrict__ u, const float* __restrict__ r,
                                                    float* __restrict__ w, double* __restrict__ partials,
                                                    MixedState* st) {
  if (step_skip(st, REFRESH)) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  StepEpi epi{u, r, w, {0.f, 0.f, 0.f}};
  for (int64_t base = warp * RPW * U; base < n; base += nwarps * RPW * U) {
    float sv[U];
    int64_t rows[U];
    csr_rows<L, U, float, IDX>(indptr, cols, vals, u, n, base, lane, sv, rows);
#pragma unroll
    for (int k = 0; k < U; ++k)
      if (rows[k] < n && sub == 0) epi(rows[k], sv[k]);
  }
  double v[3] = {(double)epi.a[0], (double)epi.a[1], (double)epi.a[2]}, tot[3];
  if (!reduce_finish<3>(v, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  step_finish<REFRESH>(st, tot);
}

// K_A: p = u + beta p; s = w + beta s; e += alpha p; r -= alpha s; u = D^-1 r (no reduction).
// All seven vectors are plan-owned and 16-byte aligned: four rows per load.
__device__ __forceinline__ void cgcg_one(float alpha, float beta, float& u, float w, float& p, float& s, float& e,
                                         float& r, float d) {
  p = fmaf(beta, p, u);
  s = fmaf(beta, s, w);
  e = fmaf(alpha, p, e);
  r = fmaf(-alpha, s, r);
  u = d * r;
}

__global__ void __launch_bounds__(kThreads) k_cgcg_update(int64_t n, float* __restrict__ u, const float* __restrict__ w,
                                                         float* __restrict__ p, float* __restrict__ s,
                                                         float* __restrict__ e, float* __restrict__ r,
                                                         const float* __restrict__ dinv, const MixedState* st) {
  if (st->done || st->hold) return;
  const float alpha = (float)st->alpha, beta = (float)st->beta;
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  const int64_t n4 = n >> 2;
  float4* u4 = reinterpret_cast<float4*>(u);
  const float4* w4 = reinterpret_cast<const float4*>(w);
  float4* p4 = reinterpret_cast<float4*>(p);
  float4* s4 = reinterpret_cast<float4*>(s);
  float4* e4 = reinterpret_cast<float4*>(e);
  float4* r4 = reinterpret_cast<float4*>(r);
  const float4* d4 = reinterpret_cast<const float4*>(dinv);
  for (int64_t i = tid; i < n4; i += nt) {
    float4 uu = u4[i], pp = p4[i], ss = s4[i], ee = e4[i], rr = r4[i];
    const float4 ww = w4[i], dd = d4[i];
    cgcg_one(alpha, beta, uu.x, ww.x, pp.x, ss.x, ee.x, rr.x, dd.x);
    cgcg_one(alpha, beta, uu.y, ww.y, pp.y, ss.y, ee.y, rr.y, dd.y);
    cgcg_one(alpha, beta, uu.z, ww.z, pp.z, ss.z, ee.z, rr.z, dd.z);
    cgcg_one(alpha, beta, uu.w, ww.w, pp.w, ss.w, ee.w, rr.w, dd.w);
    u4[i] = uu;
    p4[i] = pp;
    s4[i] = ss;
    e4[i] = ee;
    r4[i] = rr;
  }
  for (int64_t i = 4 * n4 + tid; i < n; i += nt) cgcg_one(alpha, beta, u[i], w[i], p[i], s[i], e[i], r[i], dinv[i]);
}

// x += e; e = 0 (only at a requested update)
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ e, const MixedState* st) {
  if (st->done || st->need_update != 1) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += (double)e[i];
    e[i] = 0.f;
  }
}

// r64 = b - A64 x; r = fp32(r64); u = D^-1 r; <r, u>, <r64, r64> (+ <b, b> at init)
template <int L, int U, bool INIT>
__global__ void __launch_bounds__(kThreads) k_true_resid(const int32_t* __restrict__ indptr,
                                                        const int32_t* __restrict__ indices,
                                                        const double* __restrict__ vals, int64_t n,
                                                        const double* __restrict__ x, const double* __restrict__ b,
                                                        const float* __restrict__ dinv, float* __restrict__ r,
                                                        float* __restrict__ u, double* __restrict__ partials,
                                                        MixedState* st, double tol2, double atol2) {
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
    for (int k = 0; k < U; ++k) {
      const int64_t row = rows[k];
      if (row >= n || sub != 0) continue;
      const double bi = b[row];
      const double r64 = bi - sv[k];
      const float rf = (float)r64;
      const float uf = dinv[row] * rf;
      r[row] = rf;
      u[row] = uf;
      a0 += (double)rf * (double)uf;
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
    st->iter = 0;
    st->fresh = 1;
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    st->done = (!(tot[1] > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
  } else if (!isfinite(tot[0]) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
    return;
  } else if (!(tot[1] > st->atol2) || st->iter >= st->maxiter) {
    st->done = 1;
    return;
  }
  st->gnew = tot[0];
  st->need_update = 2;  // the refresh step forms w = A u, beta and alpha
  st->hold = 1;
}

template <bool INIT>
void launch_true_resid(const femk_plan* p, const double* vals, const double* x, const double* b, const float* dinv,
                       float* r, float* u, MixedState* st, double tol2, double atol2, cudaStream_t s) {
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    const int grid = wave_grid(k_true_resid<L, U, INIT>, kThreads, p);
    k_true_resid<L, U, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
        p->indptr, p->indices, vals, p->n, x, b, dinv, r, u, p->partials, st, tol2, atol2);
  });
}

template <int S, int WPB, int WMAX, bool REFRESH>
bool launch_step32_bulk_cfg(const femk_plan* p, const float* u, const float* r, float* w, MixedState* st,
                            cudaStream_t s, bool prime) {
  auto kern = k_step32_bulk<WMAX, S, WPB, REFRESH>;
  constexpr int kSmem = WPB * BulkRing<float, int16_t, WMAX, S>::kWarpBytes;
  static int per_sm = -1;  // per instantiation: opt-in shared memory size + occupancy, queried once
  if (per_sm < 0) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WPB * 32, kSmem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
  }
  if (per_sm <= 0) return false;
  if (prime) return true;
  const int grid = p->n_sm * std::min(per_sm, 16);
  const bool tab = p->sell_cu != nullptr;  // per-slice column tables (shared-offset slices stored once)
  kern<<<::femk::counted_launch() + grid, WPB * 32, kSmem, s>>>(
      (const int64_t*)p->sell_ptr, (const int16_t*)(tab ? p->sell_cu : p->sell_c16), (const float*)p->sell_vals32,
      p->n, p->n_slices, u, r, w, p->partials, st, (const int64_t*)(tab ? p->sell_cuptr : nullptr));
  return true;
}

// bulk-copy K_B in the plan's configuration (bulk32_cfg: 10 * stages + warps per block)
// prime = true only sets the kernel attribute and reads the occupancy (before a graph capture)
template <bool REFRESH>
bool launch_step32_bulk(const femk_plan* p, const float* u, const float* r, float* w, MixedState* st, cudaStream_t s,
                        bool prime = false) {
  if (!p->bulk32_cfg || !p->sell_vals32 || !p->sell_c16 || p->max_row > 32) return false;
  if (((uintptr_t)p->sell_vals32 & 15u) || ((uintptr_t)p->sell_c16 & 15u)) return false;
  if (p->sell_cu && ((uintptr_t)p->sell_cu & 15u)) return false;
  // ring stages sized for the widest row: 8 (2-D P1 triangles), 16 (P1 tetrahedra), 32
  const int wsel = p->max_row <= 8 ? 8 : (p->max_row <= 16 ? 16 : 32);
#define FEMK_BULK_CFG(code, S, WPB)                                                                     \
  case code:                                                                                            \
    return wsel == 8    ? launch_step32_bulk_cfg<S, WPB, 8, REFRESH>(p, u, r, w, st, s, prime)  \
           : wsel == 16 ? launch_step32_bulk_cfg<S, WPB, 16, REFRESH>(p, u, r, w, st, s, prime) \
                        : launch_step32_bulk_cfg<S, WPB, 32, REFRESH>(p, u, r, w, st, s, prime);
  switch (p->bulk32_cfg) {
    FEMK_BULK_CFG(14, 1, 4)
    FEMK_BULK_CFG(18, 1, 8)
    FEMK_BULK_CFG(24, 2, 4)
    FEMK_BULK_CFG(28, 2, 8)
    FEMK_BULK_CFG(38, 3, 8)
    default:
      return false;
  }
#undef FEMK_BULK_CFG
}

template <bool REFRESH>
void launch_step32(const femk_plan* p, const float* u, const float* r, float* w, MixedState* st, cudaStream_t s) {
  if (launch_step32_bulk<REFRESH>(p, u, r, w, st, s)) return;
  if (p->sell_vals32) {
    if (p->sell_c16) {
      auto k = k_step32_sell<int16_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(
          p->sell_ptr, p->sell_c16, p->sell_vals32, p->n, p->n_slices, u, r, w, p->partials, st);
    } else {
      auto k = k_step32_sell<int32_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(
          p->sell_ptr, p->sell_cols, p->sell_vals32, p->n, p->n_slices, u, r, w, p->partials, st);
    }
    return;
  }
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    if (p->cols16) {
      auto k = k_step32<L, U, int16_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(p->indptr, p->cols16, p->vals32,
                                                                                  p->n, u, r, w, p->partials, st);
    } else {
      auto k = k_step32<L, U, int32_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(p->indptr, p->indices, p->vals32,
                                                                                  p->n, u, r, w, p->partials, st);
    }
  });
}

// occupancy queries and shared-memory attributes of every kernel a chunk may launch (before capture)
void prime_mixed(const femk_plan* p) {
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    (void)wave_grid(k_true_resid<L, U, false>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int16_t, false>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int32_t, false>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int16_t, true>, kThreads, p);
    (void)wave_grid(k_step32<L, U, int32_t, true>, kThreads, p);
  });
  (void)wave_grid(k_step32_sell<int16_t, false>, kThreads, p);
  (void)wave_grid(k_step32_sell<int32_t, false>, kThreads, p);
  (void)wave_grid(k_step32_sell<int16_t, true>, kThreads, p);
  (void)wave_grid(k_step32_sell<int32_t, true>, kThreads, p);
  (void)launch_step32_bulk<false>(p, nullptr, nullptr, nullptr, nullptr, nullptr, true);
  (void)launch_step32_bulk<true>(p, nullptr, nullptr, nullptr, nullptr, nullptr, true);
  (void)vec_grid(k_cgcg_update, kThreads, p);
  (void)wave_grid(k_fold, 256, p);
}

struct MixedPtrs {
  float *r, *u, *w, *pv, *s, *e, *d32;
  MixedState* st;
};

MixedPtrs mixed_ptrs(const femk_plan* p) {
  const int64_t vs = p->vstride;
  MixedPtrs m;
  m.r = p->work32;
  m.u = m.r + vs;
  m.w = m.u + vs;
  m.pv = m.w + vs;
  m.s = m.pv + vs;
  m.e = m.s + vs;
  m.d32 = m.e + vs;
  m.st = (MixedState*)p->work64b;
  return m;
}

// one chunk: kChunk inner iterations, then the (conditional) reliable update and refresh step
int enqueue_mixed_chunk(const femk_plan* p, const double* vals, const double* b, double* x, cudaStream_t s) {
  const MixedPtrs m = mixed_ptrs(p);
  const int64_t n = p->n;
  for (int it = 0; it < kChunk; ++it) {
    k_cgcg_update<<<::femk::counted_launch() + vec_grid(k_cgcg_update, kThreads, p), kThreads, 0, s>>>(
        n, m.u, m.w, m.pv, m.s, m.e, m.r, m.d32, m.st);
    launch_step32<false>(p, m.u, m.r, m.w, m.st, s);
  }
  k_fold<<<::femk::counted_launch() + wave_grid(k_fold, 256, p), 256, 0, s>>>(n, x, m.e, m.st);
  launch_true_resid<false>(p, vals, x, b, m.d32, m.r, m.u, m.st, 0.0, 0.0, s);
  launch_step32<true>(p, m.u, m.r, m.w, m.st, s);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int ensure_mixed(femk_plan* p) {
  FEMK_TRY(ensure_workspace(p));
  if (!p->work32) FEMK_CUDA_TRY(cudaMalloc(&p->work32, sizeof(float) * kWork32Vectors * p->vstride));
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
  const void* key[5] = {vals, b, x, p->sell_vals32 ? (const void*)p->sell_vals32 : (const void*)p->vals32, nullptr};
  bool same = p->mx_exec != nullptr;
  for (int i = 0; i < 5; ++i) same = same && key[i] == p->mx_key[i];
  if (same) return FEMK_OK;
  prime_mixed(p);
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
  for (int i = 0; i < 5; ++i) p->mx_key[i] = key[i];
  p->mx_nodes = 2 * kChunk + 3;
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
  FEMK_CHECK_ARG(tol >= 0.0 && atol >= 0.0, "femk_pcg_mixed: negative tolerance");
  femk_plan* p = const_cast<femk_plan*>(pc);
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(ensure_mixed(p));
  const int64_t n = p->n;
  const MixedPtrs m = mixed_ptrs(p);
  cudaStream_t ws = p->mx_stream;
  FEMK_CUDA_TRY(cudaEventRecord(p->mx_ev[2], s));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->mx_ev[2], 0));
  if (p->cg_graph) FEMK_TRY(ensure_mixed_graph(p, vals, b, x));
  else prime_mixed(p);
  const int g1 = p->n_sm * 8;
  if (p->sell_vals32)
    k_gather32<<<::femk::counted_launch() + g1, 256, 0, ws>>>(p->sell_src, p->sell_nnz, vals, p->sell_vals32);
  else
    k_demote<<<::femk::counted_launch() + g1, 256, 0, ws>>>(vals, p->nnz, p->vals32);
  k_demote<<<::femk::counted_launch() + g1, 256, 0, ws>>>(dinv64, n, m.d32);
  // e, p and s start at zero (beta = 0 multiplies p and s at the first step: 0 * NaN would stick)
  k_fill_f<<<::femk::counted_launch() + g1, 256, 0, ws>>>(m.e, n, 0.f);
  k_fill_f<<<::femk::counted_launch() + g1, 256, 0, ws>>>(m.pv, n, 0.f);
  k_fill_f<<<::femk::counted_launch() + g1, 256, 0, ws>>>(m.s, n, 0.f);
  MixedState init{};
  init.maxiter = maxiter;
  // reliable updates when <r, r> has fallen by delta2 since the last one: measured on B200 at P1 128^3,
  // 26.6 ms per mixed step with 1e-4 vs 27.1 ms with 1e-2 (9 FP64 updates), same 1e-8 stop rule
  init.delta2 = mode == FEMK_MIXED_RESTART ? 1e-8 : (p->mixed_delta2 > 0.0 ? p->mixed_delta2 : 1e-4);
  init.restart = mode == FEMK_MIXED_RESTART ? 1 : 0;
  init.alpha = 1.0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(m.st, &init, sizeof(MixedState), cudaMemcpyHostToDevice, ws));
  const double tol2 = tol * tol, atol2 = atol * atol;
  launch_true_resid<true>(p, vals, x, b, m.d32, m.r, m.u, m.st, tol2, atol2, ws);
  launch_step32<true>(p, m.u, m.r, m.w, m.st, ws);  // w = A u, the first alpha
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
  if (fin.status == FEMK_TIMEOUT) {
    set_error("femk_pcg_mixed: a bulk-copy wait of the FP32 SpMV gave up");
    return FEMK_TIMEOUT;
  }
  if (fin.rr64 > fin.atol2) {
    set_error("femk_pcg_mixed: iteration cap reached above tolerance");
    return FEMK_NOT_CONVERGED;
  }
  return FEMK_OK;
}
