// Mixed-precision Jacobi-PCG: FP32 values, vectors and SpMV accumulation in the inner CG; FP64
// solution and FP64 true residual r = b - A x (FP64 values) at every reliable update.
//
// The FP32 inner loop runs CG on the symmetrically scaled operator A^ = S A S, S = D^-1/2 (D the
// Jacobi diagonal), which is the Jacobi-PCG iteration in split form: with x = S x^, r^ = S r, the
// iterates map one to one, and the preconditioned residual z = D^-1 r never has to be stored
// (z^ = r^). A^ is formed in FP64 and rounded to FP32 when the values are gathered. Each iteration
// is two kernels with one grid reduction, after the single-reduction arrangement of Chronopoulos and
// Gear (J. Comput. Appl. Math. 25, 1989): w = A^ r and s = A^ p kept by recurrence,
//
//   K_A  p = r + beta p;  s = w + beta s;  e += alpha p;  r -= alpha s          (elementwise)
//        block partials of <p, s>, <r, s>, <r, r>, <r, D r>                     (no grid wait)
//   K_B  w = A^ r;  <r, w>;  the last block adds K_A's partials in block order and forms
//        gamma' = <r, r>;  beta' = gamma' / gamma;
//        <p', A^ p'> = <r, w> + 2 beta' <r, s> + beta'^2 <p, s>   (p' = r + beta' p);
//        alpha' = gamma' / <p', A^ p'>;  <r, D r> = ||r_unscaled||^2 for the stop test
//
// <p', A^ p'> is the expanded product of the next direction with itself (A^ symmetric, s = A^ p), not
// Chronopoulos and Gear's delta - beta gamma' / alpha: that identity assumes the new residual is
// orthogonal to the old direction, which a reliable update (residual replacement) breaks -- in a
// numpy model of this loop on 2-D P1 128^2 the FP32 residual then grew 4.6e3x within 68 steps. With
// the expanded form the model takes the textbook FP32 loop's iteration counts (517 vs 517 there,
// 194 vs 193 on 3-D P1 48^3), and so does oracle.pcg.mixed_pcg.
//
// A reliable update is requested when <r, D r> fell below delta2 of the FP64 <r, r> at the previous
// update, when the FP32 recurrence meets the stop test (both tested on odd steps, the ones that read
// D), or at the iteration cap. The iterations left in the chunk then return at entry, and the chunk
// ends with
//     x += S e;  e = 0;  r64 = b - A64 x;  r^ = fp32(S r64);  <r^, r^>, <p, s>, <r^, s>   (k_fold, k_true_resid)
//     K_B again on the replaced r^ (refresh): beta' = <r^, r^> / gamma (0 to restart)
// which keeps the search direction (FEMK_MIXED_RELIABLE, residual replacement: p and s = A^ p are
// unchanged) or restarts it with beta' = 0 (FEMK_MIXED_RESTART, classic iterative refinement). The
// solve stops only on the FP64 true residual: <r64, r64> <= max(tol^2 <b, b>, atol^2), femk_pcg's
// stop rule.
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
static_assert(kChunk % 2 == 0, "steps alternate even / odd within a chunk");
// K_A's block partials live past K_B's in the plan's partials buffer
constexpr int64_t kPartialsA = 16384;

struct MixedState {
  double gamma;    // <r^, r^> of the current direction's residual
  double gnew;     // <r^, r^> after a reliable update, waiting for the refresh step
  double ps, rs;   // <p, s> and <r^, s> after a reliable update (the refresh step's products)
  double rr;       // FP32 recurrence <r, r> (unscaled: <r^, D r^>)
  double rr64, bb, atol2, alpha, beta, rr_since, delta2;
  double alpha_pend;  // alpha of an even step whose e += alpha p is still owed (the next odd step or the fold pays it)
  int32_t iter, maxiter, done, status;
  int32_t need_update;  // 1: update requested this chunk; 2: update done, refresh step pending
  int32_t hold;         // inner iterations return at entry until the refresh step
  int32_t outer, restart;
  int32_t fresh;  // 1 until the first direction exists (beta = 0 at the first refresh)
  uint32_t ticket;
};

// Block sum of NV values per thread, in a fixed order; the result is valid in every thread.
template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red[NV][THREADS / 32];
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) red[j][threadIdx.x >> 5] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double t = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) t += red[j][w];
    v[j] = t;
  }
}

template <int NV, int THREADS = kThreads>
__device__ __forceinline__ bool reduce_finish(double (&v)[NV], double* partials, uint32_t* ticket, double (&out)[NV]) {
  __shared__ bool last;
  block_sum<NV, THREADS>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) partials[(int64_t)blockIdx.x * NV + j] = v[j];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) s[j] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS)
#pragma unroll
    for (int j = 0; j < NV; ++j) s[j] += __ldcg(partials + (int64_t)b * NV + j);
  block_sum<NV, THREADS>(s);
#pragma unroll
  for (int j = 0; j < NV; ++j) out[j] = s[j];
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// the NV partials of nblk blocks of an earlier kernel, summed in block order by one block
template <int NV, int THREADS>
__device__ __forceinline__ void sum_block_partials(const double* partials, int nblk, double (&out)[NV]) {
#pragma unroll
  for (int j = 0; j < NV; ++j) out[j] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += THREADS)
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] += __ldcg(partials + (int64_t)b * NV + j);
  block_sum<NV, THREADS>(out);
}

__global__ void k_fill_f(float* __restrict__ v, int64_t n, float val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = val;
}

// S = D^-1/2 from the Jacobi inverse: FP32 (the fold x += S e) and FP64 (s64, forming A^); D itself
// (FP32, for <r, D r>)
__global__ void k_scaling(const double* __restrict__ dinv, int64_t n, float* __restrict__ sc, float* __restrict__ dd,
                          double* __restrict__ s64) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double di = dinv[i];
    const double si = sqrt(di);
    sc[i] = (float)si;
    dd[i] = (float)(1.0 / di);
    s64[i] = si;
  }
}

// A^ = S A S into the FP32 sliced-ELL copy: thread per (slice, lane) row, entry k of the row being
// CSR position indptr[row] + k (padding past the row's length holds 0); each value is
// (a_ij s_i) s_j in FP64, rounded once to FP32
template <typename IDX>
__global__ void k_gather_scaled(const int64_t* __restrict__ sptr, const int32_t* __restrict__ indptr,
                                const IDX* __restrict__ cols, int64_t n, int64_t nslices, const double* __restrict__ vals,
                                int64_t nnz, int32_t cap, const double* __restrict__ s64, float* __restrict__ out,
                                int* __restrict__ err) {
  extern __shared__ double sg_buf[];
  const int wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  sell_transpose_warp<float>(
      sg_buf + (int64_t)wib * cap, cap, sptr, indptr, n, nslices, vals, nnz, out, (int64_t)blockIdx.x * wpb + wib,
      (int64_t)gridDim.x * wpb,
      [&](double v, int64_t row, int64_t j) {
        const int64_t col = sizeof(IDX) == 2 ? row + (int64_t)__ldcs(cols + j) : (int64_t)__ldcs(cols + j);
        return (float)(v * __ldg(s64 + row) * __ldg(s64 + col));
      },
      err);
}

// the same on the canonical CSR (plans without a sliced-ELL layout): thread per row
__global__ void k_scale_csr(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int64_t n,
                            const double* __restrict__ vals, const double* __restrict__ s64, float* __restrict__ out) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
    const double si = s64[row];
    for (int32_t k = indptr[row]; k < indptr[row + 1]; ++k) out[k] = (float)(vals[k] * si * s64[indices[k]]);
  }
}

// beta of the refresh step: 0 for the first direction and in restart mode, else <r^, r^> of the
// replaced residual over the old gamma
__device__ __forceinline__ double refresh_beta(const MixedState* st) {
  return (st->restart || st->fresh) ? 0.0 : st->gnew / st->gamma;
}

// K_B epilogue: w[row] = (A^ r)[row] and the row's share of <r, w>
struct StepEpi {
  const float* __restrict__ r;
  float* __restrict__ w;
  float a;
  __device__ __forceinline__ void operator()(int64_t row, float wv) {
    w[row] = wv;
    a = fmaf(__ldg(r + row), wv, a);
  }
};

__device__ __forceinline__ bool step_skip(const MixedState* st, bool refresh) {
  return st->done || (refresh ? st->need_update != 2 : st->hold != 0);
}

// Last block of K_B (all its threads): the new scalars from <r, w> and, for a normal step, K_A's
// partials (<p, s>, <r, s>, <r, r>, and on odd steps <r, D r>, which the stop and drop tests need:
// they run on odd steps only); a refresh step takes them from the update. An even step leaves its
// e += alpha p owed (alpha_pend), paid by the next odd K_A or by the fold.
// (not inlined: it runs once per launch in one block, and inlined it adds registers to the row loop)
template <bool REFRESH, int THREADS>
__device__ __noinline__ void step_finish(MixedState* st, double rw, const double* pa, int ga, int odd) {
  double t[4];
  if (!REFRESH) sum_block_partials<4, THREADS>(pa, ga, t);
  if (threadIdx.x) return;
  double ps, rs, gnew;
  if (REFRESH) {
    ps = st->ps;
    rs = st->rs;
    gnew = st->gnew;
  } else {
    ps = t[0];
    rs = t[1];
    gnew = t[2];
    if (odd) st->rr = t[3];
    st->iter += 1;
    st->alpha_pend = odd ? 0.0 : st->alpha;
  }
  if (!isfinite(rw) || !isfinite(ps) || !isfinite(rs) || !isfinite(gnew) || !isfinite(st->rr)) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
    return;
  }
  if (!REFRESH) {
    const double rho = t[3];
    const bool conv = odd && !(rho > st->atol2);
    const bool drop = odd && rho < st->delta2 * st->rr_since;
    if (conv || drop || st->iter >= st->maxiter) {  // fold e into x and replace r at the chunk end
      st->need_update = 1;
      st->hold = 1;
      return;
    }
  }
  const double beta = REFRESH ? refresh_beta(st) : gnew / st->gamma;
  const double den = rw + 2.0 * beta * rs + beta * beta * ps;  // <p', A^ p'>, p' = r + beta p
  if (!(den > 0.0)) {
    if (!REFRESH) {  // in exact arithmetic only r = 0 gets here (an untested even step): the FP64 residual decides
      st->need_update = 1;
      st->hold = 1;
      return;
    }
    st->status = FEMK_BREAKDOWN;  // <p', A^ p'> <= 0 right after a residual replacement
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

// K_B on the register-streamed sliced-ELL operator (one thread per row; the plans that reach it are
// the ones the bulk-copy ring does not take, chiefly 3-D P2 with rows of up to 65 entries and int32
// columns). 16 entries in flight a thread (48 registers, 5 blocks of 256 per SM): at P2 64^3 the
// mixed solve took 77.1 ms against 81.7 ms with 8 entries at 32 registers and 87.8 ms with 32.
template <typename IDX, bool REFRESH>
__global__ void __launch_bounds__(kThreads) k_step32_sell(const int64_t* __restrict__ sptr, const IDX* __restrict__ cols,
                                                         const float* __restrict__ vals, int64_t n, int64_t nslices,
                                                         const float* __restrict__ r, float* __restrict__ w,
                                                         double* __restrict__ partials, int ga, MixedState* st,
                                                         int odd) {
  if (step_skip(st, REFRESH)) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  StepEpi epi{r, w, 0.f};
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    if (row >= n) continue;
    const int64_t b0 = __ldg(sptr + sl);
    const int32_t wd = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
    epi(row, sell_row<float, IDX, 16>(vals + b0 + lane, cols + b0 + lane, wd, (int32_t)row,
                                      checked(GatherX<float>{r}, n, &st->status)));
  }
  double v[1] = {(double)epi.a}, tot[1];
  if (!reduce_finish<1>(v, partials, &st->ticket, tot)) return;
  step_finish<REFRESH, kThreads>(st, tot[0], partials + kPartialsA, ga, odd);
}

// K_B with the FP32 sliced-ELL stream moved into shared memory by bulk copies (femk_bulk.cuh):
// WPB warps per block, S slices in flight per warp, widths up to WMAX.
template <int WMAX, int S, int WPB, bool REFRESH>
__global__ void __launch_bounds__(WPB * 32) k_step32_bulk(const int64_t* __restrict__ sptr,
                                                         const int16_t* __restrict__ cols,
                                                         const float* __restrict__ vals, int64_t n, int64_t nslices,
                                                         const float* __restrict__ r, float* __restrict__ w,
                                                         double* __restrict__ partials, int ga, MixedState* st,
                                                         const int64_t* __restrict__ cptr, int odd) {
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  constexpr int kWarpBytes = BulkRing<float, int16_t, WMAX, S>::kWarpBytes;
  if (step_skip(st, REFRESH)) return;
  const int wib = threadIdx.x >> 5;
  StepEpi epi{r, w, 0.f};
  const bool ok = sell_bulk_rows<float, int16_t, WMAX, S>(
      bulk_smem + wib * kWarpBytes, sptr, cols, vals, n, nslices, (int64_t)blockIdx.x * WPB + wib,
      (int64_t)gridDim.x * WPB, checked(GatherX<float>{r}, n, &st->status), epi, &st->status, FEMK_TIMEOUT, cptr);
  if (!ok && (threadIdx.x & 31) == 0) st->done = 1;
  double v[1] = {(double)epi.a}, tot[1];
  if (!reduce_finish<1, WPB * 32>(v, partials, &st->ticket, tot)) return;
  step_finish<REFRESH, WPB * 32>(st, tot[0], partials + kPartialsA, ga, odd);
}

// K_B on the CSR copy (plans without a sliced-ELL layout)
template <int L, int U, typename IDX, bool REFRESH>
__global__ void __launch_bounds__(kThreads) k_step32(const int32_t* __restrict__ indptr, const IDX* __restrict__ cols,
                                                    const float* __restrict__ vals, int64_t n,
                                                    const float* __restrict__ r, float* __restrict__ w,
                                                    double* __restrict__ partials, int ga, MixedState* st,
                                                    int odd) {
  if (step_skip(st, REFRESH)) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  StepEpi epi{r, w, 0.f};
  for (int64_t base = warp * RPW * U; base < n; base += nwarps * RPW * U) {
    float sv[U];
    int64_t rows[U];
    csr_rows_g<L, U, float, IDX>(indptr, cols, vals, checked(GatherX<float>{r}, n, &st->status), n, base, lane, sv,
                                 rows);
#pragma unroll
    for (int k = 0; k < U; ++k)
      if (rows[k] < n && sub == 0) epi(rows[k], sv[k]);
  }
  double v[1] = {(double)epi.a}, tot[1];
  if (!reduce_finish<1>(v, partials, &st->ticket, tot)) return;
  step_finish<REFRESH, kThreads>(st, tot[0], partials + kPartialsA, ga, odd);
}

// K_A: p = r + beta p; s = w + beta s; r -= alpha s; block partials of <p, s>, <r, s>, <r, r>
// (+ <r, D r> on odd steps) for the next K_B (no grid-wide wait here). Steps alternate within a chunk
// (16 steps, so a chunk starts on an even step): an even step owes its e += alpha p, and the next
// odd step pays both at once from values it reads anyway,
//     e += alpha' p' + alpha p = (alpha' + alpha beta) p' + alpha r    (p = r + beta p', r before the update),
// so e moves every other step, and D (for the stop test's <r, D r>) only on odd steps. All vectors
// are plan-owned and 16-byte aligned: four rows per load.
template <bool ODD>
__device__ __forceinline__ void mx_one(float alpha, float beta, float c1, float w, float d, float& p, float& s,
                                       float& e, float& r, float (&a)[4]) {
  if (ODD) e = fmaf(c1, p, fmaf(alpha, r, e));
  p = fmaf(beta, p, r);
  s = fmaf(beta, s, w);
  r = fmaf(-alpha, s, r);
  a[0] = fmaf(p, s, a[0]);
  a[1] = fmaf(r, s, a[1]);
  a[2] = fmaf(r, r, a[2]);
  if (ODD) a[3] = fmaf(r * r, d, a[3]);
}

template <bool ODD>
__global__ void __launch_bounds__(kThreads) k_mixed_update(int64_t n, const float* __restrict__ w, float* __restrict__ p,
                                                          float* __restrict__ s, float* __restrict__ e,
                                                          float* __restrict__ r, const float* __restrict__ dd,
                                                          double* __restrict__ pa, const MixedState* st) {
  if (st->done || st->hold) return;
  const float alpha = (float)st->alpha, beta = (float)st->beta;
  const float c1 = (float)(st->alpha_pend + st->alpha * st->beta);
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  const int64_t n4 = n >> 2;
  const float4* w4 = reinterpret_cast<const float4*>(w);
  float4* p4 = reinterpret_cast<float4*>(p);
  float4* s4 = reinterpret_cast<float4*>(s);
  float4* e4 = reinterpret_cast<float4*>(e);
  float4* r4 = reinterpret_cast<float4*>(r);
  const float4* d4 = reinterpret_cast<const float4*>(dd);
  float a[4] = {0.f, 0.f, 0.f, 0.f};
  for (int64_t i = tid; i < n4; i += nt) {
    float4 pp = p4[i], ss = s4[i], rr = r4[i];
    const float4 ww = w4[i];
    float4 ee = make_float4(0.f, 0.f, 0.f, 0.f), d = ee;
    if (ODD) {
      ee = e4[i];
      d = d4[i];
    }
    mx_one<ODD>(alpha, beta, c1, ww.x, d.x, pp.x, ss.x, ee.x, rr.x, a);
    mx_one<ODD>(alpha, beta, c1, ww.y, d.y, pp.y, ss.y, ee.y, rr.y, a);
    mx_one<ODD>(alpha, beta, c1, ww.z, d.z, pp.z, ss.z, ee.z, rr.z, a);
    mx_one<ODD>(alpha, beta, c1, ww.w, d.w, pp.w, ss.w, ee.w, rr.w, a);
    p4[i] = pp;
    s4[i] = ss;
    r4[i] = rr;
    if (ODD) e4[i] = ee;
  }
  for (int64_t i = 4 * n4 + tid; i < n; i += nt) {
    float ei = ODD ? e[i] : 0.f;
    mx_one<ODD>(alpha, beta, c1, w[i], ODD ? dd[i] : 0.f, p[i], s[i], ei, r[i], a);
    if (ODD) e[i] = ei;
  }
  double v[4] = {(double)a[0], (double)a[1], (double)a[2], (double)a[3]};
  block_sum<4, kThreads>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) pa[(int64_t)blockIdx.x * 4 + j] = v[j];
  }
}

// x += S (e + alpha_pend p); e = 0 (only at a requested update; the owed term of an even last step
// is paid here)
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ e, const float* __restrict__ p,
                       const float* __restrict__ sc, const MixedState* st) {
  if (st->done || st->need_update != 1) return;
  const float ap = (float)st->alpha_pend;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += (double)sc[i] * (double)fmaf(ap, p[i], e[i]);
    e[i] = 0.f;
  }
}

// r64 = b - A64 x; r^ = fp32(S r64); <r^, r^>, <r64, r64> (+ <b, b> at init, + <p, s>, <r^, s> after)
template <int L, int U, bool INIT>
__global__ void __launch_bounds__(kThreads) k_true_resid(const int32_t* __restrict__ indptr,
                                                        const int32_t* __restrict__ indices,
                                                        const double* __restrict__ vals, int64_t n,
                                                        const double* __restrict__ x, const double* __restrict__ b,
                                                        const double* __restrict__ dinv, float* __restrict__ r,
                                                        const float* __restrict__ p, const float* __restrict__ s,
                                                        double* __restrict__ partials, MixedState* st, double tol2,
                                                        double atol2) {
  if (!INIT && (st->done || st->need_update != 1)) return;
  const int lane = threadIdx.x & 31, sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;
  double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
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
      const float rf = (float)(sqrt(dinv[row]) * r64);
      r[row] = rf;
      a[0] += (double)rf * (double)rf;
      a[1] += r64 * r64;
      if (INIT) {
        a[2] += bi * bi;
      } else {
        const float si = s[row];
        a[3] += (double)p[row] * (double)si;
        a[4] += (double)rf * (double)si;
      }
    }
  }
  double tot[5];
  if (!reduce_finish<5>(a, partials, &st->ticket, tot)) return;
  if (threadIdx.x) return;
  st->outer += 1;
  st->alpha_pend = 0.0;  // k_fold paid it
  st->rr64 = tot[1];
  st->rr_since = tot[1];
  st->rr = tot[1];
  st->ps = tot[3];
  st->rs = tot[4];
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
  st->need_update = 2;  // the refresh step forms w = A^ r^, beta and alpha
  st->hold = 1;
}

template <bool INIT>
void launch_true_resid(const femk_plan* p, const double* vals, const double* x, const double* b, const double* dinv,
                       float* r, const float* pv, const float* sv, MixedState* st, double tol2, double atol2,
                       cudaStream_t s) {
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    const int grid = wave_grid(k_true_resid<L, U, INIT>, kThreads, p);
    k_true_resid<L, U, INIT><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
        p->indptr, p->indices, vals, p->n, x, b, dinv, r, pv, sv, p->partials, st, tol2, atol2);
  });
}

// grid of K_A (fixed per plan: K_B's last block reads this many block partials)
int update_grid(const femk_plan* p) { return vec_grid(k_mixed_update<true>, kThreads, p); }

template <int S, int WPB, int WMAX, bool REFRESH>
bool launch_step32_bulk_cfg(const femk_plan* p, const float* r, float* w, MixedState* st, cudaStream_t s, bool prime,
                            int odd) {
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
      p->n, p->n_slices, r, w, p->partials, update_grid(p), st, (const int64_t*)(tab ? p->sell_cuptr : nullptr), odd);
  return true;
}

// bulk-copy K_B in the plan's configuration (bulk32_cfg: 10 * stages + warps per block)
// prime = true only sets the kernel attribute and reads the occupancy (before a graph capture)
template <bool REFRESH>
bool launch_step32_bulk(const femk_plan* p, const float* r, float* w, MixedState* st, cudaStream_t s,
                        bool prime = false, int odd = 0) {
  if (!p->bulk32_cfg || !p->sell_vals32 || !p->sell_c16 || p->max_row > 32) return false;
  if (((uintptr_t)p->sell_vals32 & 15u) || ((uintptr_t)p->sell_c16 & 15u)) return false;
  if (p->sell_cu && ((uintptr_t)p->sell_cu & 15u)) return false;
  // ring stages sized for the widest row: 8 (2-D P1 triangles), 16 (P1 tetrahedra), 32
  const int wsel = p->max_row <= 8 ? 8 : (p->max_row <= 16 ? 16 : 32);
#define FEMK_BULK_CFG(code, S, WPB)                                                             \
  case code:                                                                                    \
    return wsel == 8    ? launch_step32_bulk_cfg<S, WPB, 8, REFRESH>(p, r, w, st, s, prime, odd)  \
           : wsel == 16 ? launch_step32_bulk_cfg<S, WPB, 16, REFRESH>(p, r, w, st, s, prime, odd) \
                        : launch_step32_bulk_cfg<S, WPB, 32, REFRESH>(p, r, w, st, s, prime, odd);
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

// K_B in the plan's layout; odd: the parity of the step (normal steps; 0 for a refresh)
template <bool REFRESH>
void launch_step32(const femk_plan* p, const float* r, float* w, MixedState* st, cudaStream_t s, int odd = 0) {
  if (launch_step32_bulk<REFRESH>(p, r, w, st, s, false, odd)) return;
  const int ga = update_grid(p);
  if (p->sell_vals32) {
    if (p->sell_c16) {
      auto k = k_step32_sell<int16_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(
          p->sell_ptr, p->sell_c16, p->sell_vals32, p->n, p->n_slices, r, w, p->partials, ga, st, odd);
    } else {
      auto k = k_step32_sell<int32_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(
          p->sell_ptr, p->sell_cols, p->sell_vals32, p->n, p->n_slices, r, w, p->partials, ga, st, odd);
    }
    return;
  }
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    if (p->cols16) {
      auto k = k_step32<L, U, int16_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(p->indptr, p->cols16, p->vals32,
                                                                                  p->n, r, w, p->partials, ga, st, odd);
    } else {
      auto k = k_step32<L, U, int32_t, REFRESH>;
      k<<<::femk::counted_launch() + wave_grid(k, kThreads, p), kThreads, 0, s>>>(p->indptr, p->indices, p->vals32,
                                                                                  p->n, r, w, p->partials, ga, st, odd);
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
  (void)launch_step32_bulk<false>(p, nullptr, nullptr, nullptr, nullptr, true);
  (void)launch_step32_bulk<true>(p, nullptr, nullptr, nullptr, nullptr, true);
  (void)update_grid(p);
  (void)wave_grid(k_fold, 256, p);
}

struct MixedPtrs {
  float *r, *w, *pv, *s, *e, *sc, *dd;
  MixedState* st;
};

MixedPtrs mixed_ptrs(const femk_plan* p) {
  const int64_t vs = p->vstride;
  MixedPtrs m;
  m.r = p->work32;
  m.w = m.r + vs;
  m.pv = m.w + vs;
  m.s = m.pv + vs;
  m.e = m.s + vs;
  m.sc = m.e + vs;
  m.dd = m.sc + vs;
  m.st = (MixedState*)p->work64b;
  return m;
}

// one chunk: kChunk inner iterations, then the (conditional) reliable update and refresh step
int enqueue_mixed_chunk(const femk_plan* p, const double* vals, const double* b, double* x, const double* dinv,
                        cudaStream_t s) {
  const MixedPtrs m = mixed_ptrs(p);
  const int64_t n = p->n;
  const int ga = update_grid(p);
  for (int it = 0; it < kChunk; ++it) {
    const int odd = it & 1;  // a chunk has an even number of steps, so it starts on an even one
    auto ka = odd ? k_mixed_update<true> : k_mixed_update<false>;
    ka<<<::femk::counted_launch() + ga, kThreads, 0, s>>>(n, m.w, m.pv, m.s, m.e, m.r, m.dd, p->partials + kPartialsA,
                                                         m.st);
    launch_step32<false>(p, m.r, m.w, m.st, s, odd);
  }
  k_fold<<<::femk::counted_launch() + wave_grid(k_fold, 256, p), 256, 0, s>>>(n, x, m.e, m.pv, m.sc, m.st);
  launch_true_resid<false>(p, vals, x, b, dinv, m.r, m.pv, m.s, m.st, 0.0, 0.0, s);
  launch_step32<true>(p, m.r, m.w, m.st, s);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int ensure_mixed(femk_plan* p) {
  FEMK_TRY(ensure_workspace(p));
  if (!p->work32) FEMK_CUDA_TRY(cudaMalloc(&p->work32, sizeof(float) * kWork32Vectors * p->vstride));
  if (p->use_sell && p->sell_cols) {
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

int ensure_mixed_graph(femk_plan* p, const double* vals, const double* b, double* x, const double* dinv) {
  // every buffer the captured kernels read is allocated by ensure_mixed before this point
  if (!p->work32 || !p->work64b || !(p->sell_vals32 || p->vals32)) {
    set_error("femk_pcg_mixed: workspace missing at graph capture");
    return FEMK_EINVAL;
  }
  const void* key[5] = {vals, b, x, p->sell_vals32 ? (const void*)p->sell_vals32 : (const void*)p->vals32, dinv};
  bool same = p->mx_exec != nullptr;
  for (int i = 0; i < 5; ++i) same = same && key[i] == p->mx_key[i];
  if (same) return FEMK_OK;
  prime_mixed(p);
  cudaGraph_t g = nullptr;
  set_capturing(true);
  cudaError_t e = cudaStreamBeginCapture(p->mx_stream, cudaStreamCaptureModeThreadLocal);
  int st = e == cudaSuccess ? enqueue_mixed_chunk(p, vals, b, x, dinv, p->mx_stream) : FEMK_ECUDA;
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
  FEMK_CHECK_ARG(kPartialsA + 4 * (int64_t)update_grid(p) <= 4 * (int64_t)p->n_sm * 64 &&
                     (int64_t)p->n_sm * 16 * 5 <= kPartialsA,
                 "femk_pcg_mixed: reduction partials do not fit the plan's buffer");
  const int64_t n = p->n;
  const MixedPtrs m = mixed_ptrs(p);
  cudaStream_t ws = p->mx_stream;
  FEMK_CUDA_TRY(cudaEventRecord(p->mx_ev[2], s));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->mx_ev[2], 0));
  if (p->cg_graph) FEMK_TRY(ensure_mixed_graph(p, vals, b, x, dinv64));
  else prime_mixed(p);
  const int g1 = p->n_sm * 8;
  double* s64 = p->work;  // the FP64 CG workspace is free during a mixed solve
  k_scaling<<<::femk::counted_launch() + g1, 256, 0, ws>>>(dinv64, n, m.sc, m.dd, s64);
  if (p->sell_vals32) {
    const int gg = blocks_for(p->n_slices, 4, p->n_sm * 16);
    const int32_t cap = 32 * (p->max_row > 0 ? p->max_row : 1);
    const size_t smem = sizeof(double) * 4 * (size_t)cap;
    if (p->sell_c16) {
      FEMK_CUDA_TRY(cudaFuncSetAttribute(k_gather_scaled<int16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_gather_scaled<int16_t><<<::femk::counted_launch() + gg, 128, smem, ws>>>(
          p->sell_ptr, p->indptr, p->sell_c16, n, p->n_slices, vals, p->nnz, cap, s64, p->sell_vals32, p->dev_err);
    } else {
      FEMK_CUDA_TRY(cudaFuncSetAttribute(k_gather_scaled<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_gather_scaled<int32_t><<<::femk::counted_launch() + gg, 128, smem, ws>>>(
          p->sell_ptr, p->indptr, p->sell_cols, n, p->n_slices, vals, p->nnz, cap, s64, p->sell_vals32, p->dev_err);
    }
  } else {
    k_scale_csr<<<::femk::counted_launch() + g1, 256, 0, ws>>>(p->indptr, p->indices, n, vals, s64, p->vals32);
  }
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
  launch_true_resid<true>(p, vals, x, b, dinv64, m.r, m.pv, m.s, m.st, tol2, atol2, ws);
  launch_step32<true>(p, m.r, m.w, m.st, ws);  // w = A^ r^, the first alpha
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
      FEMK_TRY(enqueue_mixed_chunk(p, vals, b, x, dinv64, ws));
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
