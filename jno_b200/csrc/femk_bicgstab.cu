// Jacobi-preconditioned BiCGStab with jax.scipy.sparse.linalg.bicgstab semantics (jax 0.10.1), the
// iteration behind jno.solve.bicgstab (jno/solve.py:209-213) and the steady fem.solve() default
// (jno/_fem.py:110-116):
//
//   r = b - A x0;  rhat = r;  p = q = r;  rho = alpha = omega = 1;  k = 0
//   while <r, r> > max(tol^2 <b, b>, atol^2) and 0 <= k < maxiter:
//     rho' = <rhat, r>;  beta = rho' / rho * alpha / omega
//     p = r + beta (p - omega q);  phat = D^-1 p;  q = A phat;  alpha = rho' / <rhat, q>
//     s = r - alpha q;  early = <s, s> < atol2;  shat = D^-1 s;  t = A shat;  omega = <t, s> / <t, t>
//     x += alpha phat (early) | x += alpha phat + omega shat;  r = s (early) | s - omega t
//     k = -10 if rho' == 0, -11 if omega == 0 or alpha == 0, else k + 1;  rho = rho'
//
// Five kernels per iteration, steered by a device-resident BicgState like the CG loop: (1) the
// direction update, (2) q = A phat with <rhat, q>, (3) s and shat with <s, s>, (4) t = A shat with
// <t, s> and <t, t>, (5) the x and r updates with <r, r> and the next <rhat, r>. Dot products finish
// in the last block (deterministic); once the stop test holds every later kernel returns at entry,
// and the host enqueues iterations in chunks replayed as one CUDA graph.
#include <algorithm>
#include <cmath>
#include <string>

#include "femk_bulk.cuh"
#include "femk_internal.cuh"
#include "femk_reduce.cuh"
#include "femk_spmv.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 8;              // iterations per enqueued (graph-replayed) chunk
constexpr int kBulkS = 1, kBulkW = 4;  // bulk-copy SpMV ring: 1 slice buffer per warp, 4 warps (the CG step's)

struct BicgState {
  double rho;     // <rhat, r> of the previous iteration
  double rho_n;   // <rhat, r> of the current residual
  double alpha, omega;
  double rr, ss, atol2, bb;
  double tol2, atol_sq;
  int32_t k;      // jax's iteration counter: negative after a breakdown
  int32_t iters;  // iterations run
  int32_t maxiter;
  int32_t done;
  int32_t status;
  int32_t early;  // <s, s> < atol2 in the current iteration
  uint32_t ticket;
  int32_t pad;
};

struct Vecs {
  double *r, *rhat, *p, *q, *phat, *s, *shat, *t;
};

Vecs vecs_of(const femk_plan* p) {
  const int64_t vs = p->vstride;
  double* w = (double*)p->bicg_ws;
  return {w, w + vs, w + 2 * vs, w + 3 * vs, w + 4 * vs, w + 5 * vs, w + 6 * vs, w + 7 * vs};
}

enum Kind { kInitR = 0, kQ = 1, kT = 2, kResid = 3 };

// Epilogue of each SpMV kind (row, (A v)[row]):
//   kInitR: r = b - A x, rhat = p = q = r; <r, r>, <b, b>
//   kQ    : q = A phat; <rhat, q>
//   kT    : t = A shat; <t, s>, <t, t>
//   kResid: <b - A x, b - A x>, <b, b>
template <int KIND>
struct Epi {
  static constexpr int NV = KIND == kQ ? 1 : 2;
  const double* b;
  Vecs v;
  double* acc;
  __device__ __forceinline__ void operator()(int64_t row, double sv) const {
    if (KIND == kInitR) {
      const double bi = b[row];
      const double ri = bi - sv;
      v.r[row] = ri;
      v.rhat[row] = ri;
      v.p[row] = ri;
      v.q[row] = ri;
      acc[0] += ri * ri;
      acc[1] += bi * bi;
    } else if (KIND == kQ) {
      v.q[row] = sv;
      acc[0] += __ldg(v.rhat + row) * sv;
    } else if (KIND == kT) {
      v.t[row] = sv;
      acc[0] += sv * __ldg(v.s + row);
      acc[1] += sv * sv;
    } else {
      const double bi = b[row];
      const double wi = bi - sv;
      acc[0] += wi * wi;
      acc[1] += bi * bi;
    }
  }
};

template <int KIND>
__device__ __forceinline__ bool kind_skips(const BicgState* st) {
  return (KIND == kQ || KIND == kT) && st->done;
}

template <int KIND, int THREADS>
__device__ __forceinline__ void finish(BicgState* st, double (&acc)[Epi<KIND>::NV], double* partials) {
  constexpr int NV = Epi<KIND>::NV;
  double tot[NV];
  block_reduce_store<NV, THREADS>(acc, partials);
  if (!grid_finish<NV, THREADS>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  if (KIND == kInitR) {
    st->rr = tot[0];
    st->rho_n = tot[0];  // <rhat, r> with rhat = r
    st->bb = tot[1];
    st->atol2 = fmax(st->tol2 * tot[1], st->atol_sq);
    st->rho = st->alpha = st->omega = 1.0;
    st->k = 0;
    st->iters = 0;
    st->early = 0;
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    st->done = (st->status != FEMK_OK || !(tot[0] > st->atol2) || st->maxiter <= 0) ? 1 : 0;
  } else if (KIND == kQ) {
    st->alpha = st->rho_n / tot[0];
  } else if (KIND == kT) {
    st->omega = tot[0] / tot[1];
  } else {
    st->ss = tot[0];
    st->bb = tot[1];
  }
}

// Register-streaming sliced-ELL SpMV with a BiCGStab epilogue.
template <int KIND, typename IDX>
__global__ void __launch_bounds__(kThreads) k_bicg_sell(const int64_t* __restrict__ sptr, const IDX* __restrict__ cols,
                                                       const double* __restrict__ vals, int64_t n, int64_t nslices,
                                                       const double* __restrict__ x, const double* __restrict__ b,
                                                       Vecs v, double* __restrict__ partials, BicgState* st) {
  if (kind_skips<KIND>(st)) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  double acc[Epi<KIND>::NV] = {};
  const Epi<KIND> epi{b, v, acc};
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    if (row >= n) continue;
    const int64_t b0 = __ldg(sptr + sl);
    const int32_t w = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
    epi(row, sell_row<double, IDX, 16>(vals + b0 + lane, cols + b0 + lane, w, (int32_t)row,
                                                        GatherX<double>{x}));
  }
  finish<KIND, kThreads>(st, acc, partials);
}

// The same with the slices streamed into shared memory by bulk copies (femk_bulk.cuh).
template <int KIND, int WMAX>
__global__ void __launch_bounds__(kBulkW * 32) k_bicg_bulk(const int64_t* __restrict__ sptr,
                                                          const int16_t* __restrict__ cols,
                                                          const double* __restrict__ vals, int64_t n, int64_t nslices,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          Vecs v, double* __restrict__ partials, BicgState* st,
                                                          const int64_t* __restrict__ cptr) {
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  using R = BulkRing<double, int16_t, WMAX, kBulkS>;
  if (kind_skips<KIND>(st)) return;
  const int wib = threadIdx.x >> 5;
  double acc[Epi<KIND>::NV] = {};
  const bool ok = sell_bulk_rows<double, int16_t, WMAX, kBulkS>(
      bulk_smem + wib * R::kWarpBytes, sptr, cols, vals, n, nslices, (int64_t)blockIdx.x * kBulkW + wib,
      (int64_t)gridDim.x * kBulkW, GatherXL<double>{x, l2_evict_last()}, Epi<KIND>{b, v, acc}, &st->status,
      FEMK_TIMEOUT, cptr);
  if (!ok && (threadIdx.x & 31) == 0) st->done = 1;
  finish<KIND, kBulkW * 32>(st, acc, partials);
}

// (1) beta = rho' / rho * alpha / omega;  p = r + beta (p - omega q);  phat = D^-1 p
__global__ void __launch_bounds__(kThreads) k_bicg_dir(int64_t n, Vecs v, const double* __restrict__ dinv,
                                                      const BicgState* st) {
  if (st->done) return;
  const double beta = st->rho_n / st->rho * st->alpha / st->omega;
  const double omega = st->omega;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double pi = v.r[i] + beta * (v.p[i] - omega * v.q[i]);
    v.p[i] = pi;
    v.phat[i] = dinv ? dinv[i] * pi : pi;
  }
}

// (3) s = r - alpha q;  shat = D^-1 s;  <s, s> -> early
__global__ void __launch_bounds__(kThreads) k_bicg_s(int64_t n, Vecs v, const double* __restrict__ dinv,
                                                    double* __restrict__ partials, BicgState* st) {
  if (st->done) return;
  const double alpha = st->alpha;
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double si = v.r[i] - alpha * v.q[i];
    v.s[i] = si;
    v.shat[i] = dinv ? dinv[i] * si : si;
    acc[0] += si * si;
  }
  double tot[1];
  block_reduce_store<1>(acc, partials);
  if (!grid_finish<1>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->ss = tot[0];
  st->early = tot[0] < st->atol2 ? 1 : 0;
}

// (5) x and r updates;  <r, r>, <rhat, r>;  breakdown codes, counter and stop test
__global__ void __launch_bounds__(kThreads) k_bicg_xr(int64_t n, double* __restrict__ x, Vecs v,
                                                     double* __restrict__ partials, BicgState* st) {
  if (st->done) return;
  const double alpha = st->alpha, omega = st->omega;
  const bool early = st->early != 0;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double si = v.s[i];
    double ri;
    if (early) {
      x[i] = x[i] + alpha * v.phat[i];
      ri = si;
    } else {
      x[i] = x[i] + (alpha * v.phat[i] + omega * v.shat[i]);
      ri = si - omega * v.t[i];
    }
    v.r[i] = ri;
    acc[0] += ri * ri;
    acc[1] += __ldg(v.rhat + i) * ri;
  }
  double tot[2];
  block_reduce_store<2>(acc, partials);
  if (!grid_finish<2>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->iters += 1;
  if (st->rho_n == 0.0)
    st->k = -10;
  else if (st->omega == 0.0 || st->alpha == 0.0)
    st->k = -11;
  else
    st->k += 1;
  st->rho = st->rho_n;
  st->rho_n = tot[1];
  st->rr = tot[0];
  if (!isfinite(tot[0]) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(tot[0] > st->atol2) || st->k >= st->maxiter || st->k < 0) {
    st->done = 1;
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
template <int KIND, int WMAX>
bool launch_bulk_kind(const femk_plan* p, const double* x, const double* b, const Vecs& v, BicgState* st,
                      cudaStream_t s, bool prime) {
  auto kern = k_bicg_bulk<KIND, WMAX>;
  constexpr int kSmem = kBulkW * BulkRing<double, int16_t, WMAX, kBulkS>::kWarpBytes;
  static int per_sm = -1;
  if (per_sm < 0) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBulkW * 32, kSmem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
  }
  if (per_sm <= 0) return false;
  if (prime) return true;
  const bool tab = p->sell_cu != nullptr;
  kern<<<counted_launch() + p->n_sm * std::min(per_sm, 16), kBulkW * 32, kSmem, s>>>(
      p->sell_ptr, tab ? p->sell_cu : p->sell_c16, p->sell_vals, p->n, p->n_slices, x, b, v, p->partials, st,
      tab ? p->sell_cuptr : nullptr);
  return true;
}

bool bulk_usable(const femk_plan* p) {
  return p->bulk_cfg != 0 && p->sell_c16 && p->sell64_c16 && p->max_row <= 32 &&
         ((uintptr_t)p->sell_vals & 15u) == 0 && ((uintptr_t)p->sell_c16 & 15u) == 0 &&
         ((uintptr_t)p->sell_cu & 15u) == 0;
}

template <int KIND>
int launch_spmv(const femk_plan* p, const double* x, const double* b, const Vecs& v, BicgState* st, cudaStream_t s,
                bool prime = false) {
  if (bulk_usable(p)) {
    const bool ok = p->max_row <= 8    ? launch_bulk_kind<KIND, 8>(p, x, b, v, st, s, prime)
                    : p->max_row <= 16 ? launch_bulk_kind<KIND, 16>(p, x, b, v, st, s, prime)
                                       : launch_bulk_kind<KIND, 32>(p, x, b, v, st, s, prime);
    if (ok) return FEMK_OK;
  }
  if (p->sell_c16 && p->sell64_c16) {
    auto kern = k_bicg_sell<KIND, int16_t>;
    const int grid = wave_grid(kern, kThreads, p);
    if (!prime)
      kern<<<counted_launch() + grid, kThreads, 0, s>>>(p->sell_ptr, p->sell_c16, p->sell_vals, p->n, p->n_slices, x,
                                                        b, v, p->partials, st);
  } else {
    auto kern = k_bicg_sell<KIND, int32_t>;
    const int grid = wave_grid(kern, kThreads, p);
    if (!prime)
      kern<<<counted_launch() + grid, kThreads, 0, s>>>(p->sell_ptr, p->sell_cols, p->sell_vals, p->n, p->n_slices,
                                                        x, b, v, p->partials, st);
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int enqueue_chunk(const femk_plan* p, double* x, const double* dinv, int iters, cudaStream_t s) {
  const Vecs v = vecs_of(p);
  BicgState* st = (BicgState*)p->bicg_state;
  for (int it = 0; it < iters; ++it) {
    k_bicg_dir<<<counted_launch() + wave_grid(k_bicg_dir, kThreads, p), kThreads, 0, s>>>(p->n, v, dinv, st);
    FEMK_TRY(launch_spmv<kQ>(p, v.phat, nullptr, v, st, s));
    k_bicg_s<<<counted_launch() + wave_grid(k_bicg_s, kThreads, p), kThreads, 0, s>>>(p->n, v, dinv, p->partials, st);
    FEMK_TRY(launch_spmv<kT>(p, v.shat, nullptr, v, st, s));
    k_bicg_xr<<<counted_launch() + wave_grid(k_bicg_xr, kThreads, p), kThreads, 0, s>>>(p->n, x, v, p->partials, st);
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int ensure_bicg(femk_plan* p) {
  FEMK_TRY(ensure_workspace(p));
  if (!p->bicg_ws) FEMK_CUDA_TRY(cudaMalloc(&p->bicg_ws, sizeof(double) * 8 * p->vstride));
  if (!p->bicg_state) FEMK_CUDA_TRY(cudaMalloc(&p->bicg_state, sizeof(BicgState)));
  if (!p->bicg_host) FEMK_CUDA_TRY(cudaMallocHost(&p->bicg_host, 2 * sizeof(BicgState)));
  if (!p->bicg_stream) {
    FEMK_CUDA_TRY(cudaStreamCreateWithFlags(&p->bicg_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 3; ++i) FEMK_CUDA_TRY(cudaEventCreateWithFlags(&p->bicg_ev[i], cudaEventDisableTiming));
  }
  return FEMK_OK;
}

// Capture one chunk into a CUDA graph (re-captured when the caller's x or D^-1 pointer changes).
int ensure_graph(femk_plan* p, double* x, const double* dinv) {
  if (p->bicg_exec && p->bicg_key[0] == x && p->bicg_key[1] == dinv) return FEMK_OK;
  // kernel attributes and occupancies are read before capture begins
  (void)wave_grid(k_bicg_dir, kThreads, p);
  (void)wave_grid(k_bicg_s, kThreads, p);
  (void)wave_grid(k_bicg_xr, kThreads, p);
  const Vecs v = vecs_of(p);
  BicgState* st = (BicgState*)p->bicg_state;
  FEMK_TRY(launch_spmv<kQ>(p, v.phat, nullptr, v, st, nullptr, true));
  FEMK_TRY(launch_spmv<kT>(p, v.shat, nullptr, v, st, nullptr, true));
  cudaGraph_t g = nullptr;
  set_capturing(true);
  cudaError_t e = cudaStreamBeginCapture(p->bicg_stream, cudaStreamCaptureModeThreadLocal);
  int rc = e == cudaSuccess ? enqueue_chunk(p, x, dinv, kChunk, p->bicg_stream) : FEMK_ECUDA;
  const cudaError_t e2 = cudaStreamEndCapture(p->bicg_stream, &g);
  set_capturing(false);
  if (e != cudaSuccess || e2 != cudaSuccess || rc != FEMK_OK) {
    if (g) cudaGraphDestroy(g);
    set_error(std::string("femk_bicgstab: graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    return rc != FEMK_OK ? rc : FEMK_ECUDA;
  }
  if (p->bicg_exec) {
    cudaGraphExecDestroy(p->bicg_exec);
    p->bicg_exec = nullptr;
  }
  const cudaError_t e3 = cudaGraphInstantiate(&p->bicg_exec, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) {
    p->bicg_exec = nullptr;
    set_error(std::string("femk_bicgstab: graph instantiation failed: ") + cudaGetErrorString(e3));
    return FEMK_ECUDA;
  }
  p->bicg_key[0] = x;
  p->bicg_key[1] = dinv;
  return FEMK_OK;
}

__global__ void k_bicg_setup(BicgState* st, double tol2, double atol_sq, int32_t maxiter) {
  st->tol2 = tol2;
  st->atol_sq = atol_sq;
  st->maxiter = maxiter;
  st->ticket = 0u;
  st->done = 0;
}

// One BiCGStab solve on the plan's prepared sliced-ELL operator: x holds x0 on entry. Ends with the
// true-residual SpMV (kResid) and returns the final state in *out (host).
int solve_prepared(femk_plan* p, const double* b, double* x, const double* dinv, double tol, double atol,
                   int32_t maxiter, cudaStream_t ws, BicgState* out) {
  const Vecs v = vecs_of(p);
  BicgState* st = (BicgState*)p->bicg_state;
  BicgState* host = (BicgState*)p->bicg_host;
  k_bicg_setup<<<counted_launch() + 1, 1, 0, ws>>>(st, tol * tol, atol * atol, maxiter);
  FEMK_TRY(launch_spmv<kInitR>(p, x, b, v, st, ws));
  const bool graph = p->cg_graph != 0;
  if (graph) FEMK_TRY(ensure_graph(p, x, dinv));
  // chunks of kChunk iterations; the done flag of chunk c is read while chunk c + 1 runs
  int64_t chunks = 0;
  for (;;) {
    if (graph) {
      FEMK_CUDA_TRY(cudaGraphLaunch(p->bicg_exec, ws));
      count_launches(5 * kChunk);
    } else {
      FEMK_TRY(enqueue_chunk(p, x, dinv, kChunk, ws));
    }
    const int c = (int)(chunks & 1);
    FEMK_CUDA_TRY(cudaMemcpyAsync(host + c, st, sizeof(BicgState), cudaMemcpyDeviceToHost, ws));
    FEMK_CUDA_TRY(cudaEventRecord(p->bicg_ev[1 + c], ws));
    ++chunks;
    if (chunks * kChunk >= (int64_t)maxiter) break;
    if (chunks >= 2) {
      FEMK_CUDA_TRY(cudaEventSynchronize(p->bicg_ev[1 + (c ^ 1)]));
      if (host[c ^ 1].done) break;
    }
  }
  // relative true residual: ||b - A x|| / (||b|| + 1e-30)
  FEMK_TRY(launch_spmv<kResid>(p, x, b, v, st, ws));
  FEMK_CUDA_TRY(cudaMemcpyAsync(host, st, sizeof(BicgState), cudaMemcpyDeviceToHost, ws));
  FEMK_CUDA_TRY(cudaStreamSynchronize(ws));
  *out = host[0];
  return FEMK_OK;
}

// Status of a finished solve (sets the error message).
int solve_status(const BicgState& h, const char* who) {
  if (h.status == FEMK_TIMEOUT) {
    set_error(std::string(who) + ": a bounded device wait gave up");
    return FEMK_TIMEOUT;
  }
  if (h.status == FEMK_NONFINITE) {
    set_error(std::string(who) + ": non-finite value in a reduction");
    return FEMK_NONFINITE;
  }
  if (h.k < 0) {
    set_error(std::string(who) + ": breakdown (" + (h.k == -10 ? "<rhat, r> = 0" : "omega or alpha = 0") + ")");
    return FEMK_BREAKDOWN;
  }
  if (h.rr > h.atol2) {
    set_error(std::string(who) + ": iteration cap reached above tolerance");
    return FEMK_NOT_CONVERGED;
  }
  return FEMK_OK;
}

// rhs = R u + q on the canonical CSR (the theta step's right-hand side): 8 lanes per row, 2 row
// groups per warp
__global__ void __launch_bounds__(kThreads) k_theta_rhs(const int32_t* __restrict__ indptr,
                                                       const int32_t* __restrict__ indices,
                                                       const double* __restrict__ R, const double* __restrict__ u,
                                                       const double* __restrict__ q, int64_t n,
                                                       double* __restrict__ rhs) {
  constexpr int L = 8, U = 2, RPW = 32 / L;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  for (int64_t base = warp * RPW * U; base < n; base += nw * RPW * U) {
    double sv[U];
    int64_t rows[U];
    csr_rows<L, U, double, int32_t>(indptr, indices, R, u, n, base, lane, sv, rows);
#pragma unroll
    for (int k = 0; k < U; ++k)
      if (rows[k] < n && lane % L == 0) rhs[rows[k]] = sv[k] + q[rows[k]];
  }
}

}  // namespace
}  // namespace femk

extern "C" int femk_bicgstab(const femk_plan* pc, const double* vals, const double* b, double* x, const double* dinv,
                             double tol, double atol, int32_t maxiter, int32_t* iters_out, double* relres_out,
                             void* stream) {
  using namespace femk;
  clear_error();
  FEMK_CHECK_ARG(pc && vals && b && x, "femk_bicgstab: plan, vals, b and x are required");
  FEMK_CHECK_ARG(tol >= 0.0 && atol >= 0.0, "femk_bicgstab: tol and atol must be >= 0");
  femk_plan* p = const_cast<femk_plan*>(pc);
  FEMK_CHECK_ARG(p->use_sell && p->sell_cols, "femk_bicgstab: the plan has no sliced-ELL operator");
  FEMK_TRY(ensure_bicg(p));
  cudaStream_t cs = (cudaStream_t)stream;
  cudaStream_t ws = p->bicg_stream;
  // the plan's stream runs after the caller's pending work and hands back at the end
  FEMK_CUDA_TRY(cudaEventRecord(p->bicg_ev[0], cs));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->bicg_ev[0], 0));
  if (!p->sell_vals) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals, sizeof(double) * (p->sell_nnz + 1)));
  FEMK_TRY(femk_prepare_operator(p, vals, ws));
  BicgState h;
  const int rc = solve_prepared(p, b, x, dinv, tol, atol, maxiter, ws, &h);
  FEMK_CUDA_TRY(cudaEventRecord(p->bicg_ev[0], ws));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(cs, p->bicg_ev[0], 0));
  FEMK_TRY(rc);
  if (iters_out) *iters_out = h.iters;
  if (relres_out) *relres_out = std::sqrt(h.ss) / (std::sqrt(h.bb) + 1e-30);
  return solve_status(h, "femk_bicgstab");
}

extern "C" int femk_theta_march(const femk_plan* pc, const double* step_vals, const double* rhs_vals,
                                const double* q, double* u, int32_t nsteps, double tol, int32_t maxiter,
                                double step_check, double* traj, int32_t* iters_out, int32_t* gmres_out,
                                double* relres_out, void* stream) {
  using namespace femk;
  clear_error();
  FEMK_CHECK_ARG(pc && step_vals && rhs_vals && q && u, "femk_theta_march: plan, operators, q and u are required");
  FEMK_CHECK_ARG(nsteps >= 0 && tol >= 0.0 && maxiter >= 0, "femk_theta_march: nsteps, tol and maxiter must be >= 0");
  femk_plan* p = const_cast<femk_plan*>(pc);
  FEMK_CHECK_ARG(p->use_sell && p->sell_cols, "femk_theta_march: the plan has no sliced-ELL operator");
  FEMK_TRY(ensure_bicg(p));
  if (!p->theta_ws) FEMK_CUDA_TRY(cudaMalloc(&p->theta_ws, sizeof(double) * 3 * p->vstride));
  double* dinv = (double*)p->theta_ws;
  double* rhs = dinv + p->vstride;
  double* uprev = rhs + p->vstride;  // the state before the step: the GMRES rescue's x0
  cudaStream_t cs = (cudaStream_t)stream;
  cudaStream_t ws = p->bicg_stream;
  FEMK_CUDA_TRY(cudaEventRecord(p->bicg_ev[0], cs));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->bicg_ev[0], 0));
  // the step operator and its Jacobi inverse once for the whole march (the constant-operator path
  // of jno/utils/solver/solver_api.py:920-927)
  if (!p->sell_vals) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals, sizeof(double) * (p->sell_nnz + 1)));
  FEMK_TRY(femk_prepare_operator(p, step_vals, ws));
  FEMK_TRY(femk_jacobi(p, step_vals, dinv, ws));
  const int rgrid = blocks_for(p->n * 4, kThreads, p->n_sm * 16);
  double worst = 0.0;
  int rc = FEMK_OK;
  for (int32_t k = 0; k < nsteps && rc == FEMK_OK; ++k) {
    k_theta_rhs<<<counted_launch() + rgrid, kThreads, 0, ws>>>(p->indptr, p->indices, rhs_vals, u, q, p->n, rhs);
    rc = cudaGetLastError() == cudaSuccess ? FEMK_OK : FEMK_ECUDA;
    if (rc == FEMK_OK && step_check > 0.0) {
      const cudaError_t e = cudaMemcpyAsync(uprev, u, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, ws);
      if (e != cudaSuccess) {
        set_error(std::string("femk_theta_march: ") + cudaGetErrorString(e));
        rc = FEMK_ECUDA;
      }
    }
    BicgState h;
    if (rc == FEMK_OK) rc = solve_prepared(p, rhs, u, dinv, tol, 0.0, maxiter, ws, &h);
    if (rc != FEMK_OK) break;
    if (iters_out) iters_out[k] = h.iters;
    if (gmres_out) gmres_out[k] = 0;
    const int sst = solve_status(h, "femk_theta_march");
    // the reference ignores the step solve's own status: its step check decides. Without the check
    // (the solver-slot path) the status stands; a bounded device wait that gave up always does.
    if (sst == FEMK_TIMEOUT || (sst != FEMK_OK && !(step_check > 0.0))) {
      rc = sst;
      set_error(std::string(femk_last_error_string()) + " (step " + std::to_string(k) + ")");
      break;
    }
    // the step check of backend_blocks.py:402-413: ||S u - rhs|| / max(||rhs||, eps) below
    // max(1e-9, 1e4 eps) for the default step solve; a step that fails it (a NaN residual included)
    // is re-solved from x0 = the previous state by GMRES (tol max(1e-10, 100 eps), restart min(n, 40),
    // the step's Jacobi M, jax's cap of 10 n restart cycles). step_check <= 0 skips it (the
    // solver-slot path, solver_api.py:929-945)
    const double rel = std::sqrt(h.ss) / std::max(std::sqrt(h.bb), 2.220446049250313e-16);
    if (std::isfinite(rel)) worst = std::max(worst, rel);
    if (step_check > 0.0 && (sst != FEMK_OK || !(rel < step_check))) {
      if (!std::isfinite(rel)) worst = rel;
      clear_error();
      FEMK_CUDA_TRY(cudaMemcpyAsync(u, uprev, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, ws));
      GmresInfo gi;
      rc = gmres_run(p, true, nullptr, rhs, u, dinv, 1e-10, 0.0, (int)std::min<int64_t>(p->n, 40), 10 * p->n, ws,
                     &gi);
      if (gmres_out) gmres_out[k] = (int32_t)std::min<int64_t>(gi.steps, INT32_MAX);
      if (rc != FEMK_OK) {
        const std::string why = femk_last_error_string();
        set_error("femk_theta_march: step " + std::to_string(k) + " failed the residual check (" + std::to_string(rel) +
                  " >= " + std::to_string(step_check) + ") and its GMRES rescue failed: " + why);
        break;
      }
    }
    if (rc != FEMK_OK) break;
    if (traj) {
      const cudaError_t e = cudaMemcpyAsync(traj + (int64_t)k * p->n, u, sizeof(double) * p->n,
                                            cudaMemcpyDeviceToDevice, ws);
      if (e != cudaSuccess) {
        set_error(std::string("femk_theta_march: ") + cudaGetErrorString(e));
        rc = FEMK_ECUDA;
      }
    }
  }
  if (relres_out) *relres_out = worst;
  FEMK_CUDA_TRY(cudaEventRecord(p->bicg_ev[0], ws));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(cs, p->bicg_ev[0], 0));
  return rc;
}
