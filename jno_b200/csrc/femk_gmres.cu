// Restarted GMRES with jax.scipy.sparse.linalg.gmres semantics (jax 0.10.1, solve_method="batched"),
// the iteration behind jno.solve.gmres (jno/solve.py:216-221) and the rescue of a theta step that
// fails its residual check (jno/utils/solver/backend_blocks.py:402-413). With M the Jacobi inverse
// (or the identity):
//
//   m = min(restart, n);  atol' = max(tol ||b||, atol);  ptol = ||M b|| min(1, atol' / ||b||)
//   w, beta = normalize(M (b - A x0))
//   while beta > ptol and cycles < maxiter:
//     V_0 = w;  H = eye(m, m + 1)                 (row j of H is column j of the Hessenberg matrix)
//     for j < m, until breakdown:
//       v = M A V_j;  v0 = ||v||;  one classical Gram-Schmidt pass against V
//       V_{j+1}, H[j, j+1] = normalize(v, threshold eps v0);  H[j, :j+1] = the projections
//     y = (H H^T)^-1 H (beta e_0)                 (Cholesky: the normal equations of the (m+1) x m LSQ)
//     x += V[:, :m] y;  w, beta = normalize(M (b - A x))   (columns past a breakdown are zero in jax)
//
// normalize(v, t) = (v / ||v||, ||v||) if ||v|| > t (default t = eps), else (0, 0). Vectors and the
// Krylov basis live in HBM (the basis as m + 1 contiguous vectors of the plan's vector stride); every
// reduction is a fixed-grid two-stage sum (block partials, then one block per column in block order),
// so repeated solves are bitwise reproducible. The host steers each cycle: it reads every Arnoldi
// step's projections and norms (one synchronisation per Gram-Schmidt pass) and solves the small
// least-squares problem itself.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "femk_internal.cuh"
#include "femk_reduce.cuh"

namespace femk {
namespace {

constexpr int kGmThreads = 256;
constexpr int kGmCols = 8;   // basis columns per projection launch
constexpr int kGmMaxM = 64;  // largest restart length
constexpr int kGmGroups = (kGmMaxM + kGmCols) / kGmCols;  // projection partial groups + one norm group

__global__ void __launch_bounds__(kGmThreads) k_gm_norms(const double* __restrict__ b, const double* __restrict__ dinv,
                                                         int64_t n, double* __restrict__ part) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    const double bi = b[i];
    const double mb = dinv ? dinv[i] * bi : bi;
    acc[0] += mb * mb;
    acc[1] += bi * bi;
  }
  block_reduce_store<2>(acc, part);
}

// r = M (b - q) with q = A x; partials of <r, r> and <b - q, b - q>
__global__ void __launch_bounds__(kGmThreads) k_gm_resid(const double* __restrict__ b, const double* __restrict__ q,
                                                         const double* __restrict__ dinv, int64_t n,
                                                         double* __restrict__ r, double* __restrict__ part) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    const double d = b[i] - q[i];
    const double ri = dinv ? dinv[i] * d : d;
    r[i] = ri;
    acc[0] += ri * ri;
    acc[1] += d * d;
  }
  block_reduce_store<2>(acc, part);
}

// w = M w in place; partial of <w, w>
__global__ void __launch_bounds__(kGmThreads) k_gm_precond(double* __restrict__ w, const double* __restrict__ dinv,
                                                           int64_t n, double* __restrict__ part) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    const double wi = dinv ? dinv[i] * w[i] : w[i];
    w[i] = wi;
    acc[0] += wi * wi;
  }
  block_reduce_store<1>(acc, part);
}

// partials of <V_{j0 + c}, w> for c < nc <= kGmCols
__global__ void __launch_bounds__(kGmThreads) k_gm_project(const double* __restrict__ V, int64_t ld, int j0, int nc,
                                                           const double* __restrict__ w, int64_t n,
                                                           double* __restrict__ part) {
  double acc[kGmCols];
#pragma unroll
  for (int c = 0; c < kGmCols; ++c) acc[c] = 0.0;
  const double* base = V + (int64_t)j0 * ld;
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    const double wi = w[i];
#pragma unroll
    for (int c = 0; c < kGmCols; ++c)
      if (c < nc) acc[c] += base[(int64_t)c * ld + i] * wi;
  }
  block_reduce_store<kGmCols>(acc, part);
}

// w -= sum_{c < nc} h[c] V_c; partial of <w, w>
__global__ void __launch_bounds__(kGmThreads) k_gm_orth(const double* __restrict__ V, int64_t ld,
                                                        const double* __restrict__ h, int nc, double* __restrict__ w,
                                                        int64_t n, double* __restrict__ part) {
  __shared__ double hs[kGmMaxM + 1];
  for (int c = threadIdx.x; c < nc; c += kGmThreads) hs[c] = h[c];
  __syncthreads();
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    double s = 0.0;
    for (int c = 0; c < nc; ++c) s += V[(int64_t)c * ld + i] * hs[c];
    const double wi = w[i] - s;
    w[i] = wi;
    acc[0] += wi * wi;
  }
  block_reduce_store<1>(acc, part);
}

// x += V[:, :m] y
__global__ void __launch_bounds__(kGmThreads) k_gm_update(const double* __restrict__ V, int64_t ld,
                                                          const double* __restrict__ y, int m, double* __restrict__ x,
                                                          int64_t n) {
  __shared__ double ys[kGmMaxM];
  for (int c = threadIdx.x; c < m; c += kGmThreads) ys[c] = y[c];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads) {
    double s = 0.0;
    for (int c = 0; c < m; ++c) s += V[(int64_t)c * ld + i] * ys[c];
    x[i] = x[i] + s;
  }
}

// dst = src / s (s > 0), or dst = 0 (s == 0: a normalised zero vector)
__global__ void __launch_bounds__(kGmThreads) k_gm_div(const double* __restrict__ src, double s,
                                                       double* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)kGmThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kGmThreads)
    dst[i] = s > 0.0 ? src[i] / s : 0.0;
}

// out[c] = sum over blocks of the partials of column c, in block order. A launch that stored
// `stride` values per block keeps column c in group c / stride at offset c % stride.
__global__ void __launch_bounds__(kGmThreads) k_gm_colsum(const double* __restrict__ part, int nblk, int stride,
                                                          double* __restrict__ out) {
  const int c = blockIdx.x;
  const double* base = part + (int64_t)(c / stride) * nblk * stride + (c % stride);
  double v[1] = {0.0};
  for (int bk = threadIdx.x; bk < nblk; bk += kGmThreads) v[0] += base[(int64_t)bk * stride];
  block_reduce_store<1>(v, out);
}

struct Gm {
  femk_plan* p;
  const double* vals;  // canonical CSR values, used when the plan has no prepared sliced-ELL operator
  bool sell;
  const double* dinv;
  cudaStream_t s;
  int grid;
  double *V, *w, *q, *part, *small;  // small: projections [0, 65), <w, w> at 65, y at [2*65, 3*65)
  int64_t ld;
};

int gm_spmv(const Gm& g, const double* x, double* y) {
  return g.sell ? femk_spmv_prepared(g.p, x, y, g.s) : femk_spmv(g.p, g.vals, x, y, g.s);
}

// sums ncol columns of the partials into small + off; copies them to `host` (synchronising) when given
int gm_sum(const Gm& g, const double* part, int ncol, int stride, int off, double* host) {
  k_gm_colsum<<<counted_launch() + ncol, kGmThreads, 0, g.s>>>(part, g.grid, stride, g.small + off);
  FEMK_CUDA_TRY(cudaGetLastError());
  if (host) {
    FEMK_CUDA_TRY(cudaMemcpyAsync(host, g.small + off, sizeof(double) * ncol, cudaMemcpyDeviceToHost, g.s));
    FEMK_CUDA_TRY(cudaStreamSynchronize(g.s));
  }
  return FEMK_OK;
}

// M (b - A x) normalised into dst; beta = its norm (0 at or under eps, non-finite kept), rr = ||b - A x||^2
int gm_residual(const Gm& g, const double* b, const double* x, double* dst, double* beta, double* rr) {
  FEMK_TRY(gm_spmv(g, x, g.q));
  k_gm_resid<<<counted_launch() + g.grid, kGmThreads, 0, g.s>>>(b, g.q, g.dinv, g.p->n, g.w, g.part);
  FEMK_CUDA_TRY(cudaGetLastError());
  double t[2];
  FEMK_TRY(gm_sum(g, g.part, 2, 2, 0, t));
  const double nrm = std::sqrt(t[0]);
  // a NaN / Inf residual stays non-finite (NaN > eps is false and would read as convergence)
  *beta = !std::isfinite(nrm) ? nrm : (nrm > 2.220446049250313e-16 ? nrm : 0.0);
  *rr = t[1];
  k_gm_div<<<counted_launch() + g.grid, kGmThreads, 0, g.s>>>(g.w, *beta, dst, g.p->n);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

// Cholesky solve of the m x m system G y = r (G symmetric positive definite, row-major, overwritten);
// false when a pivot is not > 0
bool cholesky_solve(std::vector<double>& G, int m, std::vector<double>& r) {
  for (int j = 0; j < m; ++j) {
    double d = G[(size_t)j * m + j];
    for (int k = 0; k < j; ++k) d -= G[(size_t)j * m + k] * G[(size_t)j * m + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    G[(size_t)j * m + j] = d;
    for (int i = j + 1; i < m; ++i) {
      double v = G[(size_t)i * m + j];
      for (int k = 0; k < j; ++k) v -= G[(size_t)i * m + k] * G[(size_t)j * m + k];
      G[(size_t)i * m + j] = v / d;
    }
  }
  for (int i = 0; i < m; ++i) {
    double v = r[i];
    for (int k = 0; k < i; ++k) v -= G[(size_t)i * m + k] * r[k];
    r[i] = v / G[(size_t)i * m + i];
  }
  for (int i = m - 1; i >= 0; --i) {
    double v = r[i];
    for (int k = i + 1; k < m; ++k) v -= G[(size_t)k * m + i] * r[k];
    r[i] = v / G[(size_t)i * m + i];
  }
  return true;
}

int ensure_gmres(femk_plan* p, int m, int grid) {
  const int64_t vs = p->vstride;
  const int64_t need = (int64_t)(m + 3) * vs + (int64_t)grid * kGmCols * kGmGroups + 3 * (kGmMaxM + 1);
  if (p->gm_ws && p->gm_size >= need) return FEMK_OK;
  if (p->gm_ws) {
    cudaFree(p->gm_ws);
    p->gm_ws = nullptr;
    p->gm_size = 0;
  }
  const cudaError_t e = cudaMalloc(&p->gm_ws, sizeof(double) * need);
  if (e != cudaSuccess) {
    p->gm_ws = nullptr;
    set_error(std::string("gmres workspace: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? FEMK_ENOMEM : FEMK_ECUDA;
  }
  p->gm_size = need;
  return FEMK_OK;
}

}  // namespace

int gmres_run(femk_plan* p, bool sell, const double* vals, const double* b, double* x, const double* dinv,
              double tol, double atol, int restart, int64_t maxiter, cudaStream_t s, GmresInfo* info) {
  const int64_t n = p->n;
  const int m = (int)std::min<int64_t>(std::min(restart, kGmMaxM), n);
  *info = GmresInfo{};
  if (m <= 0) return FEMK_OK;
  Gm g;
  g.grid = p->n_sm * 4;
  FEMK_TRY(ensure_gmres(p, m, g.grid));
  g.p = p;
  g.vals = vals;
  g.sell = sell;
  g.dinv = dinv;
  g.s = s;
  g.ld = p->vstride;
  g.V = p->gm_ws;
  g.w = g.V + (int64_t)(m + 1) * g.ld;
  g.q = g.w + g.ld;
  g.part = g.q + g.ld;
  double* norm_part = g.part + (int64_t)kGmMaxM * g.grid;  // partials of <w, w> after a Gram-Schmidt pass
  g.small = g.part + (int64_t)g.grid * kGmCols * kGmGroups;
  const double eps = 2.220446049250313e-16;
  k_gm_norms<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(b, dinv, n, g.part);
  FEMK_CUDA_TRY(cudaGetLastError());
  double nb[2];
  FEMK_TRY(gm_sum(g, g.part, 2, 2, 0, nb));
  const double Mb_norm = std::sqrt(nb[0]), b_norm = std::sqrt(nb[1]);
  if (!std::isfinite(Mb_norm) || !std::isfinite(b_norm)) {
    set_error("gmres: the right-hand side is not finite");
    return FEMK_NONFINITE;
  }
  info->bb = nb[1];
  const double atol_ = std::max(tol * b_norm, atol);
  const double ptol = b_norm > 0.0 ? Mb_norm * std::min(1.0, atol_ / b_norm) : 0.0;
  double beta = 0.0, rr = 0.0;
  FEMK_TRY(gm_residual(g, b, x, g.V, &beta, &rr));
  info->beta = beta;
  info->rr = rr;
  std::vector<double> H((size_t)m * (m + 1)), h(m + 1), h2(m + 1), G((size_t)m * m), y(m);
  while (std::isfinite(beta) && beta > ptol && info->cycles < maxiter) {
    std::fill(H.begin(), H.end(), 0.0);
    for (int i = 0; i < m; ++i) H[(size_t)i * (m + 1) + i] = 1.0;
    int used = 0;  // basis columns V[:, 0..used) written in this cycle (the update reads no others)
    for (int j = 0; j < m; ++j) {
      FEMK_TRY(gm_spmv(g, g.V + (int64_t)j * g.ld, g.w));
      k_gm_precond<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(g.w, dinv, n, norm_part);
      FEMK_CUDA_TRY(cudaGetLastError());
      double v0sq;
      FEMK_TRY(gm_sum(g, norm_part, 1, 1, kGmMaxM + 1, &v0sq));
      const double v0r = std::sqrt(v0sq);
      const double v0 = v0r > eps ? v0r : 0.0;
      const int ncol = j + 1;
      std::fill(h.begin(), h.end(), 0.0);
      double vnorm_sq = v0sq;
      {  // one classical Gram-Schmidt pass: jax's _iterative_classical_gram_schmidt(max_iterations=2)
         // stops after its first pass (its loop runs while k < max_iterations - 1, and k = 1 then)
        for (int j0 = 0; j0 < ncol; j0 += kGmCols)
          k_gm_project<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(
              g.V, g.ld, j0, std::min(kGmCols, ncol - j0), g.w, n, g.part + (int64_t)(j0 / kGmCols) * g.grid * kGmCols);
        FEMK_CUDA_TRY(cudaGetLastError());
        FEMK_TRY(gm_sum(g, g.part, ncol, kGmCols, 0, nullptr));  // this pass's projections into small[0, ncol)
        k_gm_orth<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(g.V, g.ld, g.small, ncol, g.w, n, norm_part);
        FEMK_CUDA_TRY(cudaGetLastError());
        FEMK_CUDA_TRY(cudaMemcpyAsync(h2.data(), g.small, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
        FEMK_TRY(gm_sum(g, norm_part, 1, 1, kGmMaxM + 1, &vnorm_sq));  // synchronises: h2 has landed too
        for (int c = 0; c < ncol; ++c) h[c] += h2[c];
      }
      const double v1r = std::sqrt(vnorm_sq);
      if (!std::isfinite(v1r)) {
        set_error("gmres: a Krylov vector is not finite");
        return FEMK_NONFINITE;
      }
      const double v1 = v1r > eps * v0 ? v1r : 0.0;
      k_gm_div<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(g.w, v1, g.V + (int64_t)(j + 1) * g.ld, n);
      FEMK_CUDA_TRY(cudaGetLastError());
      h[j + 1] = v1;
      for (int c = 0; c <= m; ++c) H[(size_t)j * (m + 1) + c] = h[c];
      info->steps += 1;
      used = j + 1;
      if (v1 == 0.0) break;
    }
    // y = (H H^T)^-1 (H e_0 beta)
    for (int a = 0; a < m; ++a) {
      for (int c = 0; c <= a; ++c) {
        double t = 0.0;
        for (int k = 0; k <= m; ++k) t += H[(size_t)a * (m + 1) + k] * H[(size_t)c * (m + 1) + k];
        G[(size_t)a * m + c] = t;
        G[(size_t)c * m + a] = t;
      }
      y[a] = H[(size_t)a * (m + 1)] * beta;
    }
    if (!cholesky_solve(G, m, y)) {
      set_error("gmres: the least-squares system of a restart cycle is not positive definite");
      return FEMK_BREAKDOWN;
    }
    FEMK_CUDA_TRY(cudaMemcpyAsync(g.small + 2 * (kGmMaxM + 1), y.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
    // y[c] is exactly 0 for c >= used (those rows of H are the identity), but the columns past a
    // breakdown hold an earlier cycle's vectors or never-written memory: 0 * NaN would poison x
    k_gm_update<<<counted_launch() + g.grid, kGmThreads, 0, s>>>(g.V, g.ld, g.small + 2 * (kGmMaxM + 1), used, x, n);
    FEMK_CUDA_TRY(cudaGetLastError());
    FEMK_TRY(gm_residual(g, b, x, g.V, &beta, &rr));
    info->cycles += 1;
    info->beta = beta;
    info->rr = rr;
  }
  if (!std::isfinite(beta)) {
    set_error("gmres: the residual is not finite");
    return FEMK_NONFINITE;
  }
  if (beta > ptol) {
    set_error("gmres: not converged after " + std::to_string(info->cycles) + " restart cycles (" +
              std::to_string(info->steps) + " Arnoldi steps)");
    return FEMK_NOT_CONVERGED;
  }
  return FEMK_OK;
}

}  // namespace femk

extern "C" int femk_gmres(const femk_plan* pc, const double* vals, const double* b, double* x, const double* inv_diag,
                          double tol, double atol, int32_t restart, int64_t maxiter, int32_t* iters_out,
                          int32_t* cycles_out, double* relres_out, void* stream) {
  using namespace femk;
  clear_error();
  FEMK_CHECK_ARG(pc && vals && b && x, "femk_gmres: plan, vals, b and x are required");
  FEMK_CHECK_ARG(tol >= 0.0 && atol >= 0.0, "femk_gmres: tol and atol must be >= 0");
  FEMK_CHECK_ARG(restart >= 1 && restart <= kGmMaxM, "femk_gmres: restart must be in [1, 64]");
  femk_plan* p = const_cast<femk_plan*>(pc);
  cudaStream_t s = (cudaStream_t)stream;
  const bool sell = p->use_sell && p->sell_cols;
  if (sell) FEMK_TRY(femk_prepare_operator(p, vals, s));
  GmresInfo info;
  const int64_t cap = maxiter >= 0 ? maxiter : 10 * p->n;  // negative: jax's default of 10 n restart cycles
  const int rc = gmres_run(p, sell, vals, b, x, inv_diag, tol, atol, restart, cap, s, &info);
  if (iters_out) *iters_out = (int32_t)std::min<int64_t>(info.steps, INT32_MAX);
  if (cycles_out) *cycles_out = (int32_t)std::min<int64_t>(info.cycles, INT32_MAX);
  if (relres_out) *relres_out = std::sqrt(info.rr) / (std::sqrt(info.bb) + 1e-30);
  return rc;
}
