// CSR / matrix-free SpMV and the Jacobi-PCG loop with jax.scipy.sparse.linalg.cg semantics.
//
// Per iteration three kernels run on the caller's stream, all steered by a device-resident
// CgState (no host round trip per iteration):
//   1. q = A p fused with <p, q>              -> alpha = gamma / <p, q>
//   2. x += alpha p; r -= alpha q; z = D^-1 r fused with <r, z>, <r, r>  -> stop test, beta
//   3. p = z + beta p
// Dot products finish in the last block to arrive (fixed grid, fixed order: deterministic).
// Once the stop test holds every later kernel returns at entry, so the host enqueues iterations
// in chunks and only looks at the done flag of the previous chunk while the next one runs.
//
// Replaces jno.solve.cg (jno/solve.py:191-206) -> jax.scipy.sparse.linalg.cg (jax 0.10.1) with
// M = jno.precond.jacobi() (jno/precond.py:106-111) and LinearOperator.mv (solver_api.py:137-148).
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <mutex>
#include <string>

#include "femk_bulk.cuh"
#include "femk_reduce.cuh"
#include "femk_element.cuh"
#include "femk_internal.cuh"
#include "femk_spmv.cuh"
#include "femk_l2.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;  // iterations enqueued between looks at the done flag

enum SpmvMode { kPlain = 0, kCgStep = 1, kInit = 2, kResid = 3 };

// One kernel for every CSR-SpMV use of the solver (L lanes per row, U rows in flight per lane group):
//  kPlain : y = A x
//  kCgStep: q = A p, <p, q>                     (finish: alpha)
//  kInit  : r = b - A x, z = D^-1 r, p = z, <r,z>, <r,r>, <b,b>   (finish: gamma, rr, atol2, done)
//  kResid : w = b - A x, <w,w>, <b,b>           (finish: stored in st->pq / st->bb)
template <int L, int U, int MODE>
__global__ void __launch_bounds__(kThreads) k_csr(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                                 const double* __restrict__ vals, int64_t n, const double* __restrict__ x,
                                                 double* __restrict__ y, const double* __restrict__ b,
                                                 const double* __restrict__ dinv, double* __restrict__ z,
                                                 double* __restrict__ pout, double* __restrict__ partials, CgState* st,
                                                 double tol2, double atol2, int* __restrict__ err) {
  constexpr int NV = MODE == kPlain ? 1 : (MODE == kCgStep ? 1 : (MODE == kInit ? 3 : 2));
  if (MODE == kCgStep && blockIdx.x == 0 && threadIdx.x == 0) st->xpend = 0;  // the last x update is applied
  if (MODE == kCgStep && st->done) return;
  const int lane = threadIdx.x & 31;
  const int sub = lane % L;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  constexpr int RPW = 32 / L;  // rows per lane-group step
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  for (int64_t base = warp * RPW * U; base < n; base += nwarps * RPW * U) {
    double s[U];
    int64_t rows[U];
    csr_rows_g<L, U, double, int32_t>(indptr, indices, vals, checked(GatherX<double>{x}, n, err), n, base, lane, s,
                                      rows);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t row = rows[u];
      if (row >= n || sub != 0) continue;
      if (MODE == kPlain) {
        y[row] = s[u];
      } else if (MODE == kCgStep) {
        y[row] = s[u];
        acc[0] += __ldg(x + row) * s[u];
      } else if (MODE == kInit) {
        const double bi = b[row];
        const double ri = bi - s[u];
        const double zi = dinv ? dinv[row] * ri : ri;
        y[row] = ri;
        z[row] = zi;
        pout[row] = zi;
        acc[0] += ri * zi;
        acc[1] += ri * ri;
        acc[2] += bi * bi;
      } else {
        const double bi = b[row];
        const double wi = bi - s[u];
        acc[0] += wi * wi;
        acc[1] += bi * bi;
      }
    }
  }
  if (MODE == kPlain) return;
  block_reduce_store<NV>(acc, partials);
  double tot[NV];
  if (!grid_finish<NV>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  if (MODE == kCgStep) {
    st->pq = tot[0];
    st->alpha = st->gamma / tot[0];
    if (!isfinite(tot[0])) {
      st->status = FEMK_NONFINITE;
      st->done = 1;
    } else if (!(tot[0] > 0.0)) {
      st->status = FEMK_BREAKDOWN;
      st->done = 1;
    }
  } else if (MODE == kInit) {
    st->gamma = tot[0];
    st->rr = tot[1];
    st->bb = tot[2];
    st->atol2 = fmax(tol2 * tot[2], atol2);
    st->iter = 0;
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    const double rs = st->precond ? tot[1] : tot[0];
    st->done = (!(rs > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
    st->rr_since = tot[1];
    st->beta = 0.0;
    st->xpend = 0;
  } else {
    st->pq = tot[0];
    st->bb = tot[1];
  }
}

// The same modes on the sliced-ELL copy of the operator: one thread per row, 32-row slices.
template <int MODE, typename IDX, int B, int H = 0>
__global__ void __launch_bounds__(kThreads) k_sell(const int64_t* __restrict__ sptr, const IDX* __restrict__ scols,
                                                  const double* __restrict__ svals, int64_t n, int64_t nslices,
                                                  const double* __restrict__ x, double* __restrict__ y,
                                                  const double* __restrict__ b, const double* __restrict__ dinv,
                                                  double* __restrict__ z, double* __restrict__ pout,
                                                  double* __restrict__ partials, CgState* st, double tol2,
                                                  double atol2, int* __restrict__ err) {
  constexpr int NV = MODE == kPlain ? 1 : (MODE == kCgStep ? 1 : (MODE == kInit ? 3 : 2));
  if (MODE == kCgStep && blockIdx.x == 0 && threadIdx.x == 0) st->xpend = 0;  // the last x update is applied
  if (MODE == kCgStep && st->done) return;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    if (row >= n) continue;
    const int64_t b0 = __ldg(sptr + sl);
    const int32_t w = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
    double sv;
    if (H == 1)
      sv = sell_row<double, IDX, B, true>(svals + b0 + lane, scols + b0 + lane, w, (int32_t)row,
                                          checked(GatherXL<double>{x, l2_evict_last()}, n, err));
    else if (H == 2)
      sv = sell_row<double, IDX, B, true>(svals + b0 + lane, scols + b0 + lane, w, (int32_t)row,
                                          checked(GatherX<double>{x}, n, err));
    else if (H == 4)
      sv = sell_row<double, IDX, B, false>(svals + b0 + lane, scols + b0 + lane, w, (int32_t)row,
                                           checked(GatherXL<double>{x, l2_evict_last()}, n, err));
    else
      sv = sell_row<double, IDX, B>(svals + b0 + lane, scols + b0 + lane, w, (int32_t)row,
                                    checked(GatherX<double>{x}, n, err));
    if (MODE == kPlain) {
      y[row] = sv;
    } else if (MODE == kCgStep) {
      y[row] = sv;
      acc[0] += __ldg(x + row) * sv;
    } else if (MODE == kInit) {
      const double bi = b[row];
      const double ri = bi - sv;
      const double zi = dinv ? dinv[row] * ri : ri;
      y[row] = ri;
      z[row] = zi;
      pout[row] = zi;
      acc[0] += ri * zi;
      acc[1] += ri * ri;
      acc[2] += bi * bi;
    } else {
      const double bi = b[row];
      const double wi = bi - sv;
      acc[0] += wi * wi;
      acc[1] += bi * bi;
    }
  }
  if (MODE == kPlain) return;
  block_reduce_store<NV>(acc, partials);
  double tot[NV];
  if (!grid_finish<NV>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  if (MODE == kCgStep) {
    st->pq = tot[0];
    st->alpha = st->gamma / tot[0];
    if (!isfinite(tot[0])) {
      st->status = FEMK_NONFINITE;
      st->done = 1;
    } else if (!(tot[0] > 0.0)) {
      st->status = FEMK_BREAKDOWN;
      st->done = 1;
    }
  } else if (MODE == kInit) {
    st->gamma = tot[0];
    st->rr = tot[1];
    st->bb = tot[2];
    st->atol2 = fmax(tol2 * tot[2], atol2);
    st->iter = 0;
    st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
    const double rs = st->precond ? tot[1] : tot[0];
    st->done = (!(rs > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
    st->rr_since = tot[1];
    st->beta = 0.0;
    st->xpend = 0;
  } else {
    st->pq = tot[0];
    st->bb = tot[1];
  }
}

// The same SpMV (kPlain, kCgStep) with the sliced-ELL stream moved into shared memory by bulk
// copies (femk_bulk.cuh): WPB warps per block, S slices in flight per warp, widths up to WMAX.
template <int MODE, typename IDX, int WMAX, int S, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_sell_bulk(const int64_t* __restrict__ sptr,
                                                       const IDX* __restrict__ scols,
                                                       const double* __restrict__ svals, int64_t n, int64_t nslices,
                                                       const double* __restrict__ x, double* __restrict__ y,
                                                       double* __restrict__ partials, CgState* st, int* err,
                                                       const int64_t* __restrict__ cptr) {
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  constexpr int kWarpBytes = BulkRing<double, IDX, WMAX, S>::kWarpBytes;
  if (MODE == kCgStep) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->xpend = 0;  // the last x update is applied
    if (st->done) return;
  }
  const int wib = threadIdx.x >> 5;
  const int64_t g = (int64_t)blockIdx.x * WPB + wib;
  const int64_t NW = (int64_t)gridDim.x * WPB;
  double acc[1] = {0.0};
  int* errp = MODE == kCgStep ? &st->status : err;
  const bool ok = sell_bulk_rows<double, IDX, WMAX, S>(
      bulk_smem + wib * kWarpBytes, sptr, scols, svals, n, nslices, g, NW,
      checked(GatherXL<double>{x, l2_evict_last()}, n, errp),
      [&](int64_t row, double sv) {
        y[row] = sv;
        if (MODE == kCgStep) acc[0] += __ldg(x + row) * sv;
      },
      errp, FEMK_TIMEOUT, cptr);
  if (MODE == kPlain) return;
  if (!ok && (threadIdx.x & 31) == 0) st->done = 1;
  block_reduce_store<1, WPB * 32>(acc, partials);
  double tot[1];
  if (!grid_finish<1, WPB * 32>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->pq = tot[0];
  st->alpha = st->gamma / tot[0];
  if (!isfinite(tot[0])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(tot[0] > 0.0)) {
    st->status = FEMK_BREAKDOWN;
    st->done = 1;
  }
}

template <typename T>
__global__ void k_sell_gather(const int64_t* __restrict__ sptr, const int32_t* __restrict__ indptr, int64_t n,
                              int64_t nslices, const double* __restrict__ vals, int64_t nnz, int32_t cap,
                              T* __restrict__ out, int* __restrict__ err) {
  extern __shared__ double sg_buf[];
  const int wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  sell_transpose_warp<T>(sg_buf + (int64_t)wib * cap, cap, sptr, indptr, n, nslices, vals, nnz, out,
                         (int64_t)blockIdx.x * wpb + wib, (int64_t)gridDim.x * wpb,
                         [](double v, int64_t, int64_t) { return (T)v; }, err);
}

// x += alpha p; r -= alpha q; z = D^-1 r; <r, z>, <r, r>; stop test; beta.
// VEC: every vector is 16-byte aligned, so two rows move per 16-byte load and each thread keeps
// two such pairs in flight per trip (the plain form is for unaligned caller buffers).
__device__ __forceinline__ void update_one(int64_t i, double alpha, double* __restrict__ x, double* __restrict__ r,
                                           double* __restrict__ z, const double* __restrict__ p,
                                           const double* __restrict__ q, const double* __restrict__ dinv,
                                           double (&acc)[2]) {
  x[i] = x[i] + alpha * p[i];
  const double ri = r[i] - alpha * q[i];
  const double zi = dinv ? dinv[i] * ri : ri;
  r[i] = ri;
  z[i] = zi;
  acc[0] += ri * zi;
  acc[1] += ri * ri;
}

template <bool VEC, bool H = false>
__global__ void __launch_bounds__(kThreads) k_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                    double* __restrict__ z, const double* __restrict__ p,
                                                    const double* __restrict__ q, const double* __restrict__ dinv,
                                                    double* __restrict__ partials, CgState* st) {
  if (st->done) return;
  const double alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  if (VEC) {
    const int64_t n2 = n >> 1;
    double2* x2 = reinterpret_cast<double2*>(x);
    double2* r2 = reinterpret_cast<double2*>(r);
    double2* z2 = reinterpret_cast<double2*>(z);
    const double2* p2 = reinterpret_cast<const double2*>(p);
    const double2* q2 = reinterpret_cast<const double2*>(q);
    const double2* d2 = reinterpret_cast<const double2*>(dinv);
    uint64_t pol = 0;
    if (H) pol = l2_evict_last();
    auto ld = [&](const double2* a) { return H ? ld_last2(a, pol) : *a; };
    auto st2 = [&](double2* a, double2 v) {
      if (H)
        st_last2(a, v, pol);
      else
        *a = v;
    };
    for (int64_t i = tid; i < n2; i += 2 * nt) {
      const int64_t j = i + nt;
      const bool two = j < n2;
      const double2 pa = ld(p2 + i), qa = ld(q2 + i), xa = ld(x2 + i), ra = ld(r2 + i);
      double2 pb = pa, qb = qa, xb = xa, rb = ra, da = make_double2(1.0, 1.0), db = da;
      if (two) {
        pb = ld(p2 + j);
        qb = ld(q2 + j);
        xb = ld(x2 + j);
        rb = ld(r2 + j);
      }
      if (dinv) {
        da = ld(d2 + i);
        if (two) db = ld(d2 + j);
      }
      double2 ro, zo;
      st2(x2 + i, make_double2(xa.x + alpha * pa.x, xa.y + alpha * pa.y));
      ro = make_double2(ra.x - alpha * qa.x, ra.y - alpha * qa.y);
      zo = make_double2(da.x * ro.x, da.y * ro.y);
      st2(r2 + i, ro);
      st2(z2 + i, zo);
      acc[0] += ro.x * zo.x + ro.y * zo.y;
      acc[1] += ro.x * ro.x + ro.y * ro.y;
      if (two) {
        st2(x2 + j, make_double2(xb.x + alpha * pb.x, xb.y + alpha * pb.y));
        ro = make_double2(rb.x - alpha * qb.x, rb.y - alpha * qb.y);
        zo = make_double2(db.x * ro.x, db.y * ro.y);
        st2(r2 + j, ro);
        st2(z2 + j, zo);
        acc[0] += ro.x * zo.x + ro.y * zo.y;
        acc[1] += ro.x * ro.x + ro.y * ro.y;
      }
    }
    if ((n & 1) && tid == 0) update_one(n - 1, alpha, x, r, z, p, q, dinv, acc);
  } else {
    for (int64_t i = tid; i < n; i += nt) update_one(i, alpha, x, r, z, p, q, dinv, acc);
  }
  block_reduce_store<2>(acc, partials);
  double tot[2];
  if (!grid_finish<2>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  const double gamma_new = tot[0];
  st->beta = gamma_new / st->gamma;
  st->gamma = gamma_new;
  st->rr = tot[1];
  st->iter += 1;
  const double rs = st->precond ? tot[1] : gamma_new;
  if (!isfinite(gamma_new) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(rs > st->atol2) || st->iter >= st->maxiter) {
    st->done = 1;
  }
}

// p = z + beta p on plan-owned (16-byte aligned) vectors, two rows per load
template <bool H = false>
__global__ void __launch_bounds__(kThreads) k_pupdate(int64_t n, double* __restrict__ p, const double* __restrict__ z,
                                                     const CgState* st) {
  if (st->done) return;
  const double beta = st->beta;
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  const int64_t n2 = n >> 1;
  double2* p2 = reinterpret_cast<double2*>(p);
  const double2* z2 = reinterpret_cast<const double2*>(z);
  uint64_t pol = 0;
  if (H) pol = l2_evict_last();
  for (int64_t i = tid; i < n2; i += nt) {
    const double2 a = H ? ld_last2(p2 + i, pol) : p2[i];
    const double2 c = H ? ld_last2(z2 + i, pol) : z2[i];
    const double2 o = make_double2(c.x + beta * a.x, c.y + beta * a.y);
    if (H)
      st_last2(p2 + i, o, pol);
    else
      p2[i] = o;
  }
  if ((n & 1) && tid == 0) p[n - 1] = z[n - 1] + beta * p[n - 1];
}

// Split form of the two vector kernels (the default on aligned vectors): z is never stored and x
// is updated in the direction kernel, which reads p once for both uses.
//   k_update_r : r -= alpha q; <r, D^-1 r>, <r, r>; stop test; beta     (reads r, q, D^-1; writes r)
//   k_pupdate_x: x += alpha p; p = D^-1 r + beta p                         (reads x, p, r, D^-1; writes x, p)
// Every value is formed by the same floating-point operations as in k_update + k_pupdate. The
// iteration that meets the stop test still owes its x update: k_update_r raises st->xpend, the
// direction kernel applies x (and p only while the solve runs), and the next CG-step SpMV clears it.
template <bool H>
__global__ void __launch_bounds__(kThreads) k_update_r(int64_t n, double* __restrict__ r, const double* __restrict__ q,
                                                      const double* __restrict__ dinv, double* __restrict__ partials,
                                                      CgState* st) {
  if (st->done) return;
  const double alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  const int64_t n2 = n >> 1;
  double2* r2 = reinterpret_cast<double2*>(r);
  const double2* q2 = reinterpret_cast<const double2*>(q);
  const double2* d2 = reinterpret_cast<const double2*>(dinv);
  uint64_t pol = 0;
  if (H) pol = l2_evict_last();
  auto ld = [&](const double2* a) { return H ? ld_last2(a, pol) : *a; };
  auto one = [&](double2 ra, double2 qa, double2 da, double2* dst) {
    const double2 ro = make_double2(fma(-alpha, qa.x, ra.x), fma(-alpha, qa.y, ra.y));
    const double2 zo = make_double2(da.x * ro.x, da.y * ro.y);
    if (H)
      st_last2(dst, ro, pol);
    else
      *dst = ro;
    acc[0] += ro.x * zo.x + ro.y * zo.y;
    acc[1] += ro.x * ro.x + ro.y * ro.y;
  };
  // four pairs a trip, all loaded before any store (74 registers, 3 blocks per SM): the P1 128^3
  // FP64 solve took 36.2-36.3 ms against 36.7 ms with two, in the same run
  for (int64_t i = tid; i < n2; i += 4 * nt) {
    double2 ra[4], qa[4], da[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t j = i + u * nt;
      da[u] = make_double2(1.0, 1.0);
      if (j < n2) {
        ra[u] = ld(r2 + j);
        qa[u] = ld(q2 + j);
        if (dinv) da[u] = ld(d2 + j);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t j = i + u * nt;
      if (j < n2) one(ra[u], qa[u], da[u], r2 + j);
    }
  }
  if ((n & 1) && tid == 0) {
    const int64_t i = n - 1;
    const double ri = fma(-alpha, q[i], r[i]);
    const double zi = dinv ? dinv[i] * ri : ri;
    r[i] = ri;
    acc[0] += ri * zi;
    acc[1] += ri * ri;
  }
  block_reduce_store<2>(acc, partials);
  double tot[2];
  if (!grid_finish<2>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  const double gamma_new = tot[0];
  st->beta = gamma_new / st->gamma;
  st->gamma = gamma_new;
  st->rr = tot[1];
  st->iter += 1;
  st->xpend = 1;
  const double rs = st->precond ? tot[1] : gamma_new;
  if (!isfinite(gamma_new) || !isfinite(tot[1])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(rs > st->atol2) || st->iter >= st->maxiter) {
    st->done = 1;
  }
}

template <bool H>
__global__ void __launch_bounds__(kThreads) k_pupdate_x(int64_t n, double* __restrict__ x, double* __restrict__ p,
                                                       const double* __restrict__ r, const double* __restrict__ dinv,
                                                       const CgState* st) {
  if (!st->xpend) return;
  const bool dir = !st->done;
  const double alpha = st->alpha, beta = st->beta;
  const int64_t tid = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * kThreads;
  const int64_t n2 = n >> 1;
  double2* x2 = reinterpret_cast<double2*>(x);
  double2* p2 = reinterpret_cast<double2*>(p);
  const double2* r2 = reinterpret_cast<const double2*>(r);
  const double2* d2 = reinterpret_cast<const double2*>(dinv);
  uint64_t pol = 0;
  if (H) pol = l2_evict_last();
  auto ld = [&](const double2* a) { return H ? ld_last2(a, pol) : *a; };
  auto st2 = [&](double2* a, double2 v) {
    if (H)
      st_last2(a, v, pol);
    else
      *a = v;
  };
  if (dir) {
    for (int64_t i = tid; i < n2; i += nt) {
      const double2 pa = ld(p2 + i), xa = ld(x2 + i), ra = ld(r2 + i);
      const double2 da = dinv ? ld(d2 + i) : make_double2(1.0, 1.0);
      st2(x2 + i, make_double2(fma(alpha, pa.x, xa.x), fma(alpha, pa.y, xa.y)));
      st2(p2 + i, make_double2(fma(beta, pa.x, da.x * ra.x), fma(beta, pa.y, da.y * ra.y)));
    }
    if ((n & 1) && tid == 0) {
      const int64_t i = n - 1;
      const double pi = p[i];
      x[i] = fma(alpha, pi, x[i]);
      p[i] = fma(beta, pi, (dinv ? dinv[i] : 1.0) * r[i]);
    }
  } else {
    for (int64_t i = tid; i < n2; i += nt) {
      const double2 pa = ld(p2 + i), xa = ld(x2 + i);
      st2(x2 + i, make_double2(fma(alpha, pa.x, xa.x), fma(alpha, pa.y, xa.y)));
    }
    if ((n & 1) && tid == 0) x[n - 1] = fma(alpha, p[n - 1], x[n - 1]);
  }
}

// ---------------------------------------------------------------------------------------------
// matrix-free operator: y = A x, A the Dirichlet-eliminated stiffness, recomputed per element from
// the vertex coordinates (thread per element, FP64 atomics into y). mcells is the connectivity with
// each Dirichlet DOF d stored as -1 - d, so one load gives the DOF and its mask: a Dirichlet DOF
// contributes x = 0 and receives nothing (its row is the identity, k_dirichlet_identity).
// ---------------------------------------------------------------------------------------------
// (P2 tetrahedra: 6 resident blocks per SM fit the product in 80 registers without spills)
template <int ND>
__global__ void __launch_bounds__(128, ND == 10 ? 6 : 8) k_matfree(const double* __restrict__ xyz,
                                                                   const int32_t* __restrict__ mcells,
                                                 int64_t ntet, const double* __restrict__ param, int mode, double scale,
                                                 const double* __restrict__ x, double* __restrict__ y,
                                                 const CgState* st) {
  constexpr int NV = Cell<ND>::NV;
  if (st && st->done) return;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
    double xe[ND];
    if constexpr (ND == 4) {  // one 16-byte load (mcells is 256-byte aligned, c * 16 bytes in)
      const int4 d4 = __ldg(reinterpret_cast<const int4*>(mcells) + c);
      dof[0] = d4.x;
      dof[1] = d4.y;
      dof[2] = d4.z;
      dof[3] = d4.w;
    } else {
#pragma unroll
      for (int a = 0; a < ND; ++a) dof[a] = __ldg(mcells + c * ND + a);
    }
#pragma unroll
    for (int a = 0; a < ND; ++a) xe[a] = dof[a] >= 0 ? __ldg(x + dof[a]) : 0.0;
    int32_t v[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = dof[i] >= 0 ? dof[i] : -1 - dof[i];
    const double k = coef_of(param, mode, scale, c);
    double ye[ND];
    if constexpr (!Cell<ND>::P2) {
      double P[NV][3];
#pragma unroll
      for (int i = 0; i < NV; ++i)
#pragma unroll
        for (int q = 0; q < 3; ++q) P[i][q] = (q < NV - 1) ? __ldg(xyz + (int64_t)v[i] * 3 + q) : 0.0;
      p1_apply(P, xe, ye);
    } else {
      Geom<NV> T;
      cell_geometry(xyz, v, T);
      double VG[NV][NV];
      gram(T, VG);
      khat_apply<ND>(VG, xe, ye);
    }
#pragma unroll
    for (int a = 0; a < ND; ++a)
      if (dof[a] >= 0) atomicAdd(y + dof[a], k * ye[a]);
  }
}

// Kuhn blocks: six consecutive tetrahedra that split one hexahedron, tet e of a block being the
// corners kuhn_corner(e, 0..3) (corner bit 2 = x, bit 1 = y, bit 0 = z), the layout the structured box
// constructor emits (domain.py KUHN). k_kuhn_corners checks a plan's masked connectivity against it
// block by block and keeps each block's 8 corners; when every block fits, the P1 matrix-free operator
// works a hexahedron at a time (k_matfree_kuhn).
// Tet e is the corners {0, a_e, b_e, 7} with a = (4, 4, 2, 2, 1, 1) and b = (6, 5, 6, 3, 5, 3), packed a
// nibble per tet; in unrolled loops every call folds to a constant.
__host__ __device__ constexpr int kuhn_corner(int e, int j) {
  return j == 0 ? 0 : (j == 3 ? 7 : (((j == 1 ? 0x112244 : 0x353656) >> (4 * e)) & 15));
}

__global__ void k_kuhn_corners(const int32_t* __restrict__ mcells, int64_t nhex, int32_t* __restrict__ corners,
                               int* __restrict__ bad) {
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nhex; h += (int64_t)gridDim.x * blockDim.x) {
    constexpr int32_t kUnset = INT32_MIN;  // a masked id is d >= 0 or -1 - d, never this
    int32_t c[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) c[u] = kUnset;
    bool ok = true;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const int4 d4 = __ldg(reinterpret_cast<const int4*>(mcells) + 6 * h + e);
      const int32_t d[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int u = kuhn_corner(e, j);
        if (c[u] == kUnset)
          c[u] = d[j];
        else
          ok = ok && c[u] == d[j];
      }
    }
    if (!ok) atomicExch(bad, 1);
    int4* o = reinterpret_cast<int4*>(corners) + 2 * h;
    o[0] = make_int4(c[0], c[1], c[2], c[3]);
    o[1] = make_int4(c[4], c[5], c[6], c[7]);
  }
}

// y += A x over whole Kuhn blocks: one thread loads a hexahedron's 8 corners, their coordinates and
// x once (six separate elements load 24 of each), applies the six element operators (p1_apply, the
// local indices compile-time constants) and adds into the 8 corners with 8 atomics in place of 24.
__global__ void __launch_bounds__(128) k_matfree_kuhn(const double* __restrict__ xyz,
                                                      const int32_t* __restrict__ corners, int64_t nhex,
                                                      const double* __restrict__ param, int mode, double scale,
                                                      const double* __restrict__ x, double* __restrict__ y,
                                                      const CgState* st) {
  if (st && st->done) return;
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nhex; h += (int64_t)gridDim.x * blockDim.x) {
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(corners) + 2 * h);
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(corners) + 2 * h + 1);
    const int32_t c[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    double X[8][3], xv[8], ys[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t v = c[u] >= 0 ? c[u] : -1 - c[u];
#pragma unroll
      for (int q = 0; q < 3; ++q) X[u][q] = __ldg(xyz + v * 3 + q);
      xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : 0.0;
      ys[u] = 0.0;
    }
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      double P[4][3], xe[4], ye[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int q = 0; q < 3; ++q) P[i][q] = X[kuhn_corner(e, i)][q];
        xe[i] = xv[kuhn_corner(e, i)];
      }
      p1_apply(P, xe, ye);
      const double k = coef_of(param, mode, scale, 6 * h + e);
#pragma unroll
      for (int i = 0; i < 4; ++i) ys[kuhn_corner(e, i)] += k * ye[i];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (c[u] >= 0) atomicAdd(y + c[u], ys[u]);
  }
}

// the masked connectivity of the matrix-free operator
__global__ void k_mask_cells(const int32_t* __restrict__ cells, int64_t len, const uint8_t* __restrict__ dmask,
                             int32_t* __restrict__ mcells) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = cells[t];
    mcells[t] = dmask[d] ? -1 - d : d;
  }
}

__global__ void k_dirichlet_identity(const int32_t* __restrict__ dlist, int64_t nd, const double* __restrict__ x,
                                     double* __restrict__ y, const CgState* st) {
  if (st && st->done) return;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nd; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = dlist[t];
    y[d] = x[d];
  }
}

template <int ND>
__global__ void k_matfree_diag(const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet,
                               const uint8_t* __restrict__ dmask, const double* __restrict__ param, int mode,
                               double scale, double* __restrict__ d) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dof[a] = __ldg(cells + c * ND + a);
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    double VG[Cell<ND>::NV][Cell<ND>::NV];
    gram(T, VG);
    const double k = coef_of(param, mode, scale, c);
#pragma unroll
    for (int a = 0; a < ND; ++a)
      if (!__ldg(dmask + dof[a])) atomicAdd(d + dof[a], k * khat<ND>(VG, a, a));
  }
}

// The rest of a CG step for the matrix-free operator: <p, q> (q already holds A p)
__global__ void __launch_bounds__(kThreads) k_dot_pq(int64_t n, const double* __restrict__ p, const double* __restrict__ q,
                                                    double* __restrict__ partials, CgState* st) {
  if (st->done) return;
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
    acc[0] += p[i] * q[i];
  block_reduce_store<1>(acc, partials);
  double tot[1];
  if (!grid_finish<1>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->pq = tot[0];
  st->alpha = st->gamma / tot[0];
  if (!isfinite(tot[0])) {
    st->status = FEMK_NONFINITE;
    st->done = 1;
  } else if (!(tot[0] > 0.0)) {
    st->status = FEMK_BREAKDOWN;
    st->done = 1;
  }
}

// r = b - y (y = A x), z = D^-1 r, p = z and the init dots (matrix-free init)
__global__ void __launch_bounds__(kThreads) k_init_from_ax(int64_t n, const double* __restrict__ b,
                                                          const double* __restrict__ ax, const double* __restrict__ dinv,
                                                          double* __restrict__ r, double* __restrict__ z,
                                                          double* __restrict__ p, double* __restrict__ partials,
                                                          CgState* st, double tol2, double atol2) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double bi = b[i];
    const double ri = bi - ax[i];
    const double zi = dinv ? dinv[i] * ri : ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    acc[0] += ri * zi;
    acc[1] += ri * ri;
    acc[2] += bi * bi;
  }
  block_reduce_store<3>(acc, partials);
  double tot[3];
  if (!grid_finish<3>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->gamma = tot[0];
  st->rr = tot[1];
  st->bb = tot[2];
  st->atol2 = fmax(tol2 * tot[2], atol2);
  st->iter = 0;
  st->status = isfinite(tot[0]) && isfinite(tot[1]) ? FEMK_OK : FEMK_NONFINITE;
  const double rs = st->precond ? tot[1] : tot[0];
  st->done = (!(rs > st->atol2) || st->maxiter <= 0 || st->status != FEMK_OK) ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads) k_resid_from_ax(int64_t n, const double* __restrict__ b,
                                                           const double* __restrict__ ax, double* __restrict__ partials,
                                                           CgState* st) {
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double bi = b[i];
    const double w = bi - ax[i];
    acc[0] += w * w;
    acc[1] += bi * bi;
  }
  block_reduce_store<2>(acc, partials);
  double tot[2];
  if (!grid_finish<2>(partials, &st->ticket, tot)) return;
  if (threadIdx.x != 0) return;
  st->pq = tot[0];
  st->bb = tot[1];
}

__global__ void k_jacobi(const int32_t* __restrict__ diag, const double* __restrict__ vals, int64_t n, int64_t nnz,
                         double* __restrict__ inv, int* __restrict__ err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = diag[i];
    const double d = FEMK_IN_BOUNDS(k, nnz, err) ? vals[k] : 0.0;
    inv[i] = 1.0 / (fabs(d) > 1e-30 ? d : 1.0);
  }
}

__global__ void k_invert_diag(double* __restrict__ d, int64_t n, const uint8_t* __restrict__ dmask) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = dmask[i] ? 1.0 : d[i];
    d[i] = 1.0 / (fabs(v) > 1e-30 ? v : 1.0);
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
int spmv_grid(const femk_plan* p) { return p->n_sm * (2048 / kThreads); }

inline bool aligned16(const void* a) { return ((uintptr_t)a & 15u) == 0; }

void launch_pupdate(const femk_plan* p, double* pv, const double* z, const CgState* st, cudaStream_t s) {
  if (p->l2_mode != 0)
    k_pupdate<true><<<::femk::counted_launch() + wave_grid(k_pupdate<true>, kThreads, p), kThreads, 0, s>>>(p->n, pv,
                                                                                                         z, st);
  else
    k_pupdate<false><<<::femk::counted_launch() + wave_grid(k_pupdate<false>, kThreads, p), kThreads, 0, s>>>(
        p->n, pv, z, st);
}

// k_update with two-row loads when every vector it touches is 16-byte aligned
void launch_update(const femk_plan* p, double* x, double* r, double* z, const double* pv, const double* q,
                   const double* dinv, double* partials, CgState* st, cudaStream_t s) {
  const bool vec = aligned16(x) && aligned16(r) && aligned16(z) && aligned16(pv) && aligned16(q) &&
                   (dinv == nullptr || aligned16(dinv));
  const int hm = p->l2_mode;
  if (vec && (hm == 1 || hm == 2 || hm == 3 || hm == 4))
    k_update<true, true><<<::femk::counted_launch() + wave_grid(k_update<true, true>, kThreads, p), kThreads, 0, s>>>(
        p->n, x, r, z, pv, q, dinv, partials, st);
  else if (vec)
    k_update<true><<<::femk::counted_launch() + wave_grid(k_update<true>, kThreads, p), kThreads, 0, s>>>(
        p->n, x, r, z, pv, q, dinv, partials, st);
  else
    k_update<false><<<::femk::counted_launch() + wave_grid(k_update<false>, kThreads, p), kThreads, 0, s>>>(
        p->n, x, r, z, pv, q, dinv, partials, st);
}

// the split vector kernels (k_update_r, k_pupdate_x); false when a caller vector is not 16-byte aligned
bool split_ok(const femk_plan* p, const double* x, const double* dinv) {
  return p->cg_split && aligned16(x) && (dinv == nullptr || aligned16(dinv));
}

void launch_update_r(const femk_plan* p, double* r, const double* q, const double* dinv, CgState* st,
                     cudaStream_t s) {
  auto kern = p->l2_mode != 0 ? k_update_r<true> : k_update_r<false>;
  kern<<<::femk::counted_launch() + vec_grid(kern, kThreads, p), kThreads, 0, s>>>(p->n, r, q, dinv, p->partials, st);
}

void launch_pupdate_x(const femk_plan* p, double* x, double* pv, const double* r, const double* dinv,
                      const CgState* st, cudaStream_t s) {
  auto kern = p->l2_mode != 0 ? k_pupdate_x<true> : k_pupdate_x<false>;
  kern<<<::femk::counted_launch() + vec_grid(kern, kThreads, p), kThreads, 0, s>>>(p->n, x, pv, r, dinv, st);
}

template <int MODE>
int launch_csr_p(const femk_plan* p, const double* vals, const double* x, double* y, const double* b,
                 const double* dinv, double* z, double* pout, double* partials, CgState* st, double tol2, double atol2,
                 cudaStream_t s) {
  const bool ok = with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    const int grid = wave_grid(k_csr<L, U, MODE>, kThreads, p);
    k_csr<L, U, MODE><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, x, y, b,
                                                                           dinv, z, pout, partials, st, tol2, atol2,
                                                                           st ? &st->status : p->dev_err);
  });
  if (!ok) {
    set_error("unsupported SpMV configuration");
    return FEMK_EINVAL;
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

template <int MODE>
int launch_csr(const femk_plan* p, const double* vals, const double* x, double* y, const double* b, const double* dinv,
               double* z, double* pout, CgState* st, double tol2, double atol2, cudaStream_t s) {
  return launch_csr_p<MODE>(p, vals, x, y, b, dinv, z, pout, p->partials, st, tol2, atol2, s);
}

// Bulk-copy CG-step SpMV (k_sell_bulk) in the plan's configuration: p->bulk_stages slices in flight
// per warp, p->bulk_warps warps per block. Returns false (nothing launched) when the plan does not
// use it: switched off, rows wider than 32 entries, or no 16-bit column offsets.
template <int S, int WPB, int WMAX>
bool launch_sell_bulk_cfg(const femk_plan* p, const double* x, double* y, CgState* st, cudaStream_t s,
                          bool prime) {
  auto kern = k_sell_bulk<kCgStep, int16_t, WMAX, S, WPB>;
  constexpr int kSmem = WPB * BulkRing<double, int16_t, WMAX, S>::kWarpBytes;
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
      (const int64_t*)p->sell_ptr, (const int16_t*)(tab ? p->sell_cu : p->sell_c16), (const double*)p->sell_vals,
      p->n, p->n_slices, x, y, p->partials, st, (int*)nullptr, (const int64_t*)(tab ? p->sell_cuptr : nullptr));
  return true;
}

// prime = true only sets the kernel attribute and reads the occupancy (before a graph capture)
bool launch_sell_bulk(const femk_plan* p, const double* x, double* y, CgState* st, cudaStream_t s,
                      bool prime = false) {
  if (!p->bulk_cfg || !p->sell_c16 || !p->sell64_c16 || p->max_row > 32) return false;
  if (!aligned16(p->sell_vals) || !aligned16(p->sell_c16)) return false;  // bulk copies start on 16 B
  if (p->sell_cu && !aligned16(p->sell_cu)) return false;
  // ring stages sized for the widest row: 8 (2-D P1 triangles), 16 (P1 tetrahedra), 32
  const int wsel = p->max_row <= 8 ? 8 : (p->max_row <= 16 ? 16 : 32);
#define FEMK_BULK_CFG(code, S, WPB)                                                         \
  case code:                                                                                \
    return wsel == 8    ? launch_sell_bulk_cfg<S, WPB, 8>(p, x, y, st, s, prime)  \
           : wsel == 16 ? launch_sell_bulk_cfg<S, WPB, 16>(p, x, y, st, s, prime) \
                        : launch_sell_bulk_cfg<S, WPB, 32>(p, x, y, st, s, prime);
  switch (p->bulk_cfg) {
    FEMK_BULK_CFG(11, 1, 1)
    FEMK_BULK_CFG(12, 1, 2)
    FEMK_BULK_CFG(14, 1, 4)
    FEMK_BULK_CFG(18, 1, 8)
    FEMK_BULK_CFG(22, 2, 2)
    FEMK_BULK_CFG(24, 2, 4)
    FEMK_BULK_CFG(28, 2, 8)
    FEMK_BULK_CFG(34, 3, 4)
    FEMK_BULK_CFG(38, 3, 8)
    default:
      return false;
  }
#undef FEMK_BULK_CFG
}

// The operator of a solve: the sliced-ELL copy (values gathered by prepare_sell) or the CSR.
template <int MODE>
int launch_op(const femk_plan* p, bool sell, const double* vals, const double* x, double* y, const double* b,
              const double* dinv, double* z, double* pout, CgState* st, double tol2, double atol2, cudaStream_t s) {
  if (!sell) return launch_csr<MODE>(p, vals, x, y, b, dinv, z, pout, st, tol2, atol2, s);
  if (MODE == kCgStep && launch_sell_bulk(p, x, y, st, s)) {
    FEMK_CUDA_TRY(cudaGetLastError());
    return FEMK_OK;
  }
  // column offsets in 16 bits when the plan's bandwidth allows it (same values, 2 B less per entry)
  int* err = st ? &st->status : p->dev_err;
  auto go = [&](auto Bc, auto cols) {
    constexpr int B = decltype(Bc)::value;
    using I = std::remove_const_t<std::remove_pointer_t<decltype(cols)>>;
    const int hm = p->l2_mode;
    if (hm == 1) {
      const int grid = wave_grid(k_sell<MODE, I, B, 1>, kThreads, p);
      k_sell<MODE, I, B, 1><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->sell_ptr, cols, p->sell_vals, p->n, p->n_slices, x, y, b, dinv, z, pout, p->partials, st, tol2, atol2,
          err);
    } else if (hm == 2) {
      const int grid = wave_grid(k_sell<MODE, I, B, 2>, kThreads, p);
      k_sell<MODE, I, B, 2><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->sell_ptr, cols, p->sell_vals, p->n, p->n_slices, x, y, b, dinv, z, pout, p->partials, st, tol2, atol2,
          err);
    } else if (hm == 4) {
      const int grid = wave_grid(k_sell<MODE, I, B, 4>, kThreads, p);
      k_sell<MODE, I, B, 4><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->sell_ptr, cols, p->sell_vals, p->n, p->n_slices, x, y, b, dinv, z, pout, p->partials, st, tol2, atol2,
          err);
    } else {
      const int grid = wave_grid(k_sell<MODE, I, B>, kThreads, p);
      k_sell<MODE, I, B><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->sell_ptr, cols, p->sell_vals, p->n, p->n_slices, x, y, b, dinv, z, pout, p->partials, st, tol2, atol2,
          err);
    }
  };
  const bool c16 = p->sell_c16 && p->sell64_c16;
  if (p->sell_batch == 8) {
    if (c16)
      go(std::integral_constant<int, 8>{}, (const int16_t*)p->sell_c16);
    else
      go(std::integral_constant<int, 8>{}, (const int32_t*)p->sell_cols);
  } else {
    // int32 columns (3-D P2: rows of up to 65 entries) keep 32 entries in flight: 48 registers in
    // place of 32, and the P2 64^3 FP64 solve took 100.6 ms against 116.4 ms with 16
    if (c16)
      go(std::integral_constant<int, 16>{}, (const int16_t*)p->sell_c16);
    else
      go(std::integral_constant<int, 32>{}, (const int32_t*)p->sell_cols);
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

int prepare_sell(femk_plan* p, const double* vals, cudaStream_t s) {
  if (!p->sell_vals) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals, sizeof(double) * (p->sell_nnz + 1)));
  const int32_t cap = 32 * (p->max_row > 0 ? p->max_row : 1);
  const size_t smem = sizeof(double) * 4 * (size_t)cap;
  FEMK_CUDA_TRY(cudaFuncSetAttribute(k_sell_gather<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_sell_gather<double><<<::femk::counted_launch() + blocks_for(p->n_slices, 4, p->n_sm * 16), 128, smem, s>>>(
      p->sell_ptr, p->indptr, p->n, p->n_slices, vals, p->nnz, cap, p->sell_vals, p->dev_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

struct MatFree {
  const double* param;
  int mode;
  double scale;
};

__global__ void k_zero(double* __restrict__ y, int64_t n, const CgState* st) {
  if (st && st->done) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = 0.0;
}

// y = A x for the matrix-free operator; with st != NULL every launch is a no-op once st->done.
// the masked connectivity, built on first use (the Dirichlet set of a plan is fixed), and on a P1
// tetrahedral plan the Kuhn-block check (once, with a synchronous read of its flag)
int ensure_mcells(const femk_plan* pc, cudaStream_t s) {
  femk_plan* p = const_cast<femk_plan*>(pc);
  if (!p->mcells) {
    const int64_t len = p->ntet * p->nd;
    FEMK_CUDA_TRY(cudaMalloc(&p->mcells, sizeof(int32_t) * (len > 0 ? len : 1)));
    k_mask_cells<<<::femk::counted_launch() + blocks_for(len, 256, p->n_sm * 16), 256, 0, s>>>(p->cells, len, p->dmask,
                                                                                               p->mcells);
    FEMK_CUDA_TRY(cudaGetLastError());
  }
  if (p->kuhn_state == 0) {
    p->kuhn_state = -1;
    if (p->nd == 4 && p->dim == 3 && p->ntet > 0 && p->ntet % 6 == 0) {
      const int64_t nhex = p->ntet / 6;
      int* flag = nullptr;
      FEMK_CUDA_TRY(cudaMalloc(&p->kuhn, sizeof(int32_t) * 8 * nhex));
      FEMK_CUDA_TRY(cudaMalloc(&flag, sizeof(int)));
      int bad = 1;
      cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), s);
      if (e == cudaSuccess) {
        k_kuhn_corners<<<::femk::counted_launch() + blocks_for(nhex, 256, p->n_sm * 16), 256, 0, s>>>(p->mcells, nhex,
                                                                                                   p->kuhn, flag);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      cudaFree(flag);
      FEMK_CUDA_TRY(e);
      if (bad) {
        cudaFree(p->kuhn);
        p->kuhn = nullptr;
      } else {
        p->kuhn_state = 1;
      }
    }
  }
  return FEMK_OK;
}

int launch_matfree(const femk_plan* p, const MatFree& m, const double* x, double* y, cudaStream_t s,
                   const CgState* st = nullptr) {
  FEMK_TRY(ensure_mcells(p, s));
  k_zero<<<::femk::counted_launch() + p->n_sm * 8, 256, 0, s>>>(y, p->n, st);
  const int grid = blocks_for(p->ntet, 128, p->n_sm * 16);
  if (p->kuhn)
    k_matfree_kuhn<<<::femk::counted_launch() + blocks_for(p->ntet / 6, 128, p->n_sm * 16), 128, 0, s>>>(
        p->xyz, p->kuhn, p->ntet / 6, m.param, m.mode, m.scale, x, y, st);
  else
    FEMK_BY_ND(p->nd, k_matfree<ND><<<::femk::counted_launch() + grid, 128, 0, s>>>(p->xyz, p->mcells, p->ntet, m.param, m.mode, m.scale, x, y, st));
  FEMK_CUDA_TRY(cudaGetLastError());
  if (p->n_dir > 0) {
    k_dirichlet_identity<<<::femk::counted_launch() + blocks_for(p->n_dir, 256, 65535), 256, 0, s>>>(p->dlist, p->n_dir, x, y, st);
    FEMK_CUDA_TRY(cudaGetLastError());
  }
  return FEMK_OK;
}

// One chunk of CG iterations on stream ws: the step SpMV and the two vector kernels per iteration.
// Opt-in per-kernel timing of the CG loop (femk_set_profiling): events around the three kernels
// of every iteration of a chunk; the chunked path runs without graph replay while it is on.
struct ProfData {
  cudaEvent_t ev[kChunk][4];
  double ms[3] = {0.0, 0.0, 0.0};  // step SpMV, update, p update
  int64_t iters = 0;
};

int enqueue_chunk(const femk_plan* p, const double* vals, double* x, const double* dinv, bool sell, int64_t iters,
                  cudaStream_t ws) {
  const int64_t vs = p->vstride;
  double* r = p->work;
  double* z = r + vs;
  double* P0 = z + vs;
  double* q = P0 + vs;
  CgState* st = p->state;
  ProfData* pd = (ProfData*)p->prof;
  const bool split = split_ok(p, x, dinv);
  for (int64_t it = 0; it < iters; ++it) {
    if (pd) cudaEventRecord(pd->ev[it][0], ws);
    FEMK_TRY(launch_op<kCgStep>(p, sell, vals, P0, q, nullptr, nullptr, nullptr, nullptr, st, 0.0, 0.0, ws));
    if (pd) cudaEventRecord(pd->ev[it][1], ws);
    if (split)
      launch_update_r(p, r, q, dinv, st, ws);
    else
      launch_update(p, x, r, z, P0, q, dinv, p->partials, st, ws);
    if (pd) cudaEventRecord(pd->ev[it][2], ws);
    if (split)
      launch_pupdate_x(p, x, P0, r, dinv, st, ws);
    else
      launch_pupdate(p, P0, z, st, ws);
    if (pd) cudaEventRecord(pd->ev[it][3], ws);
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

// Capture one chunk into a CUDA graph (re-captured when the operand pointers change).
int ensure_chunk_graph(femk_plan* p, const double* vals, double* x, const double* dinv, bool sell) {
  if (sell && !p->sell_vals) {
    set_error("femk_pcg: sliced-ELL values missing at graph capture");
    return FEMK_EINVAL;
  }
  const void* key[5] = {vals, x, dinv, (const void*)(intptr_t)(sell ? 4 : 2), p->sell_vals};
  bool same = p->cg_exec != nullptr;
  for (int i = 0; i < 5; ++i) same = same && key[i] == p->cg_key[i];
  if (same) return FEMK_OK;
  // occupancy queries happen before capture begins
  with_spmv_cfg(p->spmv_L, p->spmv_U, [&](auto Lc, auto Uc) {
    constexpr int L = decltype(Lc)::value, U = decltype(Uc)::value;
    (void)wave_grid(k_csr<L, U, kCgStep>, kThreads, p);
  });
  (void)wave_grid(k_sell<kCgStep, int32_t, 8>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 16>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 8>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 16>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 16, 1>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 16, 1>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 8, 1>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 8, 1>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 16, 2>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 16, 2>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 8, 2>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 8, 2>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 16, 4>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 16, 4>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int16_t, 8, 4>, kThreads, p);
  (void)wave_grid(k_sell<kCgStep, int32_t, 8, 4>, kThreads, p);
  (void)wave_grid(k_update<true, true>, kThreads, p);
  (void)wave_grid(k_pupdate<true>, kThreads, p);
  (void)wave_grid(k_update<true>, kThreads, p);
  (void)wave_grid(k_update<false>, kThreads, p);
  (void)wave_grid(k_pupdate<false>, kThreads, p);
  (void)wave_grid(k_update_r<true>, kThreads, p);
  (void)wave_grid(k_update_r<false>, kThreads, p);
  (void)wave_grid(k_pupdate_x<true>, kThreads, p);
  (void)wave_grid(k_pupdate_x<false>, kThreads, p);
  if (sell) (void)launch_sell_bulk(p, nullptr, nullptr, nullptr, nullptr, true);
  cudaGraph_t g = nullptr;
  set_capturing(true);
  cudaError_t e = cudaStreamBeginCapture(p->cg_stream, cudaStreamCaptureModeThreadLocal);
  int st = e == cudaSuccess ? enqueue_chunk(p, vals, x, dinv, sell, kChunk, p->cg_stream) : FEMK_ECUDA;
  const cudaError_t e2 = cudaStreamEndCapture(p->cg_stream, &g);
  set_capturing(false);
  if (e != cudaSuccess || e2 != cudaSuccess || st != FEMK_OK) {
    if (g) cudaGraphDestroy(g);
    set_error(std::string("femk_pcg: graph capture failed: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    return st != FEMK_OK ? st : FEMK_ECUDA;
  }
  bool updated = false;
  if (p->cg_exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(p->cg_exec, g, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(p->cg_exec);
      p->cg_exec = nullptr;
    }
  }
  if (!updated) {
    const cudaError_t e3 = cudaGraphInstantiate(&p->cg_exec, g, 0);
    if (e3 != cudaSuccess) {
      cudaGraphDestroy(g);
      p->cg_exec = nullptr;
      set_error(std::string("femk_pcg: graph instantiation failed: ") + cudaGetErrorString(e3));
      return FEMK_ECUDA;
    }
  }
  cudaGraphDestroy(g);
  for (int i = 0; i < 5; ++i) p->cg_key[i] = key[i];
  p->cg_nodes = 3 * kChunk;
  return FEMK_OK;
}

int ensure_cg_stream(femk_plan* p) {
  if (p->cg_stream) return FEMK_OK;
  FEMK_CUDA_TRY(cudaStreamCreateWithFlags(&p->cg_stream, cudaStreamNonBlocking));
  for (int i = 0; i < 3; ++i) FEMK_CUDA_TRY(cudaEventCreateWithFlags(&p->cg_ev[i], cudaEventDisableTiming));
  return FEMK_OK;
}

int pcg_run(const femk_plan* pc, const double* vals, const MatFree* mf, const double* b, double* x, const double* dinv,
            double tol, double atol, int32_t maxiter, int32_t* iters_out, double* relres_out, cudaStream_t s) {
  femk_plan* p = const_cast<femk_plan*>(pc);
  FEMK_TRY(ensure_workspace(p));
  FEMK_TRY(ensure_cg_stream(p));
  const int64_t n = p->n;
  const int64_t vs = p->vstride;
  double* r = p->work;
  double* z = r + vs;
  double* pv = z + vs;
  double* q = pv + vs;
  CgState* st = p->state;
  ProfData* pd = !mf ? (ProfData*)p->prof : nullptr;
  const bool graph = !mf && p->cg_graph && !pd;
  const bool sell = !mf && p->use_sell && p->sell_cols;
  // all solver work runs on the plan's stream, ordered after the caller's stream and before
  // whatever the caller enqueues next
  cudaStream_t ws = p->cg_stream;
  FEMK_CUDA_TRY(cudaEventRecord(p->cg_ev[2], s));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(ws, p->cg_ev[2], 0));
  // the sliced-ELL values buffer must exist before a graph that reads it is captured
  if (sell) FEMK_TRY(prepare_sell(p, vals, ws));
  if (graph) FEMK_TRY(ensure_chunk_graph(p, vals, x, dinv, sell));
  CgState init{};
  init.maxiter = maxiter;
  init.precond = dinv ? 1 : 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(CgState), cudaMemcpyHostToDevice, ws));
  const double tol2 = tol * tol, atol2 = atol * atol;
  if (mf) {
    FEMK_TRY(launch_matfree(p, *mf, x, q, ws));
    k_init_from_ax<<<::femk::counted_launch() + wave_grid(k_init_from_ax, kThreads, p), kThreads, 0, ws>>>(
        n, b, q, dinv, r, z, pv, p->partials, st, tol2, atol2);
  } else {
    FEMK_TRY(launch_op<kInit>(p, sell, vals, x, r, b, dinv, z, pv, st, tol2, atol2, ws));
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  CgState* hs = p->state_host;
  int status = FEMK_OK;
  int64_t enq = 0;  // iterations enqueued
  int chunk_id = 0;
  bool have_prev = false;
  while (true) {
    if (graph) {
      FEMK_CUDA_TRY(cudaGraphLaunch(p->cg_exec, ws));
      count_launches(p->cg_nodes);
      enq += kChunk;  // iterations past convergence or maxiter return at entry
    } else if (mf) {
      const int64_t todo = std::min<int64_t>(kChunk, (int64_t)maxiter - enq);
      for (int64_t it = 0; it < todo; ++it) {
        FEMK_TRY(launch_matfree(p, *mf, pv, q, ws, st));
        k_dot_pq<<<::femk::counted_launch() + wave_grid(k_dot_pq, kThreads, p), kThreads, 0, ws>>>(n, pv, q,
                                                                                                  p->partials, st);
        launch_update(p, x, r, z, pv, q, dinv, p->partials, st, ws);
        launch_pupdate(p, pv, z, st, ws);
      }
      FEMK_CUDA_TRY(cudaGetLastError());
      enq += todo;
    } else {
      const int64_t todo = std::min<int64_t>(kChunk, (int64_t)maxiter - enq);
      FEMK_TRY(enqueue_chunk(p, vals, x, dinv, sell, todo, ws));
      if (pd) {  // time the iterations of this chunk that ran (later ones return at entry)
        CgState now{};
        FEMK_CUDA_TRY(cudaMemcpyAsync(&now, st, sizeof(CgState), cudaMemcpyDeviceToHost, ws));
        FEMK_CUDA_TRY(cudaStreamSynchronize(ws));
        const int64_t real = std::min<int64_t>(todo, std::max<int64_t>(0, (int64_t)now.iter - enq));
        for (int64_t it = 0; it < real; ++it)
          for (int k = 0; k < 3; ++k) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, pd->ev[it][k], pd->ev[it][k + 1]) == cudaSuccess) pd->ms[k] += t;
          }
        pd->iters += real;
      }
      enq += todo;
    }
    CgState* slot_h = hs + (chunk_id & 1);
    FEMK_CUDA_TRY(cudaMemcpyAsync(slot_h, st, sizeof(CgState), cudaMemcpyDeviceToHost, ws));
    FEMK_CUDA_TRY(cudaEventRecord(p->cg_ev[chunk_id & 1], ws));
    // look at the previous chunk's flag while this one runs
    if (have_prev) {
      FEMK_CUDA_TRY(cudaEventSynchronize(p->cg_ev[(chunk_id - 1) & 1]));
      if (hs[(chunk_id - 1) & 1].done) break;
    }
    have_prev = true;
    if (enq >= maxiter) break;
    ++chunk_id;
  }
  FEMK_CUDA_TRY(cudaStreamSynchronize(ws));
  CgState fin{};
  FEMK_CUDA_TRY(cudaMemcpy(&fin, st, sizeof(CgState), cudaMemcpyDeviceToHost));
  if (iters_out) *iters_out = fin.iter;
  if (fin.status != FEMK_OK) status = fin.status;
  if (relres_out) {
    if (mf) {
      FEMK_TRY(launch_matfree(p, *mf, x, q, ws));
      k_resid_from_ax<<<::femk::counted_launch() + wave_grid(k_resid_from_ax, kThreads, p), kThreads, 0, ws>>>(
          n, b, q, p->partials, st);
    } else {
      FEMK_TRY(launch_op<kResid>(p, sell, vals, x, nullptr, b, nullptr, nullptr, nullptr, st, 0.0, 0.0, ws));
    }
    FEMK_CUDA_TRY(cudaMemcpyAsync(hs, st, sizeof(CgState), cudaMemcpyDeviceToHost, ws));
    FEMK_CUDA_TRY(cudaStreamSynchronize(ws));
    *relres_out = std::sqrt(hs->pq) / (std::sqrt(hs->bb) + 1e-30);
  }
  // the caller's stream continues after the solve
  FEMK_CUDA_TRY(cudaEventRecord(p->cg_ev[2], ws));
  FEMK_CUDA_TRY(cudaStreamWaitEvent(s, p->cg_ev[2], 0));
  if (status == FEMK_OK) {
    const double rs = fin.precond ? fin.rr : fin.gamma;
    if (rs > fin.atol2) {
      set_error("femk_pcg: iteration cap reached above tolerance");
      status = FEMK_NOT_CONVERGED;
    }
  } else if (status == FEMK_BREAKDOWN) {
    set_error("femk_pcg: <p, A p> <= 0 (operator not symmetric positive definite)");
  } else if (status == FEMK_NONFINITE) {
    set_error("femk_pcg: non-finite value in a CG reduction");
  } else if (status == FEMK_TIMEOUT) {
    set_error("femk_pcg: a bulk-copy wait of the CG-step SpMV gave up");
  } else if (status == FEMK_EBOUNDS) {
    set_error("femk_pcg: an index check inside a kernel failed (bounds-checked build)");
  }
  if (status == FEMK_OK || status == FEMK_NOT_CONVERGED) {
    const int bc = check_bounds(p, s, "femk_pcg");  // the value gather and plain products of the solve
    if (bc != FEMK_OK) return bc;
  }
  return status;
}

}  // namespace

int ensure_workspace(femk_plan* p) {
  if (p->work) return FEMK_OK;
  FEMK_CUDA_TRY(cudaMalloc(&p->work, sizeof(double) * 5 * p->vstride));
  FEMK_CUDA_TRY(cudaMalloc(&p->partials, sizeof(double) * 4 * (int64_t)p->n_sm * 64));
  FEMK_CUDA_TRY(cudaMalloc(&p->state, sizeof(CgState)));
  FEMK_CUDA_TRY(cudaMemset(p->state, 0, sizeof(CgState)));
  FEMK_CUDA_TRY(cudaMallocHost(&p->state_host, 2 * sizeof(CgState)));
  FEMK_CUDA_TRY(cudaMalloc(&p->bar, 64));
  return FEMK_OK;
}

int spmv_csr(const femk_plan* p, const double* vals, const double* x, double* y, cudaStream_t s) {
  return launch_csr<kPlain>(p, vals, x, y, nullptr, nullptr, nullptr, nullptr, nullptr, 0.0, 0.0, s);
}

int ensure_sell_values(femk_plan* p, bool fp32) {
  if (!p->sell_vals) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals, sizeof(double) * (p->sell_nnz + 1)));
  if (fp32 && !p->sell_vals32) FEMK_CUDA_TRY(cudaMalloc(&p->sell_vals32, sizeof(float) * (p->sell_nnz + 1)));
  const int32_t cap = 32 * (p->max_row > 0 ? p->max_row : 1);
  const int smem = (int)(sizeof(double) * 4 * (size_t)cap);
  FEMK_CUDA_TRY(cudaFuncSetAttribute(k_sell_gather<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  FEMK_CUDA_TRY(cudaFuncSetAttribute(k_sell_gather<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  return FEMK_OK;
}

int launch_sell_values(const femk_plan* p, const double* vals, bool fp32, cudaStream_t s) {
  const int32_t cap = 32 * (p->max_row > 0 ? p->max_row : 1);
  const size_t smem = sizeof(double) * 4 * (size_t)cap;
  const int grid = blocks_for(p->n_slices, 4, p->n_sm * 16);
  k_sell_gather<double><<<::femk::counted_launch() + grid, 128, smem, s>>>(p->sell_ptr, p->indptr, p->n, p->n_slices,
                                                                           vals, p->nnz, cap, p->sell_vals, p->dev_err);
  if (fp32)
    k_sell_gather<float><<<::femk::counted_launch() + grid, 128, smem, s>>>(p->sell_ptr, p->indptr, p->n, p->n_slices,
                                                                            vals, p->nnz, cap, p->sell_vals32, p->dev_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

}  // namespace femk

using namespace femk;

extern "C" int femk_jacobi(const femk_plan* p, const double* vals, double* inv, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals && inv, "femk_jacobi: NULL argument");
  k_jacobi<<<::femk::counted_launch() + blocks_for(p->n, 256, p->n_sm * 8), 256, 0, (cudaStream_t)stream>>>(
      p->diag, vals, p->n, p->nnz, inv, p->dev_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  return check_bounds(p, (cudaStream_t)stream, "femk_jacobi");
}

extern "C" int femk_spmv(const femk_plan* p, const double* vals, const double* x, double* y, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals && x && y, "femk_spmv: NULL argument");
  FEMK_TRY(spmv_csr(p, vals, x, y, (cudaStream_t)stream));
  return check_bounds(p, (cudaStream_t)stream, "femk_spmv");
}

extern "C" int femk_set_profiling(femk_plan* p, int on) {
  clear_error();
  FEMK_CHECK_ARG(p, "femk_set_profiling: NULL plan");
  ProfData* pd = (ProfData*)p->prof;
  if (pd) {
    for (auto& row : pd->ev)
      for (cudaEvent_t e : row)
        if (e) cudaEventDestroy(e);
    delete pd;
    p->prof = nullptr;
  }
  if (on) {
    pd = new ProfData();
    for (auto& row : pd->ev)
      for (cudaEvent_t& e : row) FEMK_CUDA_TRY(cudaEventCreate(&e));
    p->prof = pd;
  }
  return FEMK_OK;
}

extern "C" int femk_get_profile(const femk_plan* p, double* step_ms, double* update_ms, double* pupdate_ms,
                                int64_t* iterations) {
  clear_error();
  FEMK_CHECK_ARG(p, "femk_get_profile: NULL plan");
  const ProfData* pd = (const ProfData*)p->prof;
  if (step_ms) *step_ms = pd ? pd->ms[0] : 0.0;
  if (update_ms) *update_ms = pd ? pd->ms[1] : 0.0;
  if (pupdate_ms) *pupdate_ms = pd ? pd->ms[2] : 0.0;
  if (iterations) *iterations = pd ? pd->iters : 0;
  return FEMK_OK;
}

extern "C" int femk_prepare_operator(const femk_plan* p, const double* vals, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals, "femk_prepare_operator: NULL argument");
  FEMK_CHECK_ARG(p->sell_cols, "femk_prepare_operator: the plan has no sliced-ELL layout");
  FEMK_TRY(prepare_sell(const_cast<femk_plan*>(p), vals, (cudaStream_t)stream));
  return check_bounds(p, (cudaStream_t)stream, "femk_prepare_operator");
}

extern "C" int femk_spmv_prepared(const femk_plan* p, const double* x, double* y, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && x && y, "femk_spmv_prepared: NULL argument");
  FEMK_CHECK_ARG(p->sell_vals, "femk_spmv_prepared: call femk_prepare_operator first");
  FEMK_TRY(launch_op<kPlain>(p, true, nullptr, x, y, nullptr, nullptr, nullptr, nullptr, nullptr, 0.0, 0.0,
                             (cudaStream_t)stream));
  return check_bounds(p, (cudaStream_t)stream, "femk_spmv_prepared");
}

extern "C" int femk_spmv_matfree(const femk_plan* p, const double* param, int mode, double scale, const double* x,
                                 double* y, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && x && y, "femk_spmv_matfree: NULL argument");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param), "femk_spmv_matfree: bad coefficient");
  FEMK_TRY(resolve_coef(p, param, mode, (cudaStream_t)stream, &param, &mode));
  MatFree m{param, mode, scale};
  return launch_matfree(p, m, x, y, (cudaStream_t)stream);
}

extern "C" int femk_jacobi_matfree(const femk_plan* p, const double* param, int mode, double scale, double* inv,
                                   void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && inv, "femk_jacobi_matfree: NULL argument");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param), "femk_jacobi_matfree: bad coefficient");
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(resolve_coef(p, param, mode, s, &param, &mode));
  FEMK_CUDA_TRY(cudaMemsetAsync(inv, 0, sizeof(double) * p->n, s));
  const int grid = blocks_for(p->ntet, 128, p->n_sm * 16);
  FEMK_BY_ND(p->nd, k_matfree_diag<ND><<<::femk::counted_launch() + grid, 128, 0, s>>>(p->xyz, p->cells, p->ntet, p->dmask, param, mode, scale, inv));
  k_invert_diag<<<::femk::counted_launch() + blocks_for(p->n, 256, p->n_sm * 8), 256, 0, s>>>(inv, p->n, p->dmask);
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

extern "C" int femk_pcg(const femk_plan* p, const double* vals, const double* b, double* x, const double* dinv,
                        double tol, double atol, int32_t maxiter, int32_t* iters_out, double* relres_out,
                        void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals && b && x, "femk_pcg: NULL argument");
  FEMK_CHECK_ARG(tol >= 0.0 && atol >= 0.0, "femk_pcg: negative tolerance");
  return pcg_run(p, vals, nullptr, b, x, dinv, tol, atol, maxiter, iters_out, relres_out, (cudaStream_t)stream);
}

extern "C" int femk_pcg_matfree(const femk_plan* p, const double* param, int mode, double scale, const double* b,
                                double* x, const double* dinv, double tol, double atol, int32_t maxiter,
                                int32_t* iters_out, double* relres_out, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && b && x, "femk_pcg_matfree: NULL argument");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param), "femk_pcg_matfree: bad coefficient");
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(resolve_coef_exp(p, param, mode, s, &param, &mode));  // every CG step applies the operator
  MatFree m{param, mode, scale};
  return pcg_run(p, nullptr, &m, b, x, dinv, tol, atol, maxiter, iters_out, relres_out, s);
}

// ---------------------------------------------------------------------------------------------
// Allocation-free PCG. Same kernels and the same iteration as femk_pcg, but the solver vectors,
// the reduction partials and the solver state live in one file-scope device array instead of
// plan-owned cudaMalloc'd workspace, and the host loop uses no events and no pinned memory.
// For callers that must not allocate device memory while they run: code inside an XLA FFI
// handler (device memory belongs to XLA's allocator), frameworks whose caching allocator already
// holds nearly all of HBM, and real-time loops with a fixed memory budget.
// ---------------------------------------------------------------------------------------------
namespace femk {
namespace {

constexpr int64_t kNoAllocMaxN = FEMK_NOALLOC_MAX_N;
constexpr int64_t kNoAllocPartials = 3 * 4096;  // NV <= 3 values per block, up to 4096 blocks
constexpr int64_t kNoAllocStateDoubles = (sizeof(CgState) + sizeof(double) - 1) / sizeof(double);
constexpr int64_t kNoAllocDoubles = 4 * kNoAllocMaxN + kNoAllocPartials + kNoAllocStateDoubles;

// 4 vectors of kNoAllocMaxN doubles (r, z, p, q) + reduction partials + CgState: about 8.5 MB,
// held by every device that loads the library until the process exits. Shared by every call.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Device address of g_noalloc_scratch per device, looked up once with that device current.
constexpr int kMaxDevices = 64;
static double* g_noalloc_addr[kMaxDevices] = {};
static std::mutex g_noalloc_mu;

int noalloc_scratch(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("femk_pcg_noalloc: device index out of range");
    return FEMK_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || addr == nullptr) {
      set_error(std::string("femk_pcg_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return FEMK_ECUDA;
    }
    g_noalloc_addr[device] = (double*)addr;
  }
  *out = g_noalloc_addr[device];
  return FEMK_OK;
}

template <int MODE>
int launch_csr_into(const femk_plan* p, const double* vals, const double* x, double* y, const double* b,
                    const double* dinv, double* z, double* pout, double* partials, CgState* st, double tol2,
                    double atol2, cudaStream_t s) {
  return launch_csr_p<MODE>(p, vals, x, y, b, dinv, z, pout, partials, st, tol2, atol2, s);
}

}  // namespace
}  // namespace femk

extern "C" int femk_pcg_noalloc(const femk_plan* p, const double* vals, const double* b, double* x,
                                const double* dinv, double tol, double atol, int32_t maxiter, int32_t* iters_out,
                                double* relres_out, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals && b && x, "femk_pcg_noalloc: NULL argument");
  FEMK_CHECK_ARG(tol >= 0.0 && atol >= 0.0, "femk_pcg_noalloc: negative tolerance");
  if (p->n > kNoAllocMaxN) {
    set_error("femk_pcg_noalloc: the system has " + std::to_string(p->n) + " DOFs; this entry point holds at most " +
              std::to_string(kNoAllocMaxN) + " (FEMK_NOALLOC_MAX_N). Use femk_pcg for larger systems.");
    return FEMK_EINVAL;
  }
  FEMK_CHECK_ARG((int64_t)spmv_grid(p) * 3 <= kNoAllocPartials && (int64_t)p->n_sm * 8 * 3 <= kNoAllocPartials,
                 "femk_pcg_noalloc: too many SMs for the static reduction scratch");
  int cur = -1;
  FEMK_CUDA_TRY(cudaGetDevice(&cur));
  FEMK_CHECK_ARG(cur == p->device, "femk_pcg_noalloc: make the plan's device current before the call");
  double* scratch = nullptr;
  FEMK_TRY(noalloc_scratch(cur, &scratch));
  cudaStream_t s = (cudaStream_t)stream;
  double* r = scratch;
  double* z = r + kNoAllocMaxN;
  double* pv = z + kNoAllocMaxN;
  double* q = pv + kNoAllocMaxN;
  double* partials = q + kNoAllocMaxN;
  CgState* st = (CgState*)(partials + kNoAllocPartials);
  // the state of the previous call is overwritten before any kernel reads it (ticket = 0 included)
  CgState init{};
  init.maxiter = maxiter;
  init.precond = dinv ? 1 : 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  const double tol2 = tol * tol, atol2 = atol * atol;
  FEMK_TRY(launch_csr_into<kInit>(p, vals, x, r, b, dinv, z, pv, partials, st, tol2, atol2, s));
  CgState h{};
  int64_t enq = 0;
  while (enq < maxiter) {
    const int64_t todo = std::min<int64_t>(kChunk, (int64_t)maxiter - enq);
    for (int64_t it = 0; it < todo; ++it) {
      FEMK_TRY(launch_csr_into<kCgStep>(p, vals, pv, q, nullptr, nullptr, nullptr, nullptr, partials, st, 0.0, 0.0, s));
      launch_update(p, x, r, z, pv, q, dinv, partials, st, s);
      launch_pupdate(p, pv, z, st, s);
    }
    FEMK_CUDA_TRY(cudaGetLastError());
    enq += todo;
    FEMK_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    FEMK_CUDA_TRY(cudaStreamSynchronize(s));
    if (h.done) break;
  }
  FEMK_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters_out) *iters_out = h.iter;
  const CgState fin = h;
  if (relres_out) {
    FEMK_TRY(launch_csr_into<kResid>(p, vals, x, nullptr, b, nullptr, nullptr, nullptr, partials, st, 0.0, 0.0, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    FEMK_CUDA_TRY(cudaStreamSynchronize(s));
    *relres_out = std::sqrt(h.pq) / (std::sqrt(h.bb) + 1e-30);
  }
  if (fin.status == FEMK_BREAKDOWN) {
    set_error("femk_pcg_noalloc: <p, A p> <= 0 (operator not symmetric positive definite)");
    return FEMK_BREAKDOWN;
  }
  if (fin.status == FEMK_NONFINITE) {
    set_error("femk_pcg_noalloc: non-finite value in a CG reduction");
    return FEMK_NONFINITE;
  }
  const double rs = fin.precond ? fin.rr : fin.gamma;
  if (rs > fin.atol2) {
    set_error("femk_pcg_noalloc: iteration cap reached above tolerance");
    return FEMK_NOT_CONVERGED;
  }
  return FEMK_OK;
}
