// Batched Jacobi-PCG: many independent problems of uneven size solved in one persistent
// cooperative launch (captured in a CUDA graph and replayed for repeated solves).
//
// The problems live in one plan built on their disjoint union (vertex ids offset per problem), so
// the plan build and one femk_assemble call serve all of them; problem k owns the contiguous rows
// [row_off[k], row_off[k+1]). Rows are cut into tiles that never cross a problem; a tile is one
// warp's work item, and every grid phase walks the tiles of the still-active problems (tile t on
// warp t mod W, W = warps in the grid, no block-wide synchronisation inside a phase). The products
// run on the plan's sliced-ELL copy (lane per row; copied from the CSR values in the same graph),
// with the vectors gathered through L1 (the barriers' acquire makes other blocks' writes visible):
//   phase 0 (once): r = b - A x0, z = D^-1 r, per-tile <r,z>, <r,r>, <b,b> | owner pass: beta_k = 0
//   phase 1: w = A z, p = z + beta_k p, q = w + beta_k q, per-tile <p, q>   | owner pass: alpha_k
//   phase 2: x, r, z updates, <r,z>, <r,r>   | owner pass: beta_k, stop test of problem k
//   phase R (once): per-problem ||b - A x|| for the residual guard
// q = A p is carried by the recurrence A (z + beta p) = A z + beta A p, so the direction update
// rides in the product phase: an iteration is two row phases, two owner passes, four grid barriers.
// After every reduction phase an owner pass (block b finishes problems b, b + G, ...) sums the
// problem's tile partials in a fixed order and writes its scalars, so tiles can be small (the
// largest problems keep every SM busy after the small ones have converged) without each tile
// re-reducing its problem. Barriers are the bounded-spin grid barriers of femk_grid.cuh. No
// reference counterpart (jNO batches only by vmap over right-hand sides,
// tests/test_fem_solver_slots.py:123-132).
//
// The mixed-precision form (k_batch_mixed) runs the same phases on FP32 values and vectors (FP32
// SpMV accumulation, dot products summed in FP64). x stays in FP64; the steps alpha p of a segment
// accumulate in an FP32 vector e that is folded into x (x += e, FP64) after each reliable update.
// Every problem gets FP64 reliable updates, as femk_pcg_mixed does for one problem: when its FP32
// <r, r> fell by delta2 since the last update, met the stop test or hit the cap, the problem's next
// phase 1 replaces r by fp32(b - A (x + e)) with the FP64 values in place of its FP32 product and
// keeps the direction (p and q = A p); its next phase 2 folds e into x in place of a step. The
// problem retires once the FP64 residual meets the stop rule. A replacement thus costs the problem
// two step slots and no extra phase or grid barrier.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "femk_grid.cuh"
#include "femk_internal.cuh"
#include "femk_spmv.cuh"

namespace femk {
namespace {

constexpr int kBT = 512;  // threads per block
constexpr int kL = 8, kU = 2;

struct BatchArgs {
  const int32_t* indptr;
  const int32_t* indices;
  const double* vals;
  // the plan's sliced-ELL copy (sptr == NULL: the products run on the CSR)
  const int64_t* sptr;
  const double* svals;
  const float* svals32;
  const int16_t* sc16;  // int16 column offsets, or NULL: absolute columns in scols
  const int32_t* scols;
  // mixed precision: FP32 values and inner vectors, per-problem update bookkeeping
  const float* vals32;
  float *r32, *z32, *p32, *q32, *d32;
  float* e32;        // FP32 increments of x not yet folded into it
  double* rr_since;  // [nprob] FP64 <r, r> at the last reliable update
  int32_t* upd;      // [nprob] per-problem step mode of the mixed form (0 normal, 1 update requested, 2 replaced)
  int32_t* outer;    // [nprob] FP64 residual evaluations
  double delta2;
  // the mixed form's FP32 product ring (shared memory, 2 stages a warp); ring_stage == 0: off
  int32_t ring_w;      // widest slice (entries a row) a stage holds
  int32_t ring_stage;  // bytes a stage: 32 ring_w FP32 values, then 32 ring_w columns
  int32_t urows;       // rows a vector in the update phase's three ring stages; 0: direct loads
  const int32_t* tile_r0;
  const int32_t* tile_r1;
  const int32_t* tile_prob;
  const int32_t* prob_t0;
  const int32_t* prob_t1;
  int32_t ntiles, nprob, maxiter;
  double tol2, atol2_abs;
  const double* b;
  double* x;
  const double* dinv;
  double *r, *z, *p, *q;
  double* P;      // partials: [7][ntiles]
  double* gam;    // [2][nprob]
  double* atol2;  // [nprob]
  double* rr;     // [nprob]
  double* relres; // [nprob]
  int32_t* iter;  // [nprob]
  int32_t* done;  // [nprob]
  int32_t* status;
  int32_t* active;
  GridBar* bar;
  long long spin;  // clock64 budget of each grid-barrier wait
  int32_t skip;    // testing: block that skips its first barrier arrival (-1: none)
};

// x[j] with a plain (L1-cached) load. The vectors a phase gathers were written in an earlier phase,
// and the grid barrier between the two (fence, then a GPU-scope acquire by every block) makes those
// writes visible to plain loads; the read-only path (__ldg) could return stale lines inside the launch.
template <typename V>
struct GatherPlain {
  const V* x;
  __device__ __forceinline__ V operator()(int64_t j) const { return x[j]; }
  __device__ __forceinline__ V operator()(int32_t j) const { return x[j]; }
};

// 16-byte asynchronous copy global -> shared through L2 (cp.async.cg), and its group bookkeeping
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// x[j] + e[j]: the FP64 iterate plus the FP32 increments not yet folded into it (plain loads, as
// GatherPlain)
struct GatherSum {
  const double* x;
  const float* e;
  __device__ __forceinline__ double operator()(int64_t j) const { return x[j] + (double)e[j]; }
  __device__ __forceinline__ double operator()(int32_t j) const { return x[j] + (double)e[j]; }
};

// One warp computes (A v)[row] for the rows of its tile. pre(row, ok) issues the row's own epilogue
// loads ahead of the product's (ok false: the lane has no row in this slice, load nothing) and
// returns them; post(row, Av, pre's values) finishes the row. V = double: the FP64 values; V = float:
// the FP32 values (FP32 accumulation). On the sliced-ELL copy a lane owns a row of each 32-row slice
// the tile covers (tiles start and end on slice boundaries except at the ends of a problem), every
// value and column load is independent of the others, and the next slice's offset is read while the
// current slice runs; on the CSR kL lanes share a row.
template <typename V, int EB, typename G, typename Pre, typename Post>
__device__ __forceinline__ void tile_product_g(const BatchArgs& a, int32_t r0, int32_t r1, const G& gx, Pre&& pre,
                                               Post&& post) {
  const int lane = threadIdx.x & 31;
  if (a.sptr) {
    const V* vals;
    if constexpr (sizeof(V) == 8)
      vals = a.svals;
    else
      vals = a.svals32;
    const int32_t s0 = r0 >> 5, s1 = (r1 - 1) >> 5;
    int64_t b0 = __ldg(a.sptr + s0), b1 = __ldg(a.sptr + s0 + 1);
    for (int32_t s = s0; s <= s1; ++s) {
      const int64_t b2 = s < s1 ? __ldg(a.sptr + s + 2) : b1;
      const int32_t row = s * 32 + lane;
      const bool ok = row >= r0 && row < r1;
      const auto ld = pre(row, ok);
      const int32_t w = ok ? (int32_t)((b1 - b0) >> 5) : 0;
      const V acc = a.sc16 ? sell_row<V, int16_t, EB>(vals + b0 + lane, a.sc16 + b0 + lane, w, row, gx)
                           : sell_row<V, int32_t, EB>(vals + b0 + lane, a.scols + b0 + lane, w, row, gx);
      if (ok) post((int64_t)row, acc, ld);
      b0 = b1;
      b1 = b2;
    }
    return;
  }
  const int sub = lane % kL;
  constexpr int RPW = 32 / kL;
  const V* vals;
  if constexpr (sizeof(V) == 8)
    vals = a.vals;
  else
    vals = a.vals32;
  for (int64_t base = r0; base < r1; base += RPW * kU) {
    V sv[kU];
    int64_t rows[kU];
    csr_rows_g<kL, kU, V, int32_t>(a.indptr, a.indices, vals, gx, r1, base, lane, sv, rows);
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (rows[u] < r1 && sub == 0) post(rows[u], sv[u], pre(rows[u], true));
  }
}

template <typename V = double, typename Pre, typename Post>
__device__ __forceinline__ void tile_product(const BatchArgs& a, int32_t r0, int32_t r1, const V* v, Pre&& pre,
                                             Post&& post) {
  // 16 entries in flight a lane: a P1 row in one round (FP64 batch 42.4-42.6 ms against 44.7 ms with
  // 8, no spills at the 64-register cap)
  tile_product_g<V, 16>(a, r0, r1, GatherPlain<V>{v}, static_cast<Pre&&>(pre), static_cast<Post&&>(post));
}

// The rows [r0, r1) of a tile, S trips of 32 at a time: load(i) for all S rows of a round first
// (every load of a round in flight together; the stores of a trip may alias the next trip's loads),
// then step(i, loaded values). The kernels use S = 1: at 2 blocks of 512 threads per SM (64
// registers a thread) S = 2 or 4 spilled and the FP64 batch took 50.7 ms against 44.7 ms, and one
// block per SM with S = 4 (104-118 registers) took 66 ms.
template <int S, typename Load, typename Step>
__device__ __forceinline__ void tile_rows(int32_t r0, int32_t r1, Load&& load, Step&& step) {
  const int lane = threadIdx.x & 31;
  for (int32_t i0 = r0 + lane; i0 < r1; i0 += 32 * S) {
    decltype(load(i0)) v[S];
#pragma unroll
    for (int u = 0; u < S; ++u)
      if (i0 + 32 * u < r1) v[u] = load(i0 + 32 * u);
#pragma unroll
    for (int u = 0; u < S; ++u)
      if (i0 + 32 * u < r1) step(i0 + 32 * u, v[u]);
  }
}

// Problem k's sums of the tile partials P[slot[j]][t], t in [t0, t1), for NV slots at once (whole
// block, fixed order, broadcast), with done[k] and the mixed form's mode read in the same round: one
// pair of block barriers per owner pass instead of one per sum and flag.
struct ProbFlags {
  int32_t done, mode;
};
template <int NV>
__device__ __forceinline__ ProbFlags prob_sums(const BatchArgs& a, const int (&slot)[NV], int32_t k, bool mode,
                                               double (&out)[NV]) {
  __shared__ double part[NV][kBT / 32];
  __shared__ ProbFlags fl;
  const int32_t t0 = __ldg(a.prob_t0 + k), t1 = __ldg(a.prob_t1 + k);
  if (threadIdx.x == 0) {
    fl.done = __ldcg(a.done + k);
    fl.mode = mode ? __ldcg(a.upd + k) : 0;
  }
  double t[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) t[j] = 0.0;
  for (int32_t i = t0 + threadIdx.x; i < t1; i += kBT)
#pragma unroll
    for (int j = 0; j < NV; ++j) t[j] += __ldcg(a.P + (int64_t)slot[j] * a.ntiles + i);
#pragma unroll
  for (int j = 0; j < NV; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t[j] += __shfl_xor_sync(0xffffffffu, t[j], o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) part[j][threadIdx.x >> 5] = t[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kBT / 32; ++w) v += part[j][w];
    out[j] = v;
  }
  const ProbFlags f = fl;
  __syncthreads();
  return f;
}

// warp sum of NV values, stored by lane 0 as tile t's partials P[slot0 + j][t]
template <int NV>
__device__ __forceinline__ void tile_partial(double (&v)[NV], double* P, int ntiles, int32_t t, const int slot0) {
#pragma unroll
  for (int j = 0; j < NV; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) P[(int64_t)(slot0 + j) * ntiles + t] = v[j];
  }
}

__device__ __forceinline__ void retire(const BatchArgs& a, int32_t k, int32_t status) {
  a.status[k] = status;
  a.done[k] = 1;
  atomicSub(a.active, 1);
}

// The tiles of one warp (tiles gw, gw + NW, ..., at most 32 of them): lane j holds tile gw + j NW's
// rows and problem, loaded once per launch. A phase then evaluates its filter for all of the warp's
// tiles in one load per lane, where a per-tile loop would wait on a chain of dependent loads
// (tile -> problem -> done flag -> rows) before each tile's work.
struct WarpTiles {
  int32_t r0, r1, k, count;
};

__device__ __forceinline__ WarpTiles warp_tiles(const BatchArgs& a, int32_t gw, int32_t NW) {
  const int lane = threadIdx.x & 31;
  const int64_t t = gw + (int64_t)lane * NW;
  const bool have = t < a.ntiles;
  WarpTiles w;
  w.r0 = have ? a.tile_r0[t] : 0;
  w.r1 = have ? a.tile_r1[t] : 0;
  w.k = have ? a.tile_prob[t] : -1;
  w.count = gw < a.ntiles ? min(32, (a.ntiles - 1 - gw) / NW + 1) : 0;
  return w;
}

// body(t, r0, r1, k) for every tile of the warp whose problem passes keep(k), in tile order; keep is
// evaluated by lane j for the warp's tile j, all lanes at once
template <typename Keep, typename Body>
__device__ __forceinline__ void for_warp_tiles(const WarpTiles& w, int32_t gw, int32_t NW, Keep&& keep, Body&& body) {
  const int lane = threadIdx.x & 31;
  const bool mine = lane < w.count && keep(w.k);
  unsigned int mask = __ballot_sync(0xffffffffu, mine);
  while (mask) {
    const int j = __ffs(mask) - 1;
    mask &= mask - 1;
    body(gw + j * NW, __shfl_sync(0xffffffffu, w.r0, j), __shfl_sync(0xffffffffu, w.r1, j),
         __shfl_sync(0xffffffffu, w.k, j));
  }
}

// As for_warp_tiles, and lane j also fetches scalar(k) and tag(k) for the warp's tile j, so a
// phase that needs a per-problem scalar (alpha_k, beta_k) or mode bit reads them for all of the
// warp's tiles in one load per lane: body(t, r0, r1, k, scalar, tag).
template <typename Keep, typename Scalar, typename Tag, typename Body>
__device__ __forceinline__ void for_warp_tiles_s(const WarpTiles& w, int32_t gw, int32_t NW, Keep&& keep,
                                                 Scalar&& scalar, Tag&& tag, Body&& body) {
  const int lane = threadIdx.x & 31;
  double sc = 0.0;
  bool mine = false, tg = false;
  if (lane < w.count) {  // independent loads, all in flight together
    sc = scalar(w.k);
    mine = keep(w.k);
    tg = tag(w.k);
  }
  const unsigned int tags = __ballot_sync(0xffffffffu, mine && tg);
  unsigned int mask = __ballot_sync(0xffffffffu, mine);
  while (mask) {
    const int j = __ffs(mask) - 1;
    mask &= mask - 1;
    body(gw + j * NW, __shfl_sync(0xffffffffu, w.r0, j), __shfl_sync(0xffffffffu, w.r1, j),
         __shfl_sync(0xffffffffu, w.k, j), __shfl_sync(0xffffffffu, sc, j), ((tags >> j) & 1u) != 0u);
  }
}

// Owner pass: block b finishes problems k = b, b + G, ... from their tile partials.
#define FEMK_OWNER_LOOP for (int32_t k = blockIdx.x; k < a.nprob; k += gridDim.x)

// The FP32 product phase of the mixed form (w = A32 z, p = z + beta p, q = w + beta q, <p, q>) over
// the warp's tiles in `mask`, with each slice's values and columns staged in the warp's two-stage
// shared-memory ring by 16-byte cp.async copies: slice i + 1 is in flight while slice i gathers, so
// a slice waits on its gathers only. A tile's slice offsets sptr[s0 .. s1 + 1] are read one tile
// ahead (lane i holds sptr[s0 + i]). Every cursor below is warp-uniform. The FP32 sums run in the
// order of sell_row, so the products are the bits of the direct path.
__device__ __forceinline__ void product32_ring(const BatchArgs& a, const WarpTiles& wt, int32_t gw, int32_t NW,
                                               unsigned int mask, double beta_lane, char* ring) {
  constexpr unsigned int kFull = 0xffffffffu;
  constexpr int EB = 16;
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  using I = int16_t;  // int16 column offsets (an int32-column instance spilled at the 64-register cap)
  const I* cols = a.sc16;
  const int32_t stage = a.ring_stage;
  const int32_t coff = 128 * a.ring_w;  // the columns follow the values in a stage
  auto first = [&](int j) { return __shfl_sync(kFull, wt.r0, j) >> 5; };
  auto last = [&](int j) { return (__shfl_sync(kFull, wt.r1, j) - 1) >> 5; };
  auto after = [&](int j) {  // the next tile of the mask after tile j, or -1
    const unsigned int rest = j < 31 ? mask & (~0u << (j + 1)) : 0u;
    return rest ? __ffs(rest) - 1 : -1;
  };
  auto offsets = [&](int j) -> int32_t {  // the ring is on only for fewer than 2^31 stored entries
    if (j < 0) return 0;
    const int32_t s0 = first(j), s1 = last(j);
    return lane <= s1 - s0 + 1 ? (int32_t)__ldg(a.sptr + s0 + lane) : 0;
  };
  // prefetch cursor: tile pj, slice ps of [ps0, pe]; pdir its offsets, ndir those of tile pn
  int pj = __ffs(mask) - 1;
  int pn = after(pj);
  int32_t pdir = offsets(pj);
  int32_t ndir = offsets(pn);
  int32_t ps0 = first(pj), ps = ps0, pe = last(pj);
  int32_t w0 = 0, w1 = 0;  // entries a row of the slice in stage 0 / 1
  auto issue = [&](int st) {
    if (pj >= 0) {
      const int32_t b0 = __shfl_sync(kFull, pdir, ps - ps0), b1 = __shfl_sync(kFull, pdir, ps - ps0 + 1);
      const int32_t wd = (int32_t)((b1 - b0) >> 5);
      char* dst = ring + st * stage;
      const char* gv = (const char*)(a.svals32 + b0);
      const char* gc = (const char*)(cols + b0);
      const int32_t nv = 8 * wd;                      // 16-byte chunks of the values (128 wd bytes)
      const int32_t nc = 4 * wd;                      // ... of the columns (64 wd bytes)
      for (int32_t c = lane; c < nv; c += 32) cp_async16(dst + 16 * c, gv + 16 * c);
      for (int32_t c = lane; c < nc; c += 32) cp_async16(dst + coff + 16 * c, gc + 16 * c);
      if (st)
        w1 = wd;
      else
        w0 = wd;
      if (ps < pe) {
        ++ps;
      } else {
        pj = pn;
        if (pj >= 0) {
          pdir = ndir;
          ps0 = ps = first(pj);
          pe = last(pj);
          pn = after(pj);
          ndir = offsets(pn);
        }
      }
    }
    cp_async_commit();  // an empty group once the sequence is exhausted keeps the counts aligned
  };
  issue(0);
  // compute cursor: tile cj, slice cs of [.., ce], rows [r0, r1), its beta
  int cj = __ffs(mask) - 1;
  int32_t cs = first(cj), ce = last(cj);
  int32_t r0 = __shfl_sync(kFull, wt.r0, cj), r1 = __shfl_sync(kFull, wt.r1, cj);
  double be = __shfl_sync(kFull, beta_lane, cj);
  double acc[1] = {0.0};
  for (int it = 0;; ++it) {
    const int st = it & 1;
    __syncwarp();  // every lane is done with the other stage (slice it - 1)
    issue(st ^ 1);
    const int32_t row = cs * 32 + lane;
    const bool ok = row >= r0 && row < r1;
    const bool step = be != 0.0;
    float zr = 0.0f, pr = 0.0f, qr = 0.0f;  // the row's own operands, loaded under the wait
    if (ok) {
      zr = __ldcg(a.z32 + row);
      if (step) {
        pr = __ldcg(a.p32 + row);
        qr = __ldcg(a.q32 + row);
      }
    }
    cp_async_wait<1>();  // this lane's copies of slice it have landed
    __syncwarp();        // ... and every other lane's
    const int32_t wd = ok ? (st ? w1 : w0) : 0;
    const float* sv = (const float*)(ring + st * stage) + lane;
    const I* sc = (const I*)(ring + st * stage + coff) + lane;
    float w = 0.0f;
    for (int32_t k0 = 0; k0 < wd; k0 += EB) {
      float g[EB];  // the gathers first (all in flight), the values re-read from the stage after
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        const int32_t k = (k0 + u) * 32;
        g[u] = k0 + u < wd ? a.z32[row + (int32_t)sc[k]] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < EB; ++u)
        if (k0 + u < wd) w += sv[(k0 + u) * 32] * g[u];
    }
    if (ok) {
      const float bf = (float)be;
      const float pi = step ? fmaf(bf, pr, zr) : zr;
      const float qi = step ? fmaf(bf, qr, w) : w;
      a.p32[row] = pi;
      a.q32[row] = qi;
      acc[0] += (double)pi * (double)qi;
    }
    if (cs < ce) {
      ++cs;
    } else {
      tile_partial<1>(acc, a.P, a.ntiles, gw + cj * NW, 3);
      acc[0] = 0.0;
      cj = after(cj);
      if (cj < 0) break;
      cs = first(cj);
      ce = last(cj);
      r0 = __shfl_sync(kFull, wt.r0, cj);
      r1 = __shfl_sync(kFull, wt.r1, cj);
      be = __shfl_sync(kFull, beta_lane, cj);
    }
  }
  cp_async_wait<0>();
  __syncwarp();
}

// The update phase of the mixed form (e += alpha p, r -= alpha q, z = D^-1 r, <r, z>, <r, r>) over
// the warp's tiles in `mask`, with each tile's e, p, q, r and D staged in the warp's shared-memory
// ring: three stages of a.urows rows a vector, so the next two tiles' operands are in flight while a
// tile computes. A stage holds whole slices (rows 32 s0 to 32 (s1 + 1)), so every copy starts on 16
// bytes and stays inside the vectors' vstride slots. The arithmetic is the direct path's.
__device__ __forceinline__ void update32_ring(const BatchArgs& a, const WarpTiles& wt, int32_t gw, int32_t NW,
                                              unsigned int mask, double al_lane, char* ring) {
  constexpr unsigned int kFull = 0xffffffffu;
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int32_t vrow = a.urows;        // rows of one vector in a stage (a multiple of 32)
  const int32_t sbytes = 5 * 4 * vrow;  // a stage: e, p, q, r, D
  const float* src[5] = {a.e32, a.p32, a.q32, a.r32, a.d32};
  auto after = [&](int j) {
    const unsigned int rest = j < 31 ? mask & (~0u << (j + 1)) : 0u;
    return rest ? __ffs(rest) - 1 : -1;
  };
  int pj = __ffs(mask) - 1;
  auto issue = [&](int st) {
    if (pj >= 0) {
      const int32_t a0 = __shfl_sync(kFull, wt.r0, pj) & ~31;
      const int32_t a1 = (__shfl_sync(kFull, wt.r1, pj) + 31) & ~31;
      const int32_t nch = (a1 - a0) >> 2;  // 16-byte chunks of one vector
      char* dst = ring + st * sbytes;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        for (int32_t c = lane; c < nch; c += 32) cp_async16(dst + v * 4 * vrow + 16 * c, src[v] + a0 + 4 * c);
      pj = after(pj);
    }
    cp_async_commit();
  };
  issue(0);
  issue(1);
  int cj = __ffs(mask) - 1;
  for (int it = 0; cj >= 0; ++it) {
    const int st = it % 3;
    __syncwarp();  // every lane is done with stage (it + 2) % 3 (tile it - 1)
    issue((it + 2) % 3);
    cp_async_wait<2>();  // this lane's copies of tile it have landed
    __syncwarp();        // ... and every other lane's
    const int32_t r0 = __shfl_sync(kFull, wt.r0, cj), r1 = __shfl_sync(kFull, wt.r1, cj);
    const int32_t a0 = r0 & ~31;
    const float alf = (float)__shfl_sync(kFull, al_lane, cj);
    const float* sb = (const float*)(ring + st * sbytes);
    double acc[2] = {0.0, 0.0};
    for (int32_t i = r0 + lane; i < r1; i += 32) {
      const int32_t li = i - a0;
      a.e32[i] = fmaf(alf, sb[vrow + li], sb[li]);
      const float ri = fmaf(-alf, sb[2 * vrow + li], sb[3 * vrow + li]);
      const float zi = sb[4 * vrow + li] * ri;
      a.r32[i] = ri;
      a.z32[i] = zi;
      acc[0] += (double)ri * (double)zi;
      acc[1] += (double)ri * (double)ri;
    }
    tile_partial<2>(acc, a.P, a.ntiles, gw + cj * NW, 4);
    cj = after(cj);
  }
  cp_async_wait<0>();
  __syncwarp();
}

// the vector operands of one row in the update phases
struct RowF64 {
  double x, p, r, q, d;
};
struct RowMixed {
  float e, p, q, r, d;
};

__global__ void __launch_bounds__(kBT, 2) k_batch_pcg(BatchArgs a) {
  unsigned int gen = 0;
  const int32_t gw = (int32_t)((blockIdx.x * (int64_t)kBT + threadIdx.x) >> 5);  // global warp
  const int32_t NW = (int32_t)(((int64_t)gridDim.x * kBT) >> 5);
  const WarpTiles wt = warp_tiles(a, gw, NW);
  auto every = [](int32_t) { return true; };
  auto live = [&](int32_t k) { return __ldcg(a.done + k) == 0; };
  auto no_tag = [](int32_t) { return false; };
  // per-problem step scalars: beta (read by phase 1, written by the second owner pass) and alpha
  // (written by the first owner pass, read by phase 2) are never live together and share a slot
  double* alpha = a.gam + a.nprob;
  double* beta = alpha;
  // ---- phase 0: residual of x0
  for_warp_tiles(wt, gw, NW, every, [&](int32_t t, int32_t tr0, int32_t tr1, int32_t) {
    double acc[3] = {0.0, 0.0, 0.0};
    tile_product(
        a, tr0, tr1, a.x,
        [&](int64_t row, bool ok) { return make_double2(ok ? a.b[row] : 0.0, ok && a.dinv ? a.dinv[row] : 1.0); },
        [&](int64_t row, double s, double2 bd) {
          const double ri = bd.x - s;
          const double zi = a.dinv ? bd.y * ri : ri;
          a.r[row] = ri;
          a.z[row] = zi;
          acc[0] += ri * zi;
          acc[1] += ri * ri;
          acc[2] += bd.x * bd.x;
        });
    tile_partial<3>(acc, a.P, a.ntiles, t, 0);
  });
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  FEMK_OWNER_LOOP {
    double v[3];
    prob_sums<3>(a, {0, 1, 2}, k, false, v);
    const double rz = v[0], rr = v[1], bb = v[2];
    if (threadIdx.x == 0) {
      const double at2 = fmax(a.tol2 * bb, a.atol2_abs);
      a.gam[k] = rz;
      a.rr[k] = rr;
      a.atol2[k] = at2;
      a.iter[k] = 0;
      beta[k] = 0.0;  // the first direction is z itself
      const double rs = a.dinv ? rr : rz;
      if (!isfinite(rz) || !isfinite(rr))
        retire(a, k, FEMK_NONFINITE);
      else if (!(rs > at2) || a.maxiter <= 0)
        retire(a, k, FEMK_OK);
    }
  }
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  while (ld_acquire_u32((const unsigned int*)a.active) != 0u) {
    // ---- phase 1: w = A z; p = z + beta p; q = w + beta q (= A p); <p, q>
    for_warp_tiles_s(
        wt, gw, NW, live, [&](int32_t k) { return __ldcg(beta + k); }, no_tag,
        [&](int32_t t, int32_t tr0, int32_t tr1, int32_t, double be, bool) {
          const bool step = be != 0.0;
          double acc[1] = {0.0};
          tile_product(
              a, tr0, tr1, a.z,
              [&](int64_t row, bool ok) {
                double3 v = make_double3(0.0, 0.0, 0.0);
                if (ok) {
                  v.x = __ldcg(a.z + row);
                  if (step) {
                    v.y = __ldcg(a.p + row);
                    v.z = __ldcg(a.q + row);
                  }
                }
                return v;
              },
              [&](int64_t row, double w, double3 v) {
                const double pi = step ? fma(be, v.y, v.x) : v.x;
                const double qi = step ? fma(be, v.z, w) : w;
                a.p[row] = pi;
                a.q[row] = qi;
                acc[0] += pi * qi;
              });
          tile_partial<1>(acc, a.P, a.ntiles, t, 3);
        });
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    FEMK_OWNER_LOOP {
      double v[1];
      if (prob_sums<1>(a, {3}, k, false, v).done) continue;
      const double pq = v[0];
      if (threadIdx.x == 0) {
        if (!(pq > 0.0) || !isfinite(pq))
          retire(a, k, isfinite(pq) ? FEMK_BREAKDOWN : FEMK_NONFINITE);
        else
          alpha[k] = a.gam[k] / pq;
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    // ---- phase 2: x, r, z updates; <r, z>, <r, r>
    for_warp_tiles_s(
        wt, gw, NW, live, [&](int32_t k) { return __ldcg(alpha + k); }, no_tag,
        [&](int32_t t, int32_t tr0, int32_t tr1, int32_t, double al, bool) {
          double acc[2] = {0.0, 0.0};
          tile_rows<1>(
              tr0, tr1,
              [&](int32_t i) {
                RowF64 v;
                v.x = a.x[i];
                v.p = __ldcg(a.p + i);
                v.r = __ldcg(a.r + i);
                v.q = __ldcg(a.q + i);
                v.d = a.dinv ? a.dinv[i] : 1.0;
                return v;
              },
              [&](int32_t i, const RowF64& v) {
                a.x[i] = v.x + al * v.p;
                const double ri = v.r - al * v.q;
                const double zi = a.dinv ? v.d * ri : ri;
                a.r[i] = ri;
                a.z[i] = zi;
                acc[0] += ri * zi;
                acc[1] += ri * ri;
              });
          tile_partial<2>(acc, a.P, a.ntiles, t, 4);
        });
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    FEMK_OWNER_LOOP {
      double v[2];
      if (prob_sums<2>(a, {4, 5}, k, false, v).done) continue;
      const double rz = v[0], rr = v[1];
      if (threadIdx.x == 0) {
        const int32_t itk = a.iter[k] + 1;
        const double rs = a.dinv ? rr : rz;
        const bool finite = isfinite(rz) && isfinite(rr);
        beta[k] = rz / a.gam[k];
        a.gam[k] = rz;
        a.rr[k] = rr;
        a.iter[k] = itk;
        if (!finite || !(rs > a.atol2[k]) || itk >= a.maxiter) retire(a, k, finite ? FEMK_OK : FEMK_NONFINITE);
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  }
  // ---- phase R: per-problem ||b - A x||, ||b||
  for_warp_tiles(wt, gw, NW, every, [&](int32_t t, int32_t tr0, int32_t tr1, int32_t) {
    double acc[2] = {0.0, 0.0};
    tile_product(
        a, tr0, tr1, a.x, [&](int64_t row, bool ok) { return ok ? a.b[row] : 0.0; },
        [&](int64_t, double s, double bi) {
          const double w = bi - s;
          acc[0] += w * w;
          acc[1] += bi * bi;
        });
    tile_partial<2>(acc, a.P, a.ntiles, t, 5);
  });
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  FEMK_OWNER_LOOP {
    double v[2];
    prob_sums<2>(a, {5, 6}, k, false, v);
    const double ww = v[0], bb = v[1];
    if (threadIdx.x == 0) a.relres[k] = sqrt(ww) / (sqrt(bb) + 1e-30);
  }
}

__global__ void __launch_bounds__(kBT, 2) k_batch_mixed(BatchArgs a) {
  extern __shared__ __align__(16) char batch_ring[];  // 2 a.ring_stage bytes a warp when the ring is on
  unsigned int gen = 0;
  const int32_t gw = (int32_t)((blockIdx.x * (int64_t)kBT + threadIdx.x) >> 5);  // global warp
  const int32_t NW = (int32_t)(((int64_t)gridDim.x * kBT) >> 5);
  const WarpTiles wt = warp_tiles(a, gw, NW);
  auto every = [](int32_t) { return true; };
  double* alpha = a.gam + a.nprob;
  double* beta = alpha;
  // ---- phase 0: FP64 residual of x0, FP32 copies; <r, z> (FP32 data), <r64, r64>, <b, b>
  for_warp_tiles(wt, gw, NW, every, [&](int32_t t, int32_t tr0, int32_t tr1, int32_t) {
    double acc[3] = {0.0, 0.0, 0.0};
    tile_product<double>(
        a, tr0, tr1, a.x,
        [&](int64_t row, bool ok) { return make_double2(ok ? a.b[row] : 0.0, ok && a.dinv ? a.dinv[row] : 1.0); },
        [&](int64_t row, double s, double2 bd) {
          const double r64 = bd.x - s;
          const float d = a.dinv ? (float)bd.y : 1.0f;
          const float rf = (float)r64;
          const float zf = d * rf;
          a.d32[row] = d;
          a.r32[row] = rf;
          a.z32[row] = zf;
          a.e32[row] = 0.0f;
          acc[0] += (double)rf * (double)zf;
          acc[1] += r64 * r64;
          acc[2] += bd.x * bd.x;
        });
    tile_partial<3>(acc, a.P, a.ntiles, t, 0);
  });
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  FEMK_OWNER_LOOP {
    double v[3];
    prob_sums<3>(a, {0, 1, 2}, k, false, v);
    const double rz = v[0], rr = v[1], bb = v[2];
    if (threadIdx.x == 0) {
      const double at2 = fmax(a.tol2 * bb, a.atol2_abs);
      a.gam[k] = rz;
      a.rr[k] = rr;
      a.rr_since[k] = rr;
      a.atol2[k] = at2;
      a.iter[k] = 0;
      a.outer[k] = 1;
      a.upd[k] = 0;
      beta[k] = 0.0;
      if (!isfinite(rz) || !isfinite(rr))
        retire(a, k, FEMK_NONFINITE);
      else if (!(rr > at2) || a.maxiter <= 0)
        retire(a, k, FEMK_OK);
    }
  }
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  // Per-problem mode (a.upd): 0 a normal step; 1 a reliable update was requested, so the next
  // phase 1 computes the FP64 residual in place of the FP32 product and leaves p and q alone; 2 the
  // residual was replaced in phase 1, so phase 2 skips the problem and the next phase 1 forms the
  // kept direction with beta = <r, z>_new / gamma. Only the owner passes change a mode, so every
  // phase sees one value per iteration, and no iteration needs an extra phase.
  while (ld_acquire_u32((const unsigned int*)a.active) != 0u) {
    // ---- phase 1: w = A32 z, p = z + beta p, q = w + beta q (= A32 p) (FP32), <p, q>;
    //      or (mode 1) r = fp32(b - A64 (x + e)), z = D^-1 r, <r, z>, <r64, r64>
    {
      const int lane = threadIdx.x & 31;
      double be_l = 0.0;
      bool lv = false, rp = false;
      if (lane < wt.count) {  // independent loads, all in flight together
        be_l = __ldcg(beta + wt.k);
        lv = __ldcg(a.done + wt.k) == 0;
        rp = __ldcg(a.upd + wt.k) == 1;
      }
      const unsigned int m_rep = __ballot_sync(0xffffffffu, lv && rp);
      const unsigned int m_step = __ballot_sync(0xffffffffu, lv && !rp);
      for (unsigned int m = m_rep; m; m &= m - 1) {
        const int j = __ffs(m) - 1;
        double acc[2] = {0.0, 0.0};
        tile_product_g<double, 4>(  // two gathers an entry: 4 entries in flight keep it unspilled
            a, __shfl_sync(0xffffffffu, wt.r0, j), __shfl_sync(0xffffffffu, wt.r1, j), GatherSum{a.x, a.e32},
            [&](int64_t row, bool ok) { return make_double2(ok ? a.b[row] : 0.0, ok ? (double)a.d32[row] : 0.0); },
            [&](int64_t row, double sv, double2 bd) {
              const double r64 = bd.x - sv;
              const float rf = (float)r64;
              const float zf = (float)bd.y * rf;
              a.r32[row] = rf;
              a.z32[row] = zf;
              acc[0] += (double)rf * (double)zf;
              acc[1] += r64 * r64;
            });
        tile_partial<2>(acc, a.P, a.ntiles, gw + j * NW, 4);
      }
      if (a.ring_stage) {
        char* ring = batch_ring + (threadIdx.x >> 5) * 2 * a.ring_stage;
        product32_ring(a, wt, gw, NW, m_step, be_l, ring);  // the host turns it on with int16 columns only
      } else {
        for (unsigned int m = m_step; m; m &= m - 1) {
          const int j = __ffs(m) - 1;
          const double be = __shfl_sync(0xffffffffu, be_l, j);
          const bool step = be != 0.0;
          const float bf = (float)be;
          double acc[1] = {0.0};
          tile_product<float>(
              a, __shfl_sync(0xffffffffu, wt.r0, j), __shfl_sync(0xffffffffu, wt.r1, j), a.z32,
              [&](int64_t row, bool ok) {
                float3 v = make_float3(0.0f, 0.0f, 0.0f);
                if (ok) {
                  v.x = __ldcg(a.z32 + row);
                  if (step) {
                    v.y = __ldcg(a.p32 + row);
                    v.z = __ldcg(a.q32 + row);
                  }
                }
                return v;
              },
              [&](int64_t row, float w, float3 v) {
                const float pi = step ? fmaf(bf, v.y, v.x) : v.x;
                const float qi = step ? fmaf(bf, v.z, w) : w;
                a.p32[row] = pi;
                a.q32[row] = qi;
                acc[0] += (double)pi * (double)qi;
              });
          tile_partial<1>(acc, a.P, a.ntiles, gw + j * NW, 3);
        }
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    FEMK_OWNER_LOOP {
      double v[3];  // slot 3 (<p, q>) of a step, slots 4, 5 (<r, z>, <r64, r64>) of a replacement
      const ProbFlags f = prob_sums<3>(a, {3, 4, 5}, k, true, v);
      if (f.done) continue;
      if (f.mode == 1) {
        const double rz = v[1], rr = v[2];
        if (threadIdx.x == 0) {
          a.outer[k] += 1;
          a.rr[k] = rr;
          if (!isfinite(rz) || !isfinite(rr)) {
            retire(a, k, FEMK_NONFINITE);
          } else if (!(rr > a.atol2[k]) || a.iter[k] >= a.maxiter) {
            retire(a, k, FEMK_OK);
          } else {
            beta[k] = rz / a.gam[k];  // residual replacement keeps the search direction
            a.gam[k] = rz;
            a.rr_since[k] = rr;
            a.upd[k] = 2;
          }
        }
      } else {
        const double pq = v[0];
        if (threadIdx.x == 0) {
          if (!(pq > 0.0) || !isfinite(pq))
            retire(a, k, isfinite(pq) ? FEMK_BREAKDOWN : FEMK_NONFINITE);
          else
            alpha[k] = a.gam[k] / pq;
        }
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    // ---- phase 2: (mode 0) e += alpha p, r -= alpha q, z = D^-1 r (FP32); <r, z>, <r, r>;
    //      (mode 2, the residual was just replaced) x += e (FP64), e = 0
    {
      const int lane = threadIdx.x & 31;
      double al_l = 0.0;
      bool lv = false;
      int32_t md = 1;
      if (lane < wt.count) {  // independent loads, all in flight together
        al_l = __ldcg(alpha + wt.k);
        lv = __ldcg(a.done + wt.k) == 0;
        md = __ldcg(a.upd + wt.k);
      }
      const unsigned int m_fold = __ballot_sync(0xffffffffu, lv && md == 2);
      const unsigned int m_step = __ballot_sync(0xffffffffu, lv && md == 0);
      for (unsigned int m = m_fold; m; m &= m - 1) {
        const int j = __ffs(m) - 1;
        const int32_t tr1 = __shfl_sync(0xffffffffu, wt.r1, j);
        for (int32_t i = __shfl_sync(0xffffffffu, wt.r0, j) + lane; i < tr1; i += 32) {
          a.x[i] = a.x[i] + (double)__ldcg(a.e32 + i);
          a.e32[i] = 0.0f;
        }
      }
      if (a.urows) {
        update32_ring(a, wt, gw, NW, m_step, al_l, batch_ring + (threadIdx.x >> 5) * 2 * a.ring_stage);
      } else {
        for (unsigned int m = m_step; m; m &= m - 1) {
          const int j = __ffs(m) - 1;
          const float alf = (float)__shfl_sync(0xffffffffu, al_l, j);
          double acc[2] = {0.0, 0.0};
          tile_rows<1>(
              __shfl_sync(0xffffffffu, wt.r0, j), __shfl_sync(0xffffffffu, wt.r1, j),
              [&](int32_t i) {
                RowMixed v;
                v.e = __ldcg(a.e32 + i);
                v.p = __ldcg(a.p32 + i);
                v.q = __ldcg(a.q32 + i);
                v.r = __ldcg(a.r32 + i);
                v.d = a.d32[i];
                return v;
              },
              [&](int32_t i, const RowMixed& v) {
                a.e32[i] = fmaf(alf, v.p, v.e);
                const float ri = fmaf(-alf, v.q, v.r);
                const float zi = v.d * ri;
                a.r32[i] = ri;
                a.z32[i] = zi;
                acc[0] += (double)ri * (double)zi;
                acc[1] += (double)ri * (double)ri;
              });
          tile_partial<2>(acc, a.P, a.ntiles, gw + j * NW, 4);
        }
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
    FEMK_OWNER_LOOP {
      double v[2];
      const ProbFlags f = prob_sums<2>(a, {4, 5}, k, true, v);
      if (f.done) continue;
      if (f.mode == 2) {  // the direction step of the replaced residual runs in the next phase 1
        if (threadIdx.x == 0) a.upd[k] = 0;
        continue;
      }
      const double rz = v[0], rr = v[1];
      if (threadIdx.x == 0) {
        const int32_t itk = a.iter[k] + 1;
        a.iter[k] = itk;
        if (!isfinite(rz) || !isfinite(rr)) {
          retire(a, k, FEMK_NONFINITE);
        } else if (!(rr > a.atol2[k]) || rr < a.delta2 * a.rr_since[k] || itk >= a.maxiter) {
          a.upd[k] = 1;  // FP64 residual replacement in the next phase 1; p and q stay as they are
        } else {
          beta[k] = rz / a.gam[k];
          a.gam[k] = rz;
          a.rr[k] = rr;
        }
      }
    }
    if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  }
  // ---- fold: x += e for every problem (a problem that retired on a replaced residual still holds
  // the increments of its last segment)
  for_warp_tiles(wt, gw, NW, every, [&](int32_t, int32_t tr0, int32_t tr1, int32_t) {
    for (int32_t i = tr0 + (threadIdx.x & 31); i < tr1; i += 32) a.x[i] = a.x[i] + (double)__ldcg(a.e32 + i);
  });
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  // ---- phase R: per-problem ||b - A x||, ||b|| (FP64)
  for_warp_tiles(wt, gw, NW, every, [&](int32_t t, int32_t tr0, int32_t tr1, int32_t) {
    double acc[2] = {0.0, 0.0};
    tile_product<double>(
        a, tr0, tr1, a.x, [&](int64_t row, bool ok) { return ok ? a.b[row] : 0.0; },
        [&](int64_t, double s, double bi) {
          const double w = bi - s;
          acc[0] += w * w;
          acc[1] += bi * bi;
        });
    tile_partial<2>(acc, a.P, a.ntiles, t, 5);
  });
  if (!grid_sync(a.bar, gen, a.spin, a.skip)) return;
  FEMK_OWNER_LOOP {
    double v[2];
    prob_sums<2>(a, {5, 6}, k, false, v);
    const double ww = v[0], bb = v[1];
    if (threadIdx.x == 0) a.relres[k] = sqrt(ww) / (sqrt(bb) + 1e-30);
  }
}

__global__ void k_to_f32(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void k_batch_reset(int32_t* done, int32_t* status, int32_t* active, int32_t nprob, GridBar* bar) {
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nprob; k += gridDim.x * blockDim.x) {
    done[k] = 0;
    status[k] = FEMK_OK;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *active = nprob;
    bar->count = 0;
    bar->gen = 0;
    bar->timeout = 0;
  }
}

}  // namespace
}  // namespace femk

using namespace femk;

namespace {

int batched_impl(const femk_plan* pc, int32_t nprob, const int64_t* row_off, const double* vals, const double* b,
                 double* x, const double* dinv, double tol, double atol, int32_t maxiter, int32_t tile_rows,
                 int32_t blocks_per_sm, int32_t* iters_out, int32_t* outer_out, double* relres_out,
                 int32_t* status_out, void* stream, bool mixed, double delta2) {
  FEMK_CHECK_ARG(pc && row_off && vals && b && x, "femk_pcg_batched: NULL argument");
  FEMK_CHECK_ARG(nprob >= 1, "femk_pcg_batched: nprob must be >= 1");
  FEMK_CHECK_ARG(tile_rows >= 32 && tile_rows <= (1 << 20), "femk_pcg_batched: tile_rows out of range");
  FEMK_CHECK_ARG(blocks_per_sm >= 1 && blocks_per_sm <= 2, "femk_pcg_batched: blocks_per_sm must be 1 or 2");
  FEMK_CHECK_ARG(pc->coop, "femk_pcg_batched: the device does not support cooperative launch");
  femk_plan* p = const_cast<femk_plan*>(pc);
  FEMK_CHECK_ARG(row_off[0] == 0 && row_off[nprob] == p->n, "femk_pcg_batched: row_off must span [0, n)");
  for (int32_t k = 0; k < nprob; ++k) FEMK_CHECK_ARG(row_off[k + 1] > row_off[k], "femk_pcg_batched: empty problem");
  const void* kern = mixed ? (const void*)k_batch_mixed : (const void*)k_batch_pcg;
  // The mixed form's FP32 products stream each slice through a two-stage shared-memory ring a warp
  // (int16 columns, rows of at most 16 entries: 96 KB a block, so 2 blocks of 512 fit an SM)
  const int32_t ring_w = std::max(1, p->max_row);
  const int32_t ring_stage = 32 * ring_w * (4 + 2);
  const int ring_smem = (kBT / 32) * 2 * ring_stage;
  bool ring = mixed && p->use_sell && p->sell_cols && p->sell_c16 && ((uintptr_t)p->sell_c16 & 15u) == 0 &&
              p->sell_nnz < ((int64_t)1 << 31) && ring_smem <= 100 * 1024;
  int per_sm = 0;
  if (ring) {
    if (cudaFuncSetAttribute(k_batch_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, ring_smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_mixed, kBT, ring_smem) != cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      ring = false;
    }
  }
  per_sm = std::min(blocks_per_sm, ring ? per_sm : resident_blocks(kern, kBT));
  const int grid = p->n_sm * std::max(1, per_sm);
  const int64_t nwarps = (int64_t)grid * (kBT / 32);
  // tiles: on the sliced-ELL copy they end on global multiples of tile_rows (rounded up to a whole
  // slice), so only the first and last tile of a problem cover part of a slice. A warp holds at
  // most 32 tiles (one per lane), so tile_rows doubles until the tiles fit.
  const bool sell = p->use_sell && p->sell_cols;
  int64_t tr = sell ? (tile_rows + 31) / 32 * 32 : tile_rows;
  std::vector<int32_t> r0, r1, tp, t0(nprob), t1(nprob);
  while (true) {
    r0.clear();
    r1.clear();
    tp.clear();
    for (int32_t k = 0; k < nprob; ++k) {
      t0[k] = (int32_t)r0.size();
      for (int64_t s0 = row_off[k]; s0 < row_off[k + 1];) {
        const int64_t e = std::min<int64_t>(sell ? (s0 / tr + 1) * tr : s0 + tr, row_off[k + 1]);
        r0.push_back((int32_t)s0);
        r1.push_back((int32_t)e);
        tp.push_back(k);
        s0 = e;
      }
      t1[k] = (int32_t)r0.size();
    }
    if ((int64_t)r0.size() <= 32 * nwarps) break;
    tr *= 2;
  }
  const int32_t ntiles = (int32_t)r0.size();
  ring = ring && tr <= 512;  // a tile's slice offsets (at most tr / 32 + 2) sit one a lane
  const int launch_smem = ring ? ring_smem : 0;
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(ensure_workspace(p));
  // batch workspace: ints (tiles + per-problem), doubles (partials + per-problem)
  const int64_t nint = 3 * (int64_t)ntiles + 7 * (int64_t)nprob + 8;
  const int64_t ndbl = 7 * (int64_t)ntiles + 7 * (int64_t)nprob + 8;
  const int64_t bytes = nint * 4 + 64 + ndbl * 8;
  if (p->batch_bytes < bytes) {
    if (p->batch_ws) cudaFree(p->batch_ws);
    p->batch_ws = nullptr;
    p->batch_bytes = 0;
    FEMK_CUDA_TRY(cudaMalloc(&p->batch_ws, bytes));
    p->batch_bytes = bytes;
  }
  int32_t* ib = (int32_t*)p->batch_ws;
  double* db = (double*)((char*)p->batch_ws + ((nint * 4 + 63) & ~int64_t(63)));
  BatchArgs a;
  a.indptr = p->indptr;
  a.indices = p->indices;
  a.vals = vals;
  a.sptr = nullptr;
  a.svals = nullptr;
  a.svals32 = nullptr;
  a.sc16 = nullptr;
  a.scols = nullptr;
  if (sell) {
    FEMK_TRY(ensure_sell_values(p, mixed));
    a.sptr = p->sell_ptr;
    a.svals = p->sell_vals;
    a.svals32 = mixed ? p->sell_vals32 : nullptr;
    a.sc16 = p->sell_c16;
    a.scols = p->sell_cols;
  }
  a.tile_r0 = ib;
  a.tile_r1 = ib + ntiles;
  a.tile_prob = ib + 2 * ntiles;
  a.prob_t0 = ib + 3 * ntiles;
  a.prob_t1 = a.prob_t0 + nprob;
  a.iter = const_cast<int32_t*>(a.prob_t1) + nprob;
  a.done = a.iter + nprob;
  a.status = a.done + nprob;
  a.active = a.status + nprob;
  a.ntiles = ntiles;
  a.nprob = nprob;
  a.maxiter = maxiter;
  a.tol2 = tol * tol;
  a.atol2_abs = atol * atol;
  a.b = b;
  a.x = x;
  a.dinv = dinv;
  const int64_t vs = p->vstride;
  a.r = p->work;
  a.z = a.r + vs;
  a.p = a.z + vs;
  a.q = a.p + vs;
  a.P = db;
  a.gam = db + 7 * (int64_t)ntiles;
  a.atol2 = a.gam + 2 * nprob;
  a.rr = a.atol2 + nprob;
  a.relres = a.rr + nprob;
  a.rr_since = a.relres + nprob;
  a.upd = a.active + 1;
  a.outer = a.upd + nprob;
  a.delta2 = delta2;
  a.ring_w = ring_w;
  a.ring_stage = ring ? ring_stage : 0;
  // the update phase's ring: three stages of e, p, q, r, D for a tile's whole slices (tr + 32 rows)
  a.urows = ring && 3 * 5 * 4 * (int32_t)(tr + 32) <= 2 * ring_stage ? (int32_t)(tr + 32) : 0;
  a.vals32 = nullptr;
  a.r32 = a.z32 = a.p32 = a.q32 = a.d32 = a.e32 = nullptr;
  if (mixed) {
    if (!sell && !p->vals32) FEMK_CUDA_TRY(cudaMalloc(&p->vals32, sizeof(float) * (p->nnz + 1)));
    if (!p->work32) FEMK_CUDA_TRY(cudaMalloc(&p->work32, sizeof(float) * kWork32Vectors * p->vstride));
    a.vals32 = p->vals32;
    a.r32 = p->work32;
    a.z32 = a.r32 + vs;
    a.p32 = a.z32 + vs;
    a.q32 = a.p32 + vs;
    a.d32 = a.q32 + vs;
    a.e32 = a.d32 + vs;
  }
  a.bar = (GridBar*)p->bar;
  a.spin = p->barrier_spin;
  a.skip = p->skip_arrival;
  // tile tables: uploaded only when the schedule changes (pageable copies stay outside the graph)
  uint64_t h = 1469598103934665603ull;
  for (int32_t k = 0; k <= nprob; ++k) h = (h ^ (uint64_t)row_off[k]) * 1099511628211ull;
  h = (h ^ (uint64_t)tr) * 1099511628211ull;
  h = (h ^ (uint64_t)grid) * 1099511628211ull;
  h = (h ^ (uint64_t)launch_smem) * 1099511628211ull;
  const bool same_tiles = p->batch_key[0] == (const void*)(uintptr_t)h && p->batch_key[1] == p->batch_ws;
  if (!same_tiles) {
    FEMK_CUDA_TRY(cudaMemcpyAsync(ib, r0.data(), 4 * ntiles, cudaMemcpyHostToDevice, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(ib + ntiles, r1.data(), 4 * ntiles, cudaMemcpyHostToDevice, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(ib + 2 * ntiles, tp.data(), 4 * ntiles, cudaMemcpyHostToDevice, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(ib + 3 * ntiles, t0.data(), 4 * nprob, cudaMemcpyHostToDevice, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(ib + 3 * ntiles + nprob, t1.data(), 4 * nprob, cudaMemcpyHostToDevice, s));
  }
  const int cgrid = blocks_for(p->nnz, 256, p->n_sm * 8);
  // the solve itself (reset + one cooperative launch) is one CUDA graph, replayed while the
  // operands and the schedule stay the same; a device that refuses to capture the cooperative
  // launch gets the same two launches directly
  const void* key[8] = {(const void*)(uintptr_t)h, p->batch_ws, vals, b, x, dinv,
                        (const void*)(uintptr_t)grid,
                        (const void*)(uintptr_t)(((uint64_t)maxiter << 1) | (mixed ? 1u : 0u))};
  bool have = p->batch_exec != nullptr;
  for (int i = 0; i < 8 && have; ++i) have = key[i] == p->batch_key[i];
  if (!have && p->batch_graph_ok) {
    if (p->batch_exec) cudaGraphExecDestroy(p->batch_exec);
    p->batch_exec = nullptr;
    if (!p->batch_stream) FEMK_CUDA_TRY(cudaStreamCreateWithFlags(&p->batch_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    set_capturing(true);
    cudaError_t e = cudaStreamBeginCapture(p->batch_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      k_batch_reset<<<8, 256, 0, p->batch_stream>>>(a.done, a.status, a.active, nprob, a.bar);
      if (sell)
        (void)launch_sell_values(p, vals, mixed, p->batch_stream);
      else if (mixed)
        k_to_f32<<<cgrid, 256, 0, p->batch_stream>>>(vals, p->nnz, p->vals32);
      void* cargs[] = {(void*)&a};
      cudaError_t el = cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kBT), cargs, launch_smem, p->batch_stream);
      cudaError_t ee = cudaStreamEndCapture(p->batch_stream, &g);
      if (el == cudaSuccess && ee == cudaSuccess && g) e = cudaGraphInstantiate(&p->batch_exec, g, 0);
      else e = el != cudaSuccess ? el : ee;
    }
    set_capturing(false);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess || !p->batch_exec) {
      cudaGetLastError();
      p->batch_exec = nullptr;
      p->batch_graph_ok = 0;  // fall back to direct launches from now on
    } else {
      for (int i = 0; i < 8; ++i) p->batch_key[i] = key[i];
      have = true;
    }
  }
  if (have && p->batch_exec) {
    if (!p->batch_ev) FEMK_CUDA_TRY(cudaEventCreateWithFlags(&p->batch_ev, cudaEventDisableTiming));
    FEMK_CUDA_TRY(cudaEventRecord(p->batch_ev, s));
    FEMK_CUDA_TRY(cudaStreamWaitEvent(p->batch_stream, p->batch_ev, 0));
    FEMK_CUDA_TRY(cudaGraphLaunch(p->batch_exec, p->batch_stream));
    count_launches(2 + (sell ? (mixed ? 2 : 1) : (mixed ? 1 : 0)));
    p->batch_graph_used = 1;
    FEMK_CUDA_TRY(cudaEventRecord(p->batch_ev, p->batch_stream));
    FEMK_CUDA_TRY(cudaStreamWaitEvent(s, p->batch_ev, 0));
  } else {
    k_batch_reset<<<::femk::counted_launch() + 8, 256, 0, s>>>(a.done, a.status, a.active, nprob, a.bar);
    if (sell)
      FEMK_TRY(launch_sell_values(p, vals, mixed, s));
    else if (mixed)
      k_to_f32<<<::femk::counted_launch() + cgrid, 256, 0, s>>>(vals, p->nnz, p->vals32);
    FEMK_CUDA_TRY(cudaGetLastError());
    void* args[] = {(void*)&a};
    counted_launch();
    FEMK_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kBT), args, launch_smem, s));
    p->batch_key[0] = (const void*)(uintptr_t)h;
    p->batch_key[1] = p->batch_ws;
    p->batch_graph_used = 0;
  }
  std::vector<int32_t> it(nprob), stv(nprob), outer(nprob);
  std::vector<double> rel(nprob);
  unsigned int timeout = 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(it.data(), a.iter, 4 * nprob, cudaMemcpyDeviceToHost, s));
  if (mixed) FEMK_CUDA_TRY(cudaMemcpyAsync(outer.data(), a.outer, 4 * nprob, cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(stv.data(), a.status, 4 * nprob, cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(rel.data(), a.relres, 8 * nprob, cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(&timeout, &a.bar->timeout, 4, cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters_out) std::copy(it.begin(), it.end(), iters_out);
  if (outer_out && mixed) std::copy(outer.begin(), outer.end(), outer_out);
  if (relres_out) std::copy(rel.begin(), rel.end(), relres_out);
  if (status_out) std::copy(stv.begin(), stv.end(), status_out);
  if (timeout) {
    set_error("femk_pcg_batched: a grid barrier gave up waiting");
    return FEMK_TIMEOUT;
  }
  int worst = FEMK_OK;
  for (int32_t k = 0; k < nprob; ++k) {
    if (stv[k] != FEMK_OK) worst = stv[k];
  }
  if (worst != FEMK_OK) {
    set_error("femk_pcg_batched: at least one problem did not solve (see status_out)");
    return worst;
  }
  return FEMK_OK;
}

}  // namespace

extern "C" int femk_pcg_batched(const femk_plan* pc, int32_t nprob, const int64_t* row_off, const double* vals,
                                const double* b, double* x, const double* dinv, double tol, double atol,
                                int32_t maxiter, int32_t tile_rows, int32_t blocks_per_sm, int32_t* iters_out,
                                double* relres_out, int32_t* status_out, void* stream) {
  clear_error();
  return batched_impl(pc, nprob, row_off, vals, b, x, dinv, tol, atol, maxiter, tile_rows, blocks_per_sm, iters_out,
                      nullptr, relres_out, status_out, stream, false, 0.0);
}

extern "C" int femk_pcg_batched_mixed(const femk_plan* pc, int32_t nprob, const int64_t* row_off, const double* vals,
                                      const double* b, double* x, const double* dinv, double tol, double atol,
                                      int32_t maxiter, int32_t tile_rows, int32_t blocks_per_sm, int32_t* iters_out,
                                      int32_t* outer_out, double* relres_out, int32_t* status_out, void* stream) {
  clear_error();
  // reliable-update threshold of the single-problem mixed solver (femk_pcg_mixed)
  const double delta2 = pc && pc->mixed_delta2 > 0.0 ? pc->mixed_delta2 : 1e-4;
  return batched_impl(pc, nprob, row_off, vals, b, x, dinv, tol, atol, maxiter, tile_rows, blocks_per_sm, iters_out,
                      outer_out, relres_out, status_out, stream, true, delta2);
}
