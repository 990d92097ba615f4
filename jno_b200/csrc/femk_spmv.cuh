// CSR row sums with several rows' loads in flight per lane group (device, FP64 or FP32).
//
// A warp owns RPW*U consecutive rows per step: lanes [g*L, (g+1)*L) work on rows base + u*RPW + g,
// u = 0..U-1 (RPW = 32/L). All U row extents are loaded first, then the first L-wide slice of
// every row's values and columns, then all U gathers of x, so each lane keeps U independent
// chains of HBM loads in flight instead of one. Rows longer than L continue in a tail loop (rare
// for P1, where interior rows hold 15 entries). Values and column indices are streamed with
// evict-first loads (__ldcs) so they do not push the solver vectors out of L2; x is gathered
// through the read-only path.
#pragma once

#include <stdint.h>

#include <type_traits>

#include "femk_internal.cuh"
#include "femk_l2.cuh"

namespace femk {

// column of entry k of `row`: an absolute int32 index, or an int16 offset from the row
__device__ __forceinline__ int64_t col_at(const int32_t* __restrict__ cols, int32_t k, int64_t) {
  return (int64_t)__ldcs(cols + k);
}
__device__ __forceinline__ int64_t col_at(const int16_t* __restrict__ cols, int32_t k, int64_t row) {
  return row + (int64_t)__ldcs(cols + k);
}

// Sliced-ELL copy of CSR values, one warp per 32-row slice (global warp g takes slices g, g + NW,
// ...): rows 32s ... 32s+31 are one contiguous CSR range, read coalesced into the warp's shared
// buffer wbuf (room for 32 rows of the plan's longest row), then entry k of row 32s + l is written
// to out[sptr[s] + 32 k + l] as f(value, row, out index), and padding past the row's length as 0.
// Both the reads and the writes are coalesced; only the shared-memory reads are strided.
template <typename T, typename F>
__device__ __forceinline__ void sell_transpose_warp(double* wbuf, int32_t cap, const int64_t* __restrict__ sptr,
                                                    const int32_t* __restrict__ indptr, int64_t n, int64_t nslices,
                                                    const double* __restrict__ vals, int64_t nnz, T* __restrict__ out,
                                                    int64_t g, int64_t NW, F f, int* err) {
  const int lane = threadIdx.x & 31;
  for (int64_t sl = g; sl < nslices; sl += NW) {
    const int64_t r0 = sl * 32, row = r0 + lane;
    const int64_t rl = r0 + 32 < n ? r0 + 32 : n;
    const int32_t base = __ldg(indptr + r0);
    const int32_t end = __ldg(indptr + rl);
    for (int32_t e = base + lane; e < end; e += 32)
      if (FEMK_IN_BOUNDS(e - base, cap, err) && FEMK_IN_BOUNDS(e, nnz, err)) wbuf[e - base] = __ldcs(vals + e);
    __syncwarp();
    const int32_t beg = row < n ? __ldg(indptr + row) - base : 0;
    const int32_t len = row < n ? __ldg(indptr + row + 1) - base - beg : 0;
    const int64_t b0 = sptr[sl] + lane;
    const int32_t w = (int32_t)((sptr[sl + 1] - sptr[sl]) >> 5);
    for (int32_t k = 0; k < w; ++k) {
      const int64_t j = b0 + 32 * k;
      out[j] = (k < len && FEMK_IN_BOUNDS(beg + k, cap, err)) ? f(wbuf[beg + k], row, j) : T(0);
    }
    __syncwarp();  // the buffer is refilled for the next slice
  }
}

// gather functors: x[j], or the CG direction z[j] + beta p[j] formed on the fly
template <typename V>
struct GatherX {
  const V* __restrict__ x;
  __device__ __forceinline__ V operator()(int64_t j) const { return __ldg(x + j); }
  __device__ __forceinline__ V operator()(int32_t j) const { return __ldg(x + j); }  // 32-bit index math
};
// x[j] through L2 only: for vectors that other blocks rewrite inside the same (persistent) launch,
// where the non-coherent read-only path could return a stale line
template <typename V>
struct GatherXcg {
  const V* __restrict__ x;
  __device__ __forceinline__ V operator()(int64_t j) const { return __ldcg(x + j); }
};
// x[j] through the read-only path with an L2 evict_last hint (vectors stay resident)
template <typename V>
struct GatherXL {
  const V* __restrict__ x;
  uint64_t pol;
  __device__ __forceinline__ V operator()(int64_t j) const;
  __device__ __forceinline__ V operator()(int32_t j) const { return (*this)((int64_t)j); }
};
template <>
__device__ __forceinline__ double GatherXL<double>::operator()(int64_t j) const {
  double v;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(x + j), "l"(pol));
  return v;
}
template <>
__device__ __forceinline__ float GatherXL<float>::operator()(int64_t j) const {
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(x + j), "l"(pol));
  return v;
}

struct GatherDirection {
  const double* __restrict__ z;
  const double* __restrict__ p;
  double beta;
  __device__ __forceinline__ double operator()(int64_t j) const { return fma(beta, __ldg(p + j), __ldg(z + j)); }
};
struct GatherDirection32 {
  const float* __restrict__ z;
  const float* __restrict__ p;
  float beta;
  __device__ __forceinline__ float operator()(int64_t j) const { return fmaf(beta, __ldg(p + j), __ldg(z + j)); }
};

template <int L, int U, typename V, typename I, typename G>
__device__ __forceinline__ void csr_rows_g(const int32_t* __restrict__ indptr, const I* __restrict__ cols,
                                           const V* __restrict__ vals, const G& gx, int64_t n, int64_t base, int lane,
                                           V (&s)[U], int64_t (&row)[U]) {
  constexpr int RPW = 32 / L;
  const int sub = lane % L;
  int32_t beg[U], end[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    row[u] = base + u * RPW + lane / L;
    const bool valid = row[u] < n;
    beg[u] = valid ? __ldg(indptr + row[u]) : 0;
    end[u] = valid ? __ldg(indptr + row[u] + 1) : 0;
  }
  V v[U];
  int64_t c[U];
  bool ok[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int32_t k = beg[u] + sub;
    ok[u] = k < end[u];
    v[u] = ok[u] ? __ldcs(vals + k) : V(0);
    c[u] = ok[u] ? col_at(cols, k, row[u]) : 0;
  }
#pragma unroll
  for (int u = 0; u < U; ++u) s[u] = ok[u] ? v[u] * gx(c[u]) : V(0);
#pragma unroll
  for (int u = 0; u < U; ++u)
    for (int32_t k = beg[u] + sub + L; k < end[u]; k += L) s[u] += __ldcs(vals + k) * gx(col_at(cols, k, row[u]));
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
}

template <int L, int U, typename V, typename I>
__device__ __forceinline__ void csr_rows(const int32_t* __restrict__ indptr, const I* __restrict__ cols,
                                         const V* __restrict__ vals, const V* __restrict__ x, int64_t n, int64_t base,
                                         int lane, V (&s)[U], int64_t (&row)[U]) {
  csr_rows_g<L, U, V, I>(indptr, cols, vals, GatherX<V>{x}, n, base, lane, s, row);
}

// ---------------------------------------------------------------------------------------------
// Sliced ELL (SELL-32): rows in slices of 32 (one warp), each slice padded to its longest row and
// stored column-major, entry k of row 32s+l at sell_ptr[s] + 32k + l. A thread owns a row: no
// row-pointer chase per row, no shuffles, and the loads of up to 8 entries are issued before any
// of them is used. Padding entries carry value 0 and the row's own column.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int32_t sell_col(const int32_t* __restrict__ cb, int32_t j, int32_t) { return __ldcs(cb + j); }
__device__ __forceinline__ int32_t sell_col(const int16_t* __restrict__ cb, int32_t j, int32_t row) {
  return row + (int32_t)__ldcs(cb + j);
}

// Row sum of one thread's row. vals/cols point at the row's first entry (slice base + lane);
// entry k sits at offset 32k. Index arithmetic is 32-bit (n < 2^31 is checked at plan build).
template <typename V, typename I, int B = 8, bool HINT = false, typename G>
__device__ __forceinline__ V sell_row(const V* __restrict__ vb, const I* __restrict__ cb, int32_t w, int32_t row,
                                      const G& gx) {
  V acc = V(0);
  uint64_t pol = 0;
  if (HINT) pol = l2_evict_first();
  for (int32_t k0 = 0; k0 < w; k0 += B) {
    V v[B];
    int32_t c[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const bool ok = k0 + u < w;
      const int32_t j = (k0 + u) * 32;
      if (HINT) {
        v[u] = ok ? ld_first(vb + j, pol) : V(0);
        c[u] = ok ? (sizeof(I) == 2 ? row + (int32_t)ld_first(cb + j, pol) : (int32_t)ld_first(cb + j, pol)) : row;
      } else {
        v[u] = ok ? __ldcs(vb + j) : V(0);
        c[u] = ok ? sell_col(cb, j, row) : row;
      }
    }
#pragma unroll
    for (int u = 0; u < B; ++u)
      if (k0 + u < w) acc += v[u] * gx(c[u]);
  }
  return acc;
}

// Call f(integral_constant<L>, integral_constant<U>) for a supported (lanes per row, rows in
// flight) pair; returns false for an unsupported one.
template <typename F>
inline bool with_spmv_cfg(int L, int U, F&& f) {
  using std::integral_constant;
#define FEMK_CFG(l, u)                                                  \
  if (L == l && U == u) {                                               \
    f(integral_constant<int, l>{}, integral_constant<int, u>{});        \
    return true;                                                        \
  }
  FEMK_CFG(4, 4)
  FEMK_CFG(8, 2)
  FEMK_CFG(8, 4)
  FEMK_CFG(16, 1)
  FEMK_CFG(16, 2)
  FEMK_CFG(16, 4)
  FEMK_CFG(32, 1)
  FEMK_CFG(32, 2)
#undef FEMK_CFG
  return false;
}

// Default (L, U) from the mean row length (a plan's csr_lanes / csr_rows options override it).
// Called once per plan.
void choose_spmv_cfg(double mean_row, int* L, int* U);

}  // namespace femk
