// Sliced-ELL SpMV with both the matrix and the x values it reads staged in shared memory.
//
// A tile is W consecutive 32-row slices (one per warp of the CTA). The plan records, per tile, the
// few contiguous windows of x that hold every column the tile's rows touch (a structured-mesh tile
// reads three: the plane below, its own plane and the plane above) and rewrites every column as a
// slot in the tile's staged x buffer: per slice either one slot sequence shared by all 32 rows
// (slot of lane l = table[k] + l) or 32*w per-entry slots, in the layout of the per-slice column
// tables. One thread per CTA streams a tile's values, its slot table and its x windows into a
// shared-memory stage with cp.async.bulk (completion on the stage's mbarrier) while the warps
// compute the previous tile from shared memory alone: no global gathers are left on the critical
// path. Rows sum in k order like sell_row, so row sums are bit-identical to the other SELL kernels.
//
// Waits are bounded (kBulkSpinCycles): a stage that never completes sets *err, and thread 0 waits
// (bounded again) for its copies in flight before the CTA exits.
#pragma once

#include <stdint.h>

#include "femk_bulk.cuh"

namespace femk {

constexpr int kTileMaxWin = 10;  // x windows per tile

struct TileMeta {  // 128 bytes per tile, built with the plan
  int64_t v0, v1;  // the tile's value entries [v0, v1) (sell_ptr of its first and one-past-last slice)
  int64_t c0, c1;  // its slot-table entries [c0, c1)
  int32_t nwin;    // x windows
  int32_t xlen;    // staged x elements (sum of window lengths)
  int32_t self_base;  // slot of row r = r + self_base (the window holding the tile's own rows)
  int32_t pad;
  int32_t wstart[kTileMaxWin];  // window starts (multiples of 4 elements)
  int32_t wlen[kTileMaxWin];    // window lengths (multiples of 4 elements)
};
static_assert(sizeof(TileMeta) == 128, "TileMeta layout");

// Shared-memory stage of one tile: values, slot table, staged x. All three start 128-B aligned.
template <typename V, int W, int WMAX>
struct TileStage {
  static constexpr int kVal = W * 32 * WMAX * (int)sizeof(V);
  static constexpr int kTab = (W * 32 * WMAX * 2 + 127) / 128 * 128;
  static __host__ __device__ int bytes(int xcap) { return kVal + kTab + (xcap * (int)sizeof(V) + 127) / 128 * 128; }
};

// Every tile of this CTA (tiles blockIdx.x, blockIdx.x + gridDim.x, ...): for each row,
// epi(row, row_sum, x[row]). Returns false if a wait timed out (and sets *err to errval).
// smem: 2 stages of TileStage::bytes(xcap) followed by 2 mbarriers.
template <typename V, int W, int WMAX, typename Epi>
__device__ __forceinline__ bool sell_tile_rows(unsigned char* smem, int xcap, const TileMeta* __restrict__ meta,
                                               int64_t ntiles, const int64_t* __restrict__ sptr,
                                               const int64_t* __restrict__ cptr, const int16_t* __restrict__ slots,
                                               const V* __restrict__ vals, const V* __restrict__ x, int64_t n,
                                               int64_t nslices, Epi&& epi, int* err, int errval) {
  using TS = TileStage<V, W, WMAX>;
  const int stage_bytes = TS::bytes(xcap);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * stage_bytes);
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  uint64_t pol = 0;
  if (tid == 0) {
    pol = l2_evict_first();
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_fence_init();
  }
  __syncthreads();
  // thread 0: stream tile t into stage s (values, slot table, x windows; one transaction count)
  auto issue = [&](int64_t t, int s) {
    const TileMeta& m = meta[t];
    const int64_t v0 = m.v0, v1 = m.v1, c0 = m.c0, c1 = m.c1;
    const int nwin = m.nwin;
    unsigned char* st = smem + s * stage_bytes;
    const uint32_t vb = (uint32_t)((v1 - v0) * (int64_t)sizeof(V));
    const uint32_t cb = (uint32_t)((c1 - c0) * 2);
    uint32_t xb = 0;
    for (int j = 0; j < nwin; ++j) xb += (uint32_t)(m.wlen[j] * (int)sizeof(V));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar + s, vb + cb + xb);
    if (vb) bulk_g2s(st, vals + v0, vb, bar + s, pol);
    if (cb) bulk_g2s(st + TS::kVal, slots + c0, cb, bar + s, pol);
    unsigned char* xs = st + TS::kVal + TS::kTab;
    for (int j = 0; j < nwin; ++j) {
      const uint32_t b = (uint32_t)(m.wlen[j] * (int)sizeof(V));
      bulk_g2s_plain(xs, x + m.wstart[j], b, bar + s);  // x is reused by other tiles: no evict-first hint
      xs += b;
    }
  };
  int64_t issued = 0;  // thread 0's count of tiles issued (tile i of this CTA lives in stage i & 1)
  if (tid == 0)
    for (int s = 0; s < 2; ++s) {
      const int64_t t = blockIdx.x + (int64_t)s * gridDim.x;
      if (t >= ntiles) break;
      issue(t, s);
      ++issued;
    }
  bool ok = true;
  int64_t i = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
    const int s = (int)(i & 1);
    // this warp's slice: offsets and width from global memory, loaded before the stage wait
    const int64_t sl = t * W + wib;
    const bool have = sl < nslices;
    int64_t sb = 0, se = 0, cb0 = 0, ce = 0, mv0 = 0, mc0 = 0;
    int32_t self_base = 0;
    if (have) {
      sb = __ldg(sptr + sl);
      se = __ldg(sptr + sl + 1);
      cb0 = __ldg(cptr + sl);
      ce = __ldg(cptr + sl + 1);
      mv0 = __ldg(&meta[t].v0);
      mc0 = __ldg(&meta[t].c0);
      self_base = __ldg(&meta[t].self_base);
    }
    const bool done = mbar_wait(bar + s, (uint32_t)((i >> 1) & 1));
    if (!__syncthreads_and(done)) {
      ok = false;
      break;
    }
    const unsigned char* st = smem + s * stage_bytes;
    if (have) {
      const int32_t w = (int32_t)((se - sb) >> 5);
      const bool uni = (ce - cb0) != 32 * (int64_t)w;
      const V* sv = reinterpret_cast<const V*>(st) + (sb - mv0);
      const int16_t* sc = reinterpret_cast<const int16_t*>(st + TS::kVal) + (cb0 - mc0);
      const V* xs = reinterpret_cast<const V*>(st + TS::kVal + TS::kTab);
      const int64_t row = sl * 32 + lane;
      V acc = V(0);
      if (row < n) {
#pragma unroll
        for (int k = 0; k < WMAX; ++k)
          if (k < w) {
            const int c = uni ? (int)sc[k] + lane : (int)sc[k * 32 + lane];
            acc += sv[k * 32 + lane] * xs[c];
          }
        epi(row, acc, xs[row + self_base]);
      }
    }
    __syncthreads();  // every warp is done with stage s before it is refilled
    if (tid == 0) {
      const int64_t nt = t + 2 * (int64_t)gridDim.x;
      if (nt < ntiles) {
        issue(nt, s);
        ++issued;
      }
    }
  }
  if (!ok && tid == 0) {
    atomicExch(err, errval);
    for (int64_t j = i; j < issued; ++j) mbar_wait(bar + (int)(j & 1), (uint32_t)((j >> 1) & 1));
  }
  __syncthreads();
  return ok;
}

}  // namespace femk
