// Sliced-ELL SpMV with the matrix streamed into shared memory by the bulk-copy (TMA) engine.
//
// The thread-per-row SELL kernel issues every matrix load itself and then gathers x through the
// columns it loaded: two dependent round trips per slice, so a warp has DRAM bytes in flight only
// during the first. Here each warp keeps a ring of S slice buffers in shared memory: lane 0 issues
// one cp.async.bulk for a slice's values and one for its columns (completion counted in bytes on
// the stage's mbarrier) S slices ahead of the slice the warp computes, so the copy engine keeps the
// next slices' bytes in flight while the lanes gather and accumulate the current one.
//
// Slice layout (unchanged from the SELL-32 operator): slice s holds entries [sptr[s], sptr[s+1]),
// column-major, entry k of row 32s + l at sptr[s] + 32k + l; the width w = (sptr[s+1]-sptr[s])/32
// must be <= WMAX. Values start 256-byte and columns 64-byte aligned (sptr is a multiple of 32),
// and both byte counts are multiples of 16, as cp.async.bulk requires.
//
// Row sums are accumulated in k order exactly as sell_row does (acc += v_k * x[c_k]), so a row's
// result is bit-identical to the register-streaming kernel's.
//
// Waits are bounded: a stage that does not complete within kBulkSpinCycles sets *err and the warp
// stops issuing; before returning it waits (bounded again) for the copies it has in flight, so no
// copy lands in shared memory after the block has exited.
#pragma once

#include <stdint.h>

#include <type_traits>

#include "femk_l2.cuh"
#include "femk_spmv.cuh"

namespace femk {

constexpr long long kBulkSpinCycles = 2000000000LL;  // about one second at the B200 boost clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// try_wait that lets the hardware suspend the thread until the phase completes (or the hint, in
// nanoseconds, elapses) instead of returning at once: waiting warps stop taking issue slots
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
      : "memory");
  return done != 0;
}

// bounded wait for the phase with the given parity to complete; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait_suspend(bar, parity)) {
    if (clock64() - t0 > kBulkSpinCycles) return false;
  }
  return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ void bulk_g2s_plain(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Where the copies of one slice come from: values at vals + b0 (32 w entries), columns at cols + c0
// (cn entries; cn < 32 w marks a shared-offset table).
struct SliceDir {
  int64_t b0, c0;
  int32_t w, cn;
};

// Shared memory one warp needs: S mbarriers + S widths (128 B), a directory of the
// warp's next kDir slices, then S stages of [32*WMAX values][32*WMAX columns].
template <typename V, typename IDX, int WMAX, int S>
struct BulkRing {
  static constexpr int kVal = 32 * WMAX * (int)sizeof(V);
  static constexpr int kCol = ((32 * WMAX * (int)sizeof(IDX)) + 127) / 128 * 128;
  static constexpr int kStage = kVal + kCol;
  static constexpr int kDir = 16;
  static constexpr int kHead = 128 + (kDir * (int)sizeof(SliceDir) + 127) / 128 * 128;
  static constexpr int kWarpBytes = kHead + S * kStage;
  static_assert(S * 16 <= 128, "ring header too small");
  static_assert(S < kDir, "the directory must cover the slices issued ahead");
  static_assert(kVal % 128 == 0 && kHead % 128 == 0, "stage alignment");
};

// Bounded warp-wide wait for the phase with the given parity: every lane polls (one warp
// instruction whether one lane or all poll) and so observes the completed phase itself, which is
// what makes the bulk-copy writes visible to it. Returns the same outcome in every lane.
__device__ __forceinline__ bool mbar_wait_all(uint64_t* bar, uint32_t parity) {
  bool ok = mbar_try_wait(bar, parity);
  if (!__all_sync(0xffffffffu, ok)) {
    const long long t0 = clock64();
    while (!(ok = mbar_try_wait_suspend(bar, parity)))
      if (clock64() - t0 > kBulkSpinCycles) break;
  }
  return __all_sync(0xffffffffu, ok);
}

// Every slice of this warp (global warp g takes slices g, g + NW, ...): for each row,
// epi(row, row_sum). Returns false if a wait timed out (and sets *err to errval). Rows and slices
// fit in 32 bits (the plan's column indices are int32), so the loop runs on 32-bit indices.
//
// cptr == NULL: cols holds one column (or offset) per stored entry, like vals. cptr != NULL: cols is
// the per-slice column table (int16 offsets): slice s's table starts at cptr[s] and holds either w
// offsets shared by all 32 rows (padded to 8) or the 32*w per-entry offsets.
template <typename V, typename IDX, int WMAX, int S, typename G, typename Epi>
__device__ __forceinline__ bool sell_bulk_rows(unsigned char* wsmem, const int64_t* __restrict__ sptr,
                                               const IDX* __restrict__ cols, const V* __restrict__ vals, int64_t n,
                                               int64_t nslices64, int64_t g64, int64_t NW64, const G& gx, Epi&& epi,
                                               int* err, int errval, const int64_t* __restrict__ cptr = nullptr) {
  using R = BulkRing<V, IDX, WMAX, S>;
  const int lane = threadIdx.x & 31;
  const int32_t nslices = (int32_t)nslices64, g = (int32_t)g64, NW = (int32_t)NW64;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsmem);
  int32_t* wid = reinterpret_cast<int32_t*>(wsmem + 8 * S);  // slice width per stage; negative: shared offsets
  SliceDir* dir = reinterpret_cast<SliceDir*>(wsmem + 128);
  unsigned char* stages = wsmem + R::kHead;
  uint64_t pol = 0;
  if (lane == 0) {
    pol = l2_evict_first();
    for (int s = 0; s < S; ++s) mbar_init(bar + s, 1);
    mbar_fence_init();
  }
  // All lanes: the directory entries of this warp's slices with ordinals [base, base + kDir) (the
  // slice of ordinal j is g + j NW), one slice per lane, so the offsets of kDir slices cost one round
  // trip instead of one dependent load per slice on lane 0's refill path.
  int32_t dbase = 0;
  auto fill_dir = [&](int32_t base) {
    if (lane < R::kDir) {
      const int32_t sl = g + (base + lane) * NW;
      if (sl < nslices) {
        const int64_t b0 = __ldg(sptr + sl);
        const int32_t w = (int32_t)((__ldg(sptr + sl + 1) - b0) >> 5);
        int64_t c0 = b0;
        int32_t cn = 32 * w;
        if (cptr) {
          c0 = __ldg(cptr + sl);
          cn = (int32_t)(__ldg(cptr + sl + 1) - c0);
        }
        dir[lane] = SliceDir{b0, c0, w, cn};
      }
    }
    __syncwarp();
  };
  fill_dir(0);
  // lane 0: stream the slice of ordinal j (in the directory) into stage `s`
  auto issue = [&](int32_t j, int s) {
    const SliceDir d = dir[j - dbase];
    wid[s] = d.cn == 32 * d.w ? d.w : -d.w;
    const uint32_t vb = (uint32_t)(32 * d.w * (int)sizeof(V));
    const uint32_t cb = (uint32_t)(d.cn * (int)sizeof(IDX));
    unsigned char* st = stages + s * R::kStage;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar + s, vb + cb);  // with w == 0 this arrival alone completes the phase
    if (d.w > 0) {
      bulk_g2s(st, vals + d.b0, vb, bar + s, pol);
      bulk_g2s(st + R::kVal, cols + d.c0, cb, bar + s, pol);
    }
  };
  int32_t issued = 0;  // slices issued so far (lane 0's count; ordinal j lives in stage j % S)
  if (lane == 0)
    for (int s = 0; s < S; ++s) {
      if (g + s * NW >= nslices) break;
      issue(s, s);
      ++issued;
    }
  __syncwarp();
  bool ok = true;
  int32_t j = 0;
  for (int32_t sl = g; sl < nslices; sl += NW, ++j) {
    const int s = j % S;
    const uint32_t parity = (uint32_t)((j / S) & 1);
    // warp-uniform outcome: a timed-out wait takes the whole warp out of the loop
    if (!mbar_wait_all(bar + s, parity)) {
      ok = false;
      break;
    }
    const int32_t ws = wid[s];
    const int32_t w = ws < 0 ? -ws : ws;
    const V* sv = reinterpret_cast<const V*>(stages + s * R::kStage) + lane;
    const IDX* sc = reinterpret_cast<const IDX*>(stages + s * R::kStage + R::kVal);
    const int32_t row = sl * 32 + lane;
    const bool live = row < n;  // rows past n in the last slice gather nothing
    V acc = V(0);
    // Row sum in k order. The common widths (WMAX, WMAX - 1) run without per-entry predicates, and
    // the shared-offset and per-entry column layouts each get compile-time strides, so an entry costs
    // a shared load of its column, the gather, a shared load of its value and one FMA.
    auto run = [&](auto KC, auto UC) {
      constexpr int K = decltype(KC)::value;
      constexpr bool U = decltype(UC)::value;
      const IDX* cb = U ? sc : sc + lane;
      V xg[K];
      if constexpr (U && sizeof(IDX) == 2 && sizeof(V) == 4) {
        // FP32 rows, shared offsets: broadcast 16-byte loads of 8 offsets each (the table is padded
        // to 8, and the stage's column area starts 128-byte aligned). Measured on one B200 at P1
        // 128^3: the mixed solve 25.87 -> 25.24 ms, while the same loads slowed the FP64 solve
        // 35.78 -> 38.51 ms, so FP64 rows keep the per-entry loads.
        constexpr int NQ = (K + 7) / 8;
        int4 cq[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) cq[q] = reinterpret_cast<const int4*>(sc)[q];
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int4 q4 = cq[k / 8];
          const int w2 = (k % 8) / 2;
          const int32_t word = w2 == 0 ? q4.x : (w2 == 1 ? q4.y : (w2 == 2 ? q4.z : q4.w));
          const int32_t c = (k & 1) ? (word >> 16) : (int32_t)(int16_t)(word & 0xffff);
          xg[k] = gx(row + c);
        }
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const IDX c = cb[U ? k : k * 32];
          xg[k] = gx(sizeof(IDX) == 2 ? row + (int32_t)c : (int32_t)c);
        }
      }
#pragma unroll
      for (int k = 0; k < K; ++k) acc += sv[k * 32] * xg[k];
    };
    if (live) {
      using std::integral_constant;
      const bool u = ws < 0;
      if (w == WMAX) {
        u ? run(integral_constant<int, WMAX>{}, std::true_type{}) : run(integral_constant<int, WMAX>{}, std::false_type{});
      } else if (w == WMAX - 1) {
        u ? run(integral_constant<int, WMAX - 1>{}, std::true_type{})
          : run(integral_constant<int, WMAX - 1>{}, std::false_type{});
      } else {
        const int cstride = u ? 1 : 32;  // shared offsets: every lane reads entry k (a broadcast)
        const int clane = u ? 0 : lane;
        V xg[WMAX];
#pragma unroll
        for (int k = 0; k < WMAX; ++k) {
          if (k < w) {
            const IDX c = sc[k * cstride + clane];
            xg[k] = gx(sizeof(IDX) == 2 ? row + (int32_t)c : (int32_t)c);
          }
        }
#pragma unroll
        for (int k = 0; k < WMAX; ++k)
          if (k < w) acc += sv[k * 32] * xg[k];
      }
    }
    __syncwarp();  // every lane is done with stage s before it is refilled
    const int32_t nj = j + S;  // next ordinal to issue (every smaller one is issued)
    if (g + nj * NW < nslices) {
      if (nj >= dbase + R::kDir) {  // warp-uniform: the directory moves on to [nj, nj + kDir)
        dbase = nj;
        fill_dir(dbase);
      }
      if (lane == 0) {
        issue(nj, s);
        ++issued;
      }
    }
    __syncwarp();
    if (live) epi((int64_t)row, acc);
  }
  if (!ok) {
    if (lane == 0) {
      atomicExch(err, errval);
      // drain: wait (bounded) for every copy this warp still has in flight
      for (int32_t q = j; q < issued; ++q) mbar_wait(bar + (q % S), (uint32_t)((q / S) & 1));
    }
    __syncwarp();
  }
  return ok;
}

}  // namespace femk
