// Compact export of an assembled operator: the canonical CSR with its exact zeros dropped.
//
// On the non-parametric linear route the reference collapses the Dirichlet-eliminated triplets
// once with compress_eager (jno/utils/solver/fem_utils.py:4063-4091, called from
// fem_native.py:3371-3379): segment_sum over the compress plan, then keep the entries with
// abs(data) > 0 in plan order (rows ascending, columns ascending within a row). The plan of the
// eliminated triplets equals the plan's canonical pattern (every appended (d, d) pair is already
// a diagonal slot), so the compact operator is the canonical CSR filtered by |v| > 0: the zeroed
// Dirichlet rows and columns go, as do values that summed to exactly zero; NaN fails the test and
// is dropped too.
//
// Two passes over the values, half a warp per row (P1 rows hold 7-27 entries, P2 rows up to 65):
// count kept entries per row, exclusive scan of the counts, then write each kept (column, value)
// at its row offset plus its rank among the kept entries of the row (ballot + popc).
#include "femk_internal.cuh"

namespace femk {
namespace {

constexpr int kThreads = 256;
constexpr int kLanes = 16;  // lanes per row

struct HalfWarpRow {
  int64_t row;
  int32_t beg, len, maxlen;  // maxlen: the longer row of the two halves, so both run the same trips
  int sub, half;
};

__device__ __forceinline__ HalfWarpRow half_warp_row(const int32_t* __restrict__ indptr, int64_t row_pair, int64_t n) {
  HalfWarpRow h;
  const int lane = threadIdx.x & 31;
  h.sub = lane & (kLanes - 1);
  h.half = lane / kLanes;
  h.row = 2 * row_pair + h.half;
  h.beg = 0;
  h.len = 0;
  if (h.row < n) {
    h.beg = __ldg(indptr + h.row);
    h.len = __ldg(indptr + h.row + 1) - h.beg;
  }
  h.maxlen = max(h.len, __shfl_xor_sync(0xffffffffu, h.len, kLanes));
  return h;
}

// keep mask of this lane's half of the warp for entries [j, j + 16) of its row
__device__ __forceinline__ uint32_t half_ballot(bool keep, int half) {
  const uint32_t m = __ballot_sync(0xffffffffu, keep);
  return (m >> (kLanes * half)) & 0xffffu;
}

__global__ void __launch_bounds__(kThreads) k_compact_count(const int32_t* __restrict__ indptr,
                                                            const double* __restrict__ vals, int64_t n,
                                                            int64_t* __restrict__ count) {
  const int64_t pairs = (n + 1) / 2;
  const int64_t w0 = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  for (int64_t rp = w0; rp < pairs; rp += nw) {
    const HalfWarpRow h = half_warp_row(indptr, rp, n);
    int32_t c = 0;
    for (int32_t j = 0; j < h.maxlen; j += kLanes) {
      const bool in = j + h.sub < h.len;
      const bool keep = in && fabs(__ldcs(vals + h.beg + j + h.sub)) > 0.0;
      c += __popc(half_ballot(keep, h.half));
    }
    if (h.sub == 0 && h.row < n) count[h.row] = c;
  }
}

__global__ void __launch_bounds__(kThreads) k_compact_fill(const int32_t* __restrict__ indptr,
                                                           const int32_t* __restrict__ indices,
                                                           const double* __restrict__ vals, int64_t n,
                                                           const int64_t* __restrict__ offs,
                                                           int32_t* __restrict__ out_ptr,
                                                           int32_t* __restrict__ out_idx,
                                                           double* __restrict__ out_val) {
  const int64_t pairs = (n + 1) / 2;
  const int64_t w0 = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  if (blockIdx.x == 0 && threadIdx.x == 0) out_ptr[n] = (int32_t)offs[n];
  for (int64_t rp = w0; rp < pairs; rp += nw) {
    const HalfWarpRow h = half_warp_row(indptr, rp, n);
    int64_t o = h.row < n ? __ldg(offs + h.row) : 0;
    if (h.sub == 0 && h.row < n) out_ptr[h.row] = (int32_t)o;
    const uint32_t below = (1u << h.sub) - 1u;
    for (int32_t j = 0; j < h.maxlen; j += kLanes) {
      const bool in = j + h.sub < h.len;
      const int32_t k = h.beg + j + h.sub;
      const double v = in ? __ldcs(vals + k) : 0.0;
      const bool keep = in && fabs(v) > 0.0;
      const uint32_t m = half_ballot(keep, h.half);
      if (keep) {
        const int64_t pos = o + __popc(m & below);
        out_idx[pos] = __ldcs(indices + k);
        out_val[pos] = v;
      }
      o += __popc(m);
    }
  }
}

}  // namespace
}  // namespace femk

extern "C" int femk_compact(const femk_plan* p, const double* vals, int32_t* indptr_out, int32_t* indices_out,
                            double* vals_out, int64_t cap, int64_t* nnz_out, void* stream) {
  using namespace femk;
  clear_error();
  FEMK_CHECK_ARG(p, "femk_compact: plan is NULL");
  FEMK_CHECK_ARG(vals && indptr_out && nnz_out, "femk_compact: vals, indptr_out and nnz_out are required");
  FEMK_CHECK_ARG(cap >= 0, "femk_compact: cap must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  // plan-owned scratch (allocated on the first call): a per-call stream-ordered allocation went back
  // to the driver at the count read's synchronize, and its cost varied between calls
  femk_plan* pm = const_cast<femk_plan*>(p);
  if (!pm->cmp_ws) {
    const cudaError_t ea = cudaMalloc(&pm->cmp_ws, sizeof(int64_t) * (2 * p->n + 2));
    if (ea != cudaSuccess) {
      pm->cmp_ws = nullptr;
      set_error(std::string("femk_compact: ") + cudaGetErrorString(ea));
      return ea == cudaErrorMemoryAllocation ? FEMK_ENOMEM : FEMK_ECUDA;
    }
  }
  int64_t* count = pm->cmp_ws;
  int64_t* offs = pm->cmp_ws + (p->n > 0 ? p->n : 1);
  cudaError_t e = cudaSuccess;
  int st = FEMK_OK;
  const int64_t pairs = (p->n + 1) / 2;
  const int grid = blocks_for(pairs * 32, kThreads, p->n_sm * 8);
  int64_t total = 0;
  if (p->n > 0) {
    k_compact_count<<<counted_launch() + grid, kThreads, 0, s>>>(p->indptr, vals, p->n, count);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("femk_compact count: ") + cudaGetErrorString(e));
      st = FEMK_ECUDA;
    }
  }
  if (st == FEMK_OK) st = scan_exclusive_i64(count, offs, p->n, s);
  if (st == FEMK_OK) {
    e = cudaMemcpyAsync(&total, offs + p->n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error(std::string("femk_compact: reading the count: ") + cudaGetErrorString(e));
      st = FEMK_ECUDA;
    }
  }
  if (st == FEMK_OK && total > cap) {
    set_error("femk_compact: " + std::to_string(total) + " entries kept, more than cap = " + std::to_string(cap));
    st = FEMK_EINVAL;
  }
  if (st == FEMK_OK && total > 0 && !(indices_out && vals_out)) {
    set_error("femk_compact: indices_out and vals_out are required when entries are kept");
    st = FEMK_EINVAL;
  }
  if (st == FEMK_OK) {
    *nnz_out = total;
    k_compact_fill<<<counted_launch() + grid, kThreads, 0, s>>>(p->indptr, p->indices, vals, p->n, offs, indptr_out,
                                                                indices_out, vals_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("femk_compact fill: ") + cudaGetErrorString(e));
      st = FEMK_ECUDA;
    }
  }
  return st;
}
